// Guard of a captured collide graph.  A PIC collide's launch schedule -- the pairs of each wavefront and their
// tasks, planes and luminosity jobs -- is a function of the wavefront batching of the collision order and of
// which slices are empty (slicing.jl:561-647, pic_cpu.jl:82-275); everything else the host derives from the
// slice tables -- slice starts and counts, the fixed-point scales, the drifts, the kick's block map -- is data
// in device tables, and every kernel's result is independent of how its particles are split over blocks
// (fixed-point deposits, extrema, per-particle kicks).  So a graph captured from one collide is the next
// collide's graph whenever the batching and the empty slices agree and the next collide's slices fit the
// capacity the capture left: this kernel checks exactly that on the device, rewrites the device tables with the
// host's expressions, and opens the graph's conditional body.  When anything differs it leaves the body closed
// and the host runs the ordinary path on the untouched beams.
#pragma once
#include <cuda_runtime.h>

#include "k_slicing.cuh"
#include "octo_internal.cuh"

namespace octo {

constexpr int kReplayMaxPairs = 1024;  // slice pairs a guarded graph may hold (the guard's shared tables)

struct ReplayCheck {
    const SliceInfo *info[2];  // the device slice tables of this collide
    const long long *sig;      // count > 0 for the ns1 then the ns2 slices, then per pair index (i-1)*ns2 + (j-1)
                               // its wavefront and its place in it (front * 65536 + place), all of the captured
                               // collide
    int ns1, ns2;
    int fp32;                  // the precision form's fixed-point scale
    const FrontKick *fronts;   // per wavefront of the graph: its tasks and block map entries
    int nfronts;
    int2 *blockmap;
    long long node_cap;        // :node: the largest slice the captured node-box chunking covers
    long long *node_counts;    // :node: the slice counts k_node_plan reads (null otherwise)
    Task *tasks;
    int ntasks;
    Plane *planes;
    int nplanes;
    LumJob *lumjobs;
    int nlum;
    FirstLum *first;
    int nfirst;
    double *node_ref;          // :node drift references (null otherwise), the host's staging layout
    int *ok;                   // 1: body opened, 0: the schedule differs
    cudaGraphConditionalHandle handle;
};

// One block of 1024 threads.  The schedule is the wavefront batching of the collision order (slicing.jl:601-647):
// its greedy rounds take, in collision order, every pair that is the next pending pair of both its slices, which
// puts each pair in the wavefront one past the later of the previous pairs of its two slices -- so the fronts
// follow from the order in one sequential pass.  The graph's kernels depend on that batching and on the slice
// counts and starts, not on the order itself (a pair's place in it only names the slot its luminosity is stored
// in; the host folds the slots in this collide's order).
__global__ void __launch_bounds__(1024) k_replay_check(ReplayCheck A) {
    __shared__ int bad;
    __shared__ double tpair[kReplayMaxPairs];  // collision times, then reused as the order and the fronts
    __shared__ int rk[kReplayMaxPairs];
    __shared__ int last[2][kMaxSlices];
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    const SliceInfo &S1 = *A.info[0], &S2 = *A.info[1];
    const int ns1 = A.ns1, ns2 = A.ns2, np = ns1 * ns2;
    const bool fits = ns1 >= 1 && ns2 >= 1 && ns1 <= kMaxSlices && ns2 <= kMaxSlices && np <= kReplayMaxPairs;
    if (threadIdx.x == 0 && (!fits || S1.ns != ns1 || S2.ns != ns2 || S1.nonfinite || S2.nonfinite)) bad = 1;
    __syncthreads();
    if (bad) {
        if (threadIdx.x == 0) *A.ok = 0;
        return;
    }
    for (int k = threadIdx.x; k < ns1; k += blockDim.x)
        if ((S1.count[k] > 0) != (A.sig[k] != 0)) bad = 1;
    for (int k = threadIdx.x; k < ns2; k += blockDim.x)
        if ((S2.count[k] > 0) != (A.sig[ns1 + k] != 0)) bad = 1;
    // the stable sort by collision time -(c1 + c2)/2 (slicing.jl:561-568): the rank of every pair
    for (int p = threadIdx.x; p < np; p += blockDim.x) tpair[p] = -(S1.center[p / ns2] + S2.center[p % ns2]) / 2;
    __syncthreads();
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const double tp = tpair[p];
        int rank = 0;
        for (int q = 0; q < np; ++q) {
            const double tq = tpair[q];
            rank += (tq < tp) || (tq == tp && q < p);
        }
        rk[p] = rank;
    }
    __syncthreads();
    int *ord = reinterpret_cast<int *>(tpair);  // rank -> pair
    int *front = ord + kReplayMaxPairs;         // pair -> wavefront
    for (int p = threadIdx.x; p < np; p += blockDim.x) ord[rk[p]] = p;
    for (int k = threadIdx.x; k < 2 * kMaxSlices; k += blockDim.x) last[k / kMaxSlices][k % kMaxSlices] = 0;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int r = 0; r < np; ++r) {
            const int p = ord[r], i = p / ns2, j = p % ns2;
            const int f = max(last[0][i], last[1][j]) + 1;
            front[p] = f - 1;
            last[0][i] = f;
            last[1][j] = f;
        }
    __syncthreads();
    const long long *code = A.sig + ns1 + ns2;
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        int place = 0;
        for (int q = 0; q < np; ++q) place += front[q] == front[p] && rk[q] < rk[p];
        if (code[p] != (long long)front[p] * 65536 + place) bad = 1;
    }
    __syncthreads();
    if (bad) {
        if (threadIdx.x == 0) *A.ok = 0;
        return;  // the conditional keeps its default, 0
    }
    // the task ranges and drifts, as CollideJob::run computes them (pic_cpu.jl:954-1003, 1540-1548)
    for (int t = threadIdx.x; t < A.ntasks; t += blockDim.x) {
        Task &T = A.tasks[t];
        const SliceInfo &SS = T.dir == 1 ? S1 : S2, &SF = T.dir == 1 ? S2 : S1;
        const int ss = T.dir == 1 ? T.i - 1 : T.j - 1, sf = T.dir == 1 ? T.j - 1 : T.i - 1;
        T.src_start = SS.start[ss];
        T.src_n = SS.count[ss];
        T.fld_start = SF.start[sf];
        T.fld_n = SF.count[sf];
        T.c_src = SS.center[ss];
        T.c_fld = SF.center[sf];
        T.lb_fld = SF.boundary[sf];
        T.rb_fld = SF.boundary[sf + 1];
        T.sL = 0.5 * (T.c_src - T.lb_fld);
        T.sR = 0.5 * (T.c_src - T.rb_fld);
        T.sM = 0.5 * (T.c_src - T.c_fld);
        const double denom = T.rb_fld - T.lb_fld;
        if (!isfinite(denom) || denom == 0.0) { T.hzi = 0.0; T.zbias = 0.5; }
        else { T.hzi = 1.0 / denom; T.zbias = T.rb_fld * T.hzi; }
    }
    // luminosity job k belongs to the pair of tasks 2k (direction 1) and 2k + 1
    for (int k = threadIdx.x; k < A.nlum; k += blockDim.x) {
        const Task &T = A.tasks[2 * k];
        LumJob &J = A.lumjobs[k];
        J.s1_start = S1.start[T.i - 1];
        J.s1_n = S1.count[T.i - 1];
        J.s2_start = S2.start[T.j - 1];
        J.s2_n = S2.count[T.j - 1];
        J.bits1 = A.fp32 ? fixed_bits_for32(J.s1_n) : fixed_bits_for(J.s1_n);
        J.bits2 = A.fp32 ? fixed_bits_for32(J.s2_n) : fixed_bits_for(J.s2_n);
        J.sM1 = 0.5 * (S1.center[T.i - 1] - S2.center[T.j - 1]);
        J.sM2 = 0.5 * (S2.center[T.j - 1] - S1.center[T.i - 1]);
    }
    if (A.node_counts) {  // k_node_plan's counts, and the captured node-box chunking must still cover them
        for (int k = threadIdx.x; k < ns1 + ns2; k += blockDim.x) {
            const long long n = k < ns1 ? S1.count[k] : S2.count[k - ns1];
            A.node_counts[k] = n;
            if (n > A.node_cap) bad = 1;
        }
    }
    if (A.node_ref) {  // build_node_meshes' staging: per beam, per slice, o + 1 node drifts then o centres
        const int nref1 = 2 * ns2 + 1, nref2 = 2 * ns1 + 1;
        const int tot = ns1 * nref1 + ns2 * nref2;
        for (int k = threadIdx.x; k < tot; k += blockDim.x) {
            const int bm = k < ns1 * nref1 ? 0 : 1;
            const int r = bm ? k - ns1 * nref1 : k;
            const int nref = bm ? nref2 : nref1, o = bm ? ns1 : ns2;
            const SliceInfo &SS = bm ? S2 : S1, &SO = bm ? S1 : S2;
            const int sl = r / nref, b = r % nref;
            A.node_ref[k] = b <= o ? 0.5 * (SS.center[sl] - SO.boundary[b]) : SO.center[b - o - 1];
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < A.nplanes; k += blockDim.x) {
        Plane &P = A.planes[k];
        const Task &T = A.tasks[P.task];
        P.src_start = T.src_start;
        P.src_n = T.src_n;
        P.fixed_bits = A.fp32 ? fixed_bits_for32(T.src_n) : fixed_bits_for(T.src_n);
        // kinds: 0 L (sL), 1 R (sR), 2 M (midpoint), 3 Z (:node, the R drift)
        P.s = P.kind == 0 ? T.sL : (P.kind == 2 ? 0.5 * (T.sL + T.sR) : T.sR);
    }
    for (int k = threadIdx.x; k < A.nfirst; k += blockDim.x) {
        FirstLum &F = A.first[k];
        const LumJob &J = A.lumjobs[F.task / 2];
        F.start = F.beam == 0 ? J.s1_start : J.s2_start;
        F.count = F.beam == 0 ? J.s1_n : J.s2_n;
        F.sM = F.beam == 0 ? J.sM1 : J.sM2;
    }
    // :node with luminosity: the drift at which each kick reduces its field slice for that slice's next pair
    for (int t = threadIdx.x; t < A.ntasks; t += blockDim.x) {
        Task &T = A.tasks[t];
        if (T.next_task < 0) continue;
        const LumJob &J = A.lumjobs[T.next_task / 2];
        T.next_sM = T.fld_beam == 0 ? J.sM1 : J.sM2;
    }
    // each wavefront's kick blocks of kchunk field particles (CollideJob::run's block map), then spare entries
    // (task -1) up to the map's room; a front whose blocks no longer fit closes the body.  Tasks of a front are
    // consecutive: each task's block count in parallel, a prefix per front, then every task writes its blocks.
    __shared__ int tfront[2 * kReplayMaxPairs], tcount[2 * kReplayMaxPairs], tbase[2 * kReplayMaxPairs];
    __shared__ int fcount[kReplayMaxPairs];
    const bool maps_fit = A.ntasks <= 2 * kReplayMaxPairs && A.nfronts <= kReplayMaxPairs;
    if (!maps_fit) bad = 1;
    if (maps_fit) {
        for (int f = threadIdx.x; f < A.nfronts; f += blockDim.x)
            for (int t = A.fronts[f].t0; t < A.fronts[f].t0 + A.fronts[f].nt; ++t) tfront[t] = f;
        __syncthreads();
        for (int t = threadIdx.x; t < A.ntasks; t += blockDim.x) {
            const long long kc = A.fronts[tfront[t]].kchunk;
            tcount[t] = (int)((A.tasks[t].fld_n + kc - 1) / kc);
        }
        __syncthreads();
        for (int f = threadIdx.x; f < A.nfronts; f += blockDim.x) {
            const FrontKick F = A.fronts[f];
            int k = 0;
            for (int t = F.t0; t < F.t0 + F.nt; ++t) { tbase[t] = k; k += tcount[t]; }
            fcount[f] = k;
            if (k > F.cap) bad = 1;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < A.ntasks; t += blockDim.x) {
            const int f = tfront[t];
            const FrontKick F = A.fronts[f];
            if (fcount[f] > F.cap) continue;
            for (int q = 0; q < tcount[t]; ++q)
                A.blockmap[F.b0 + tbase[t] + q] = make_int2(t, (int)((long long)q * F.kchunk));
        }
        for (int f = threadIdx.x; f < A.nfronts; f += blockDim.x) {
            const FrontKick F = A.fronts[f];
            for (int k = fcount[f]; k < F.cap; ++k) A.blockmap[F.b0 + k] = make_int2(-1, 0);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *A.ok = bad ? 0 : 1;
        if (!bad) cudaGraphSetConditional(A.handle, 1u);
    }
}

}  // namespace octo
