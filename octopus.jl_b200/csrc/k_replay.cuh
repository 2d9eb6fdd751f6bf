// Guard of a captured collide graph.  A PIC collide's launch schedule -- the pairs of each wavefront, the
// tasks, planes and luminosity jobs, every grid size -- is a function of the slice counts and starts and of
// the collision order alone (slicing.jl:561-647, pic_cpu.jl:82-275); the drifts the host derives from the
// slice centres and boundaries are the only other inputs it uploads.  When a collide's slicing reproduces
// the counts, starts and order of the collide the graph was captured from, the graph's kernels are that
// collide's kernels: this kernel checks exactly that on the device, recomputes the drifts into the resident
// task tables with the host's expressions, and opens the graph's conditional body.  When anything differs it
// leaves the body closed and the host runs the ordinary path on the untouched beams.
#pragma once
#include <cuda_runtime.h>

#include "k_slicing.cuh"
#include "octo_internal.cuh"

namespace octo {

struct ReplayCheck {
    const SliceInfo *info[2];  // the device slice tables of this collide
    const long long *sig;      // count[ns1], start[ns1], count[ns2], start[ns2], then the collision order as pair
                               // indices (i-1)*ns2 + (j-1), all of the captured collide
    int ns1, ns2;
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

// One block of 1024 threads: the tables hold at most a few thousand entries.
__global__ void __launch_bounds__(1024) k_replay_check(ReplayCheck A) {
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    const SliceInfo &S1 = *A.info[0], &S2 = *A.info[1];
    const int ns1 = A.ns1, ns2 = A.ns2, np = ns1 * ns2;
    if (threadIdx.x == 0 && (S1.ns != ns1 || S2.ns != ns2 || S1.nonfinite || S2.nonfinite)) bad = 1;
    for (int k = threadIdx.x; k < ns1; k += blockDim.x)
        if (S1.count[k] != A.sig[k] || S1.start[k] != A.sig[ns1 + k]) bad = 1;
    for (int k = threadIdx.x; k < ns2; k += blockDim.x)
        if (S2.count[k] != A.sig[2 * ns1 + k] || S2.start[k] != A.sig[2 * ns1 + ns2 + k]) bad = 1;
    // the stable sort by collision time -(c1 + c2)/2 (slicing.jl:561-568): the rank of pair p among all pairs
    __shared__ double tpair[kMaxSlices * kMaxSlices];
    const bool fits = ns1 >= 1 && ns2 >= 1 && ns1 <= kMaxSlices && ns2 <= kMaxSlices;
    if (fits)
        for (int p = threadIdx.x; p < np; p += blockDim.x) tpair[p] = -(S1.center[p / ns2] + S2.center[p % ns2]) / 2;
    else if (threadIdx.x == 0)
        bad = 1;
    __syncthreads();
    const long long *order = A.sig + 2 * ns1 + 2 * ns2;
    if (fits)
        for (int p = threadIdx.x; p < np; p += blockDim.x) {
            const double tp = tpair[p];
            int rank = 0;
            for (int q = 0; q < np; ++q) {
                const double tq = tpair[q];
                rank += (tq < tp) || (tq == tp && q < p);
            }
            if (order[rank] != p) bad = 1;
        }
    __syncthreads();
    if (bad) {
        if (threadIdx.x == 0) *A.ok = 0;
        return;  // the conditional keeps its default, 0
    }
    // the task drifts, as CollideJob::run computes them (pic_cpu.jl:954-1003, 1540-1548)
    for (int t = threadIdx.x; t < A.ntasks; t += blockDim.x) {
        Task &T = A.tasks[t];
        const SliceInfo &SS = T.dir == 1 ? S1 : S2, &SF = T.dir == 1 ? S2 : S1;
        const int ss = T.dir == 1 ? T.i - 1 : T.j - 1, sf = T.dir == 1 ? T.j - 1 : T.i - 1;
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
        J.sM1 = 0.5 * (S1.center[T.i - 1] - S2.center[T.j - 1]);
        J.sM2 = 0.5 * (S2.center[T.j - 1] - S1.center[T.i - 1]);
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
        // kinds: 0 L (sL), 1 R (sR), 2 M (midpoint), 3 Z (:node, the R drift)
        P.s = P.kind == 0 ? T.sL : (P.kind == 2 ? 0.5 * (T.sL + T.sR) : T.sR);
    }
    for (int k = threadIdx.x; k < A.nfirst; k += blockDim.x) {
        FirstLum &F = A.first[k];
        const LumJob &J = A.lumjobs[F.task / 2];
        F.sM = F.beam == 0 ? J.sM1 : J.sM2;
    }
    for (int t = threadIdx.x; t < A.ntasks; t += blockDim.x) {
        Task &T = A.tasks[t];
        if (T.next_task < 0) continue;
        const LumJob &J = A.lumjobs[T.next_task / 2];
        T.next_sM = T.fld_beam == 0 ? J.sM1 : J.sM2;
    }
    if (threadIdx.x == 0) {
        *A.ok = 1;
        cudaGraphSetConditional(A.handle, 1u);
    }
}

}  // namespace octo
