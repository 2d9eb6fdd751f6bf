// Longitudinal slicing on the device (slicing.jl:51-75, 405-460, 523-559).
//
// The particle arrays have element type R (double, or float in the precision form); every statistic
// is folded in FP64.  Order-dependent statistics use the reference's canonical 4096-lane fold (slicing.jl:208-257):
// lane t folds elements t, t+4096, ... in order and the lanes are folded serially, so the
// mean, sigma and slice centroids are bit-identical to the reference's.  Membership is a
// stable partition: each slice's members keep ascending particle order, the order the
// reference's index lists have, and the particles are gathered into slice-contiguous
// structure-of-arrays buffers in the same pass.
#pragma once
#include "octo_internal.cuh"

namespace octo {

struct SliceInfo {          // device-resident, read back once per collide
    double boundary[kMaxSlices + 1];
    double center[kMaxSlices];
    double weight[kMaxSlices];
    long long count[kMaxSlices];
    long long start[kMaxSlices];
    double mu, sigma, zmin, zmax;
    int ns;
    int zero_width;
    int nonfinite;
    int pad;
};

// Both beams are sliced by the same launches: blockIdx.z (or blockIdx.x for the one-block kernels)
// selects the beam, so the two serial lane folds run side by side.
template <class R>
struct SliceArgs {
    const R *c[2][6];        // caller-order coordinates x, px, y, py, z, pz
    R *s[2][6];              // slice-sorted copies
    int *dest[2];            // caller index -> slice-sorted position
    SliceInfo *info[2];
    double *lane_sum[2], *lane_min[2], *lane_max[2], *lanes[2];
    const double *q[2];      // quantile table (see k_fold_stats)
    int *counts[2];
    long long *blockoff[2];
    long long n[2], nblocks[2];
    int method[2], ns[2], cpos[2];
};

// Lane partial sums / extrema over all particles.  square != 0 folds (z - mu)^2.
// Lane t must add elements t, t+4096, ... strictly in order, so the parallelism is across lanes.  A block
// owns 32 lanes: all its threads stage up to kLaneFoldRows rows of the 32 lane columns in shared memory
// (one tile covers the production beams), then one thread per lane adds its column in order from shared
// memory, eight loads ahead.  The extrema do not depend on order (min and max with Julia's signed-zero
// and NaN rules), so the staging threads fold them and a final pass combines the 16 threads of each lane.
// grid (128, 1, 2); dynamic shared memory rows x 33 doubles.
constexpr int kLaneFoldThreads = 512, kLaneFoldRows = 640;
template <class R>
__global__ void __launch_bounds__(kLaneFoldThreads) k_lane_fold(const SliceArgs<R> A, int square, int rows) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    const R *__restrict__ z = A.c[bm][4];
    const long long n = A.n[bm];
    const SliceInfo *info = A.info[bm];
    double *lane_sum = A.lane_sum[bm], *lane_min = A.lane_min[bm], *lane_max = A.lane_max[bm];
    double *tile = (double *)g_smem;  // [rows][33]
    __shared__ double red_lo[kLaneFoldThreads], red_hi[kLaneFoldThreads];
    const int lane0 = blockIdx.x * 32, t = threadIdx.x, l = t & 31;  // every element a thread stages is lane l's
    const double mu = square ? info->mu : 0.0;
    const long long first = lane0 + l;
    const long long cnt = first < n ? (n - first + kFoldLanes - 1) / kFoldLanes : 0;  // elements of lane l
    const long long iters = (n + kFoldLanes - 1) / kFoldLanes;
    double s = 0.0, lo = INFINITY, hi = -INFINITY;
    for (long long k0 = 0; k0 < iters; k0 += rows) {
        const int nr = (int)min((long long)rows, iters - k0);
        for (int e = t; e < nr * 32; e += blockDim.x) {
            const int kk = e >> 5;
            const long long k = k0 + kk;
            double v = 0.0;
            if (k < cnt) {
                v = (double)z[k * kFoldLanes + first];
                if (!square) {
                    lo = jmin(lo, v);
                    hi = jmax(hi, v);
                }
            }
            tile[kk * 33 + l] = v;
        }
        __syncthreads();
        if (t < 32) {
            const int m = (int)max(0LL, min((long long)nr, cnt - k0));  // lane t's rows in this tile
            int kk = 0;
            for (; kk + 8 <= m; kk += 8) {
                double v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = tile[(kk + u) * 33 + t];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (square) {
                        const double d = v[u] - mu;
                        s += d * d;
                    } else {
                        s += v[u];
                    }
                }
            }
            for (; kk < m; ++kk) {
                const double v = tile[kk * 33 + t];
                if (square) {
                    const double d = v - mu;
                    s += d * d;
                } else {
                    s += v;
                }
            }
        }
        __syncthreads();
    }
    if (!square) {
        red_lo[t] = lo;
        red_hi[t] = hi;
        __syncthreads();
        if (t < 32) {
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
                lo = jmin(lo, red_lo[t + 32 * w]);
                hi = jmax(hi, red_hi[t + 32 * w]);
            }
            lane_min[lane0 + t] = lo;
            lane_max[lane0 + t] = hi;
        }
    }
    if (t < 32) lane_sum[lane0 + t] = s;
}

// In-order sum of n shared-memory values, sixteen loads ahead of the adds (the order of a plain loop).
__device__ __forceinline__ double serial_sum(const double *v, int n) {
    double s = 0.0;
    int t = 0;
    for (; t + 16 <= n; t += 16) {
        double w[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) w[u] = v[t + u];
#pragma unroll
        for (int u = 0; u < 16; ++u) s += w[u];
    }
    for (; t < n; ++t) s += v[t];
    return s;
}

// Serial fold of the lanes (slicing.jl:254-257), staged through shared memory so the single adding
// thread reads at shared-memory latency.  stage 0: mean and extrema; stage 1: sigma and boundaries.
// q[s] for s = 1..ns-1 holds sqrt(2)*erfinv(2s/ns - 1) (:normal_quantile) or the :specified positions.
// grid (2): one block per beam.
template <class R>
__global__ void __launch_bounds__(1024) k_fold_stats(const SliceArgs<R> A, int stage) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.x;
    const double *lane_sum = A.lane_sum[bm], *lane_min = A.lane_min[bm], *lane_max = A.lane_max[bm];
    const long long n = A.n[bm];
    const int method = A.method[bm], ns = A.ns[bm];
    const double *q = A.q[bm];
    SliceInfo *info = A.info[bm];
    __shared__ double sl[kFoldLanes];
    __shared__ double rlo[32], rhi[32];
    for (int t = threadIdx.x; t < kFoldLanes; t += blockDim.x) sl[t] = lane_sum[t];
    if (stage == 0) {  // extrema are order independent: parallel reduce
        double lo = INFINITY, hi = -INFINITY;
        for (int t = threadIdx.x; t < kFoldLanes; t += blockDim.x) { lo = jmin(lo, lane_min[t]); hi = jmax(hi, lane_max[t]); }
        for (int o = 16; o; o >>= 1) {
            lo = jmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = jmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if ((threadIdx.x & 31) == 0) { rlo[threadIdx.x >> 5] = lo; rhi[threadIdx.x >> 5] = hi; }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double s = serial_sum(sl, kFoldLanes);
    if (stage == 0) {
        double lo = INFINITY, hi = -INFINITY;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { lo = jmin(lo, rlo[w]); hi = jmax(hi, rhi[w]); }
        info->mu = s / (double)n;
        info->zmin = lo;
        info->zmax = hi;
        return;
    }
    double mu = info->mu;
    double sigma = sqrt(jmax(s / (double)n, 0.0));
    info->sigma = sigma;
    double *b = info->boundary;
    if (method == 0) {  // :normal_quantile (slicing.jl:405-429)
        if (sigma == 0.0) {
            for (int k = 0; k <= ns; ++k) b[k] = mu;
        } else {
            b[0] = info->zmin;
            b[ns] = info->zmax;
            for (int k = 1; k <= ns - 1; ++k) b[k] = jclamp(mu + sigma * q[k], b[0], b[ns]);
        }
    } else {  // :specified (slicing.jl:393-403): internal = sort(mu + p*sigma)
        double internal[kMaxSlices];
        int m = ns - 1;
        for (int k = 0; k < m; ++k) internal[k] = mu + q[k + 1] * sigma;
        for (int a = 1; a < m; ++a) {  // stable insertion sort
            double v = internal[a];
            int c = a - 1;
            while (c >= 0 && v < internal[c]) { internal[c + 1] = internal[c]; --c; }
            internal[c + 1] = v;
        }
        b[0] = info->zmin;
        b[ns] = info->zmax;
        for (int k = 0; k < m; ++k) b[k + 1] = jclamp(internal[k], b[0], b[ns]);
    }
    int bad = 0;
    for (int k = 0; k <= ns; ++k)
        if (!isfinite(b[k])) bad = 1;
    info->nonfinite = bad;
    info->zero_width = (b[0] == b[ns]) ? 1 : 0;
    info->ns = ns;
}

// searchsortedlast(boundary, z) clamped to [1, ns], returned 0-based (slicing.jl:454-457).
__device__ __forceinline__ int slice_of(double z, const double *b, int ns, int zero_width) {
    if (zero_width) return 0;
    int k = 0;
    for (int t = 0; t <= ns; ++t) k += (b[t] <= z) ? 1 : 0;
    k = k < 1 ? 1 : (k > ns ? ns : k);
    return k - 1;
}

// Per-block slice counts over contiguous chunks.  grid (max blocks, 1, 2).
template <class R>
__global__ void k_slice_count(const SliceArgs<R> A, long long chunk) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (blockIdx.x >= A.nblocks[bm]) return;
    const R *__restrict__ z = A.c[bm][4];
    const long long n = A.n[bm];
    const SliceInfo *info = A.info[bm];
    __shared__ double b[kMaxSlices + 1];
    __shared__ int c[kMaxSlices];
    int ns = info->ns;
    for (int t = threadIdx.x; t <= ns; t += blockDim.x) b[t] = info->boundary[t];
    for (int t = threadIdx.x; t < ns; t += blockDim.x) c[t] = 0;
    __syncthreads();
    int zw = info->zero_width;
    long long lo = (long long)blockIdx.x * chunk, hi = min(n, lo + chunk);
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&c[slice_of((double)z[i], b, ns, zw)], 1);
    __syncthreads();
    for (int t = threadIdx.x; t < ns; t += blockDim.x) A.counts[bm][(long long)blockIdx.x * ns + t] = c[t];
}

// Slice starts (aligned to `align` elements) and per-block write offsets: one warp per slice sums its
// per-block counts and scans them in chunks of 32 blocks (integer sums: any order is exact).
// grid (2): one block per beam, 1024 threads.
__device__ __forceinline__ long long warp_incl_scan(long long v) {
    const int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        const long long w = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += w;
    }
    return v;
}
template <class R>
__global__ void __launch_bounds__(1024) k_slice_offsets(const SliceArgs<R> A, int align) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.x;
    const int *counts = A.counts[bm];
    const int nblocks = (int)A.nblocks[bm];
    SliceInfo *info = A.info[bm];
    long long *blockoff = A.blockoff[bm];
    const int ns = info->ns;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __shared__ long long tot[kMaxSlices];
    for (int s = warp; s < ns; s += nw) {
        long long acc = 0;
        for (int b = lane; b < nblocks; b += 32) acc += counts[(long long)b * ns + s];
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) tot[s] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long pos = 0;
        for (int s = 0; s < ns; ++s) {
            info->start[s] = pos;
            info->count[s] = tot[s];
            pos += (tot[s] + align - 1) / align * align;
        }
    }
    __syncthreads();
    for (int s = warp; s < ns; s += nw) {
        long long base = info->start[s];
        for (int b0 = 0; b0 < nblocks; b0 += 32) {
            const int b = b0 + lane;
            const long long v = b < nblocks ? counts[(long long)b * ns + s] : 0;
            const long long incl = warp_incl_scan(v);
            if (b < nblocks) blockoff[(long long)b * ns + s] = base + incl - v;
            base += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
}

// Stable scatter into slice-contiguous SoA buffers; dest[original index] = pos.
// Each block walks its chunk in rounds of blockDim (1024) particles: warps rank their particles per slice
// with match_any, one warp per slice scans the per-warp counts into write positions, and every particle
// writes its six coordinates.  grid (max blocks, 1, 2).
constexpr int kScatterThreads = 1024;
template <class R>
__global__ void __launch_bounds__(kScatterThreads) k_slice_scatter(const SliceArgs<R> A, long long chunk) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (blockIdx.x >= A.nblocks[bm]) return;
    const long long n = A.n[bm];
    const SliceInfo *info = A.info[bm];
    const long long *blockoff = A.blockoff[bm];
    int *dest = A.dest[bm];
    __shared__ double b[kMaxSlices + 1];
    __shared__ long long run[kMaxSlices];
    __shared__ long long wpos[kScatterThreads / 32][kMaxSlices];  // per-warp count, then write base
    const int ns = info->ns;
    const int zw = info->zero_width;
    for (int t = threadIdx.x; t <= ns; t += blockDim.x) b[t] = info->boundary[t];
    for (int t = threadIdx.x; t < ns; t += blockDim.x) run[t] = blockoff[(long long)blockIdx.x * ns + t];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const long long lo = (long long)blockIdx.x * chunk, hi = min(n, lo + chunk);
    for (long long base = lo; base < hi; base += blockDim.x) {
        for (int t = threadIdx.x; t < nwarps * ns; t += blockDim.x) wpos[t / ns][t % ns] = 0;
        __syncthreads();  // the previous round's reads of wpos are done (its closing barrier) and b, run are loaded
        const long long i = base + threadIdx.x;
        const bool live = i < hi;
        const int s = live ? slice_of((double)A.c[bm][4][i], b, ns, zw) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, s);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (live && rank == 0) wpos[warp][s] = __popc(peers);
        __syncthreads();
        for (int sl = warp; sl < ns; sl += nwarps) {  // exclusive scan over warps, one warp per slice
            const long long v = lane < nwarps ? wpos[lane][sl] : 0;
            const long long incl = warp_incl_scan(v);
            if (lane < nwarps) wpos[lane][sl] = run[sl] + incl - v;
            __syncwarp();
            if (lane == 31) run[sl] += incl;
        }
        __syncthreads();
        if (live) {
            const long long pos = wpos[warp][s] + rank;
            dest[i] = (int)pos;
#pragma unroll
            for (int k = 0; k < 6; ++k) A.s[bm][k][pos] = A.c[bm][k][i];
        }
        __syncthreads();
    }
}

// Centroid lane sums per slice: lane t folds members t, t+4096, ... of the slice list (slicing.jl:240-257).
// grid (kFoldLanes / 256, max slices, 2).
template <class R>
__global__ void k_slice_lanes(const SliceArgs<R> A) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    const SliceInfo *info = A.info[bm];
    int s = blockIdx.y;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kFoldLanes || s >= info->ns) return;
    const R *__restrict__ sz = A.s[bm][4];
    long long st = info->start[s], cnt = info->count[s];
    double acc = 0.0;
    for (long long k = t; k < cnt; k += kFoldLanes) acc += (double)sz[st + k];
    A.lanes[bm][(long long)s * kFoldLanes + t] = acc;
}

// Serial lane fold per slice (one block per slice, lanes staged in shared memory); centers and
// weights (slicing.jl:523-559).  grid (max slices, 2).
template <class R>
__global__ void __launch_bounds__(1024) k_slice_finish(const SliceArgs<R> A) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.y;
    SliceInfo *info = A.info[bm];
    const double *lanes = A.lanes[bm];
    const long long n = A.n[bm];
    const int center_position = A.cpos[bm];
    __shared__ double sl[kFoldLanes];
    const int s = blockIdx.x;
    if (s >= info->ns) return;
    const long long cnt = info->count[s];
    const bool fold = center_position == 0 && cnt > 0;
    if (fold)
        for (int t = threadIdx.x; t < kFoldLanes; t += blockDim.x) sl[t] = lanes[(long long)s * kFoldLanes + t];
    __syncthreads();
    if (threadIdx.x != 0) return;
    info->weight[s] = (double)cnt / (double)n;
    const double *b = info->boundary;
    if (fold) {
        info->center[s] = serial_sum(sl, kFoldLanes) / (double)cnt;
    } else {
        info->center[s] = (b[s] + b[s + 1]) / 2;
    }
}

// Write the kicked slice-sorted coordinates back in caller order, both beams (blockIdx.y), as a gather
// over caller indices: the stores are coalesced and the loads follow the slices' ascending runs (the
// slice scatter is stable).  z is left alone: a collide never changes it, so the caller's z array
// already holds the final values.
template <class R>
struct UnsortArgs {
    const int *dest[2];
    const R *s[2][5];  // sorted x, px, y, py, pz
    R *c[2][5];        // caller-order x, px, y, py, pz
    const R *sz[2];    // sorted z, when the collide moved z (a z-moving virtual drift), else NULL
    R *cz[2];
    long long n[2];
};
template <class R>
__global__ void k_unsort(const UnsortArgs<R> A) {
    pdl_wait();
    pdl_release();
    const int b = blockIdx.y;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n[b]) return;
    const int p = A.dest[b][i];
#pragma unroll
    for (int k = 0; k < 5; ++k) A.c[b][k][i] = A.s[b][k][p];
    if (A.sz[b]) A.cz[b][i] = A.sz[b][p];
}

}  // namespace octo
