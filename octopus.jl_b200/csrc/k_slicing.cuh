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
    int resolution[2];                 // :equal_area bins per slice
    long long *hist[2];                // :equal_area histogram counts
    unsigned long long *rkey[2], *rkey_sorted[2];  // :equal_count rank sort
    int *rval[2], *rval_sorted[2];
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
__global__ void __launch_bounds__(kLaneFoldThreads, 1) k_lane_fold(const SliceArgs<R> A, int square, int rows) {
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
        // eight independent loads in flight per thread before any of them is folded or staged
        for (int e0 = t; e0 < nr * 32; e0 += 8 * blockDim.x) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * (int)blockDim.x;
                const long long k = k0 + (e >> 5);
                v[u] = e < nr * 32 && k < cnt ? (double)z[k * kFoldLanes + first] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * (int)blockDim.x;
                if (e >= nr * 32) break;
                const int kk = e >> 5;
                if (!square && k0 + kk < cnt) {
                    lo = jmin(lo, v[u]);
                    hi = jmax(hi, v[u]);
                }
                tile[kk * 33 + l] = v[u];
            }
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

// Methods (OCTO_SLICING_*): 0 :normal_quantile, 1 :specified, 2 :equal_area, 3 :equal_count, 4 :equal_width.
constexpr int kEqualArea = 2, kEqualCount = 3, kEqualWidth = 4;

// Julia's collect(range(start, stop; length = len)) for Float64 endpoints (Base twiceprecision.jl, _linspace):
// the element of smallest magnitude as reference, the step split into a truncated high part and a low part
// fitted so both endpoints come out exactly, each element in double-double arithmetic around the reference
// index.  (Julia first tries an exact-rational construction for endpoints that are ratios of integers below
// 2^24; that branch is not restated -- it can differ in the last bit of an interior element.)
__device__ void julia_range(double start, double stop, int len, double *out) {
    if (len == 1) { out[0] = start; return; }
    if (start == stop) { for (int i = 0; i < len; ++i) out[i] = start; return; }
    auto add12 = [](double x, double y, double &h, double &l) {
        if (fabs(y) > fabs(x)) { const double t = x; x = y; y = t; }
        h = x + y;
        l = (x - h) + y;
    };
    double delta = stop - start;
    long long dfac = 1;
    if (!isfinite(delta)) { delta = stop / (double)len - start / (double)len; dfac = len; }
    const double tmin = -(start / delta) / (double)dfac;
    long long imin = (long long)rint(tmin * (double)(len - 1) + 1);
    double ref, step;
    if (1 < imin && imin < len) {
        const double t = (double)(imin - 1) / (double)(len - 1);
        ref = (1 - t) * start + t * stop;
        step = imin - 1 < len - imin ? (ref - start) / (double)(imin - 1) : (stop - ref) / (double)(len - imin);
    } else if (imin <= 1) {
        imin = 1;
        ref = start;
        step = (delta / (double)(len - 1)) * (double)dfac;
    } else {
        imin = len;
        ref = stop;
        step = (delta / (double)(len - 1)) * (double)dfac;
    }
    const double m = __longlong_as_double(0x7FEFFFFFFFFFFFFELL);  // prevfloat(floatmax(Float64))
    const double k = (double)max(imin - 1, (long long)len - imin);
    const double lo = jmax(-(m + ref) / k, (-m + ref) / k), hi = jmin((m - ref) / k, (m + ref) / k);
    const double step_pre = jclamp(step, lo, hi);
    const unsigned long long span = (unsigned long long)(max(imin - 1, (long long)len - imin) - 1);
    const int nb = min(span ? 64 - __clzll((long long)span) : 0, 27);  // nbitslen(Float64, len, imin)
    const double step_hi = __longlong_as_double((long long)((unsigned long long)__double_as_longlong(step_pre) &
                                                           ((~0ull) << nb)));
    double x1h, x1l, x2h, x2l;
    add12((double)(1 - imin) * step_hi, ref, x1h, x1l);
    add12((double)(len - imin) * step_hi, ref, x2h, x2l);
    const double a = (start - x1h) - x1l, b = (stop - x2h) - x2l;
    const double step_lo = (b - a) / (double)(len - 1);
    const double ref_lo = a - (double)(1 - imin) * step_lo;
    for (long long i = 1; i <= len; ++i) {
        const double u = (double)(i - imin);
        const double sh = u * step_hi, sl = u * step_lo;
        double xh, xl;
        add12(ref, sh, xh, xl);
        out[i - 1] = xh + (xl + (sl + ref_lo));
    }
}

// _slice_bin (slicing.jl:177-181), 0-based: the bin of zi, or -1 for a coordinate with none.  zi lies within
// the extrema that made zmin and width, so the clamp never meets an overflowing floor.
__device__ __forceinline__ long long slice_bin0(double zi, double zmin, double width, long long bins) {
    const double d = (zi - zmin) / width;
    if (!(d > -INFINITY && d < INFINITY)) return -1;
    const double f = floor(d);
    if (f >= (double)bins) return bins - 1;
    if (f < 0.0) return 0;
    const long long b = (long long)f;
    return b < 0 ? 0 : (b > bins - 1 ? bins - 1 : b);
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
    } else if (method == kEqualWidth) {  // :equal_width (slicing.jl:367-388)
        julia_range(info->zmin, info->zmax, ns + 1, b);
    } else if (method == kEqualArea || method == kEqualCount) {  // interior boundaries: k_area_bounds, k_rank_bounds
        b[0] = info->zmin;
        b[ns] = info->zmax;
        for (int k = 1; k < ns; ++k) b[k] = info->zmin;
        info->ns = ns;
        return;
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
// Slice of z under the beam's method: :equal_width files by _slice_bin on (zmin, (zmax - zmin) / ns)
// (slicing.jl:381-386; a zero-width beam goes to slice 1), the boundary methods by searchsortedlast.
__device__ __forceinline__ int slice_member(double z, const double *b, int ns, int zero_width, int method) {
    if (method == kEqualWidth) {
        if (zero_width) return 0;
        const long long s = slice_bin0(z, b[0], (b[ns] - b[0]) / (double)ns, ns);
        return s < 0 ? 0 : (int)s;
    }
    return slice_of(z, b, ns, zero_width);
}

// Per-block slice counts over contiguous chunks.  grid (max blocks, 1, 2).
template <class R>
__global__ void k_slice_count(const SliceArgs<R> A, long long chunk) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (blockIdx.x >= A.nblocks[bm] || A.method[bm] == kEqualCount) return;
    const R *__restrict__ z = A.c[bm][4];
    const long long n = A.n[bm];
    const SliceInfo *info = A.info[bm];
    __shared__ double b[kMaxSlices + 1];
    __shared__ int c[kMaxSlices];
    int ns = info->ns;
    const int method = A.method[bm];
    for (int t = threadIdx.x; t <= ns; t += blockDim.x) b[t] = info->boundary[t];
    for (int t = threadIdx.x; t < ns; t += blockDim.x) c[t] = 0;
    __syncthreads();
    int zw = info->zero_width;
    long long lo = (long long)blockIdx.x * chunk, hi = min(n, lo + chunk);
    // eight independent loads in flight per thread before any of them is counted
    for (long long i0 = lo + threadIdx.x; i0 < hi; i0 += 8LL * blockDim.x) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const long long i = i0 + (long long)u * blockDim.x;
            v[u] = i < hi ? (double)z[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (i0 + (long long)u * blockDim.x < hi) atomicAdd(&c[slice_member(v[u], b, ns, zw, method)], 1);
    }
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
    if (A.method[bm] == kEqualCount) return;  // ranks: k_rank_bounds set the starts
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
    if (blockIdx.x >= A.nblocks[bm] || A.method[bm] == kEqualCount) return;
    const long long n = A.n[bm];
    const SliceInfo *info = A.info[bm];
    const long long *blockoff = A.blockoff[bm];
    int *dest = A.dest[bm];
    const int method = A.method[bm];
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
        const int s = live ? slice_member((double)A.c[bm][4][i], b, ns, zw, method) : -1;
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

// ---------------------------------------------------------------- :equal_area (slicing.jl:104-156)
// Histogram of z over ns * resolution equal bins of [zmin, zmax] (_threaded_histogram with _slice_bin):
// block-private shared-memory counts, merged with global atomics (integer counts: any order is exact).
// grid (blocks of kChunk particles, 1, 2); dynamic shared memory bins * 4 bytes.
template <class R>
__global__ void __launch_bounds__(256) k_area_hist(const SliceArgs<R> A, long long chunk) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (blockIdx.x >= A.nblocks[bm] || A.method[bm] != kEqualArea) return;
    const SliceInfo *info = A.info[bm];
    const double zmin = info->zmin, zmax = info->zmax;
    if (!(zmin != zmax)) return;  // zero width (or non-finite): no histogram
    const long long bins = (long long)A.ns[bm] * A.resolution[bm];
    const double width = (zmax - zmin) / (double)bins;
    int *h = (int *)g_smem;
    for (long long t = threadIdx.x; t < bins; t += blockDim.x) h[t] = 0;
    __syncthreads();
    const R *__restrict__ z = A.c[bm][4];
    const long long lo = (long long)blockIdx.x * chunk, hi = min(A.n[bm], lo + chunk);
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const long long k = slice_bin0((double)z[i], zmin, width, bins);
        if (k >= 0) atomicAdd(&h[k], 1);
    }
    __syncthreads();
    for (long long t = threadIdx.x; t < bins; t += blockDim.x)
        if (h[t]) atomicAdd((unsigned long long *)&A.hist[bm][t], (unsigned long long)h[t]);
}

// Cumulative fractions of the histogram (one block per beam, an exact integer scan), then the interpolated
// equal-area boundaries by the reference's single pass over the bins.  Dynamic shared memory bins * 8 bytes.
template <class R>
__global__ void __launch_bounds__(1024) k_area_bounds(const SliceArgs<R> A) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.x;
    if (A.method[bm] != kEqualArea) return;
    SliceInfo *info = A.info[bm];
    const int ns = A.ns[bm];
    double *b = info->boundary;
    const double zmin = info->zmin, zmax = info->zmax;
    const long long bins = (long long)ns * A.resolution[bm];
    const double width = (zmax - zmin) / (double)bins;
    double *cum = (double *)g_smem;
    __shared__ long long wsum[32];
    const bool flat = !(zmin != zmax);
    if (!flat) {
        // inclusive scan of the counts in tiles of 1024, each thread one bin per tile
        const long long *cnt = A.hist[bm];
        const double nn = (double)(A.n[bm] > 1 ? A.n[bm] : 1);
        long long carry = 0;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (long long t0 = 0; t0 < bins; t0 += blockDim.x) {
            const long long t = t0 + threadIdx.x;
            const long long v = t < bins ? cnt[t] : 0;
            long long incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const long long w = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += w;
            }
            if (lane == 31) wsum[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                long long x = wsum[lane];
                for (int o = 1; o < 32; o <<= 1) {
                    const long long w = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += w;
                }
                wsum[lane] = x;
            }
            __syncthreads();
            const long long run = carry + (warp ? wsum[warp - 1] : 0) + incl;
            if (t < bins) cum[t] = (double)run / nn;
            carry += wsum[31];
            __syncthreads();
        }
        if (threadIdx.x == 0) cum[bins - 1] = 1.0;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    if (flat) {
        for (int k = 0; k <= ns; ++k) b[k] = zmin;
    } else {
        b[0] = zmin;
        b[ns] = zmax;
        long long current = 1;
        for (int s = 1; s <= ns - 1; ++s) {
            const double target = (double)s / (double)ns;
            while (current <= bins && cum[current - 1] <= target) ++current;
            double x1, x2, y1, y2;
            if (current <= 1) {
                x1 = b[0]; x2 = zmin + (1.0 - 0.5) * width; y1 = 0.0; y2 = cum[0];
            } else if (current > bins) {
                x1 = zmin + ((double)bins - 0.5) * width; x2 = b[ns]; y1 = cum[bins - 2]; y2 = 1.0;
            } else {
                x1 = zmin + ((double)(current - 1) - 0.5) * width; x2 = zmin + ((double)current - 0.5) * width;
                y1 = cum[current - 2]; y2 = cum[current - 1];
            }
            b[s] = y2 == y1 ? (x1 + x2) / 2 : x2 * (target - y1) / (y2 - y1) + x1 * (target - y2) / (y1 - y2);
        }
    }
    int bad = 0;
    for (int k = 0; k <= ns; ++k)
        if (!isfinite(b[k])) bad = 1;
    info->nonfinite = bad;
    info->zero_width = (b[0] == b[ns]) ? 1 : 0;
    info->ns = ns;
}

// ---------------------------------------------------------------- :equal_count (slicing.jl:330-365)
// Rank order: keys are z in Julia's isless order (the ordered-bits map), values the particle index; a stable
// radix sort (CUB) then yields sortperm(z) -- equal keys keep ascending index.  grid (blocks, 1, 2).
template <class R>
__global__ void k_rank_keys(const SliceArgs<R> A) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (A.method[bm] != kEqualCount) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < A.n[bm]; i += (long long)gridDim.x * blockDim.x) {
        A.rkey[bm][i] = ord_encode((double)A.c[bm][4][i]);
        A.rval[bm][i] = (int)i;
    }
}

// First rank of slice s (0-based): floor((s - 1) n / ns) of the 1-based formula.
__device__ __forceinline__ long long rank_first(int s, long long n, int ns) {
    return (long long)floor((double)((long long)s * n) / (double)ns);
}

// Boundaries at the rank midpoints, slice counts and (aligned) starts.  grid (2), one thread per beam.
template <class R>
__global__ void k_rank_bounds(const SliceArgs<R> A, int align) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.x;
    if (A.method[bm] != kEqualCount || threadIdx.x != 0) return;
    SliceInfo *info = A.info[bm];
    const int ns = A.ns[bm];
    const long long n = A.n[bm];
    const unsigned long long *key = A.rkey_sorted[bm];
    double *b = info->boundary;
    b[0] = info->zmin;
    b[ns] = info->zmax;
    for (int s = 1; s <= ns - 1; ++s) {
        const long long pos = rank_first(s, n, ns);
        b[s] = pos == 0 ? ord_decode(key[0])
                        : (pos == n ? ord_decode(key[n - 1]) : (ord_decode(key[pos - 1]) + ord_decode(key[pos])) / 2);
    }
    long long start = 0;
    for (int s = 0; s < ns; ++s) {
        const long long cnt = rank_first(s + 1, n, ns) - rank_first(s, n, ns);
        info->start[s] = start;
        info->count[s] = cnt;
        start += (cnt + align - 1) / align * align;
    }
    int bad = 0;
    for (int k = 0; k <= ns; ++k)
        if (!isfinite(b[k])) bad = 1;
    info->nonfinite = bad;
    info->zero_width = 0;
    info->ns = ns;
}

// Rank r goes to slice s with rank_first(s) <= r < rank_first(s + 1), at start[s] + r - rank_first(s).
// grid (blocks, 1, 2).
template <class R>
__global__ void k_rank_scatter(const SliceArgs<R> A) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (A.method[bm] != kEqualCount) return;
    const SliceInfo *info = A.info[bm];
    const int ns = A.ns[bm];
    const long long n = A.n[bm];
    __shared__ long long first[kMaxSlices + 1], st[kMaxSlices];
    for (int s = threadIdx.x; s <= ns; s += blockDim.x) first[s] = rank_first(s, n, ns);
    for (int s = threadIdx.x; s < ns; s += blockDim.x) st[s] = info->start[s];
    __syncthreads();
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        int s = 0;
        while (s < ns - 1 && first[s + 1] <= r) ++s;
        const int i = A.rval_sorted[bm][r];
        const long long pos = st[s] + (r - first[s]);
        A.dest[bm][i] = (int)pos;
#pragma unroll
        for (int k = 0; k < 6; ++k) A.s[bm][k][pos] = A.c[bm][k][i];
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

// ---------------------------------------------------------------- spatial order inside slices
// The plain PIC collide is independent of the order of particles inside a slice (int64 fixed-point charge
// and luminosity grids, per-particle kicks, order-free extrema), so its working copy can hold each slice's
// particles grouped by transverse position: a kick warp then gathers its field taps from a few neighbouring
// cells instead of 32 random ones.  Each slice's box is cut into kSpatialBins x kSpatialBins bins (row-major,
// y slow); a counting sort places the particles bin by bin (the order inside a bin is the order the atomic
// cursors hand out positions, which changes no result).  A particle's slice is read from its position in the
// stable copy (dest), whatever the slicing method.  The centroid lanes were folded from the stable copy before
// this pass.  grid (blocks of kChunk caller-order particles, 1, 2 beams) unless noted.
constexpr int kSpatialBins = 64;
constexpr int kSpatialCells = kSpatialBins * kSpatialBins;
template <class R>
struct SpatialArgs {
    const R *c[2][6];          // caller-order coordinates
    R *t[2][6];                // spatially ordered slice-contiguous copies
    int *dest[2];              // caller index -> working-copy position
    const SliceInfo *info[2];
    unsigned long long *box[2];  // [slice][4] ordered x min, x max, y min, y max
    int *cursor[2];            // [slice][kSpatialCells] counts, then write cursors
    long long n[2], nblocks[2];
};

// Slice of stable-copy position p (the slices are contiguous, in order): the last s with start[s] <= p.
__device__ __forceinline__ int slice_at(long long p, const long long *start, int ns) {
    int s = 0;
    while (s < ns - 1 && start[s + 1] <= p) ++s;
    return s;
}

template <class R>
__global__ void __launch_bounds__(256) k_spatial_boxes(const SpatialArgs<R> A, long long chunk) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (blockIdx.x >= A.nblocks[bm]) return;
    const SliceInfo *info = A.info[bm];
    __shared__ long long st[kMaxSlices];
    __shared__ unsigned long long bx[kMaxSlices][4];
    const int ns = info->ns;
    for (int t = threadIdx.x; t < ns; t += blockDim.x) st[t] = info->start[t];
    for (int t = threadIdx.x; t < ns * 4; t += blockDim.x) bx[t >> 2][t & 3] = (t & 1) ? kOrdMaxInit : kOrdMinInit;
    __syncthreads();
    const long long lo = (long long)blockIdx.x * chunk, hi = min(A.n[bm], lo + chunk);
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const int s = slice_at(A.dest[bm][i], st, ns);
        const unsigned long long ex = ord_encode((double)A.c[bm][0][i]), ey = ord_encode((double)A.c[bm][2][i]);
        atomicMin(&bx[s][0], ex); atomicMax(&bx[s][1], ex);
        atomicMin(&bx[s][2], ey); atomicMax(&bx[s][3], ey);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ns * 4; t += blockDim.x) {
        unsigned long long *g = &A.box[bm][t];
        if (t & 1) atomicMax(g, bx[t >> 2][t & 3]);
        else atomicMin(g, bx[t >> 2][t & 3]);
    }
}

// Bin of a particle in its slice's box (non-finite coordinates land in bin 0; the collide rejects them).
__device__ __forceinline__ int spatial_bin(double x, double y, const double *bb) {
    const double ux = (x - bb[0]) * bb[1], uy = (y - bb[2]) * bb[3];
    const int ix = ux >= 0.0 ? (ux < (double)kSpatialBins ? (int)ux : kSpatialBins - 1) : 0;
    const int iy = uy >= 0.0 ? (uy < (double)kSpatialBins ? (int)uy : kSpatialBins - 1) : 0;
    return iy * kSpatialBins + ix;
}
// x0, bins per unit x, y0, bins per unit y of every slice box, in shared memory
__device__ __forceinline__ void load_spatial_boxes(const unsigned long long *box, int ns, double (*bb)[4]) {
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
        const double x0 = ord_decode(box[4 * s]), x1 = ord_decode(box[4 * s + 1]);
        const double y0 = ord_decode(box[4 * s + 2]), y1 = ord_decode(box[4 * s + 3]);
        bb[s][0] = x0;
        bb[s][1] = x1 > x0 ? (double)kSpatialBins / (x1 - x0) : 0.0;
        bb[s][2] = y0;
        bb[s][3] = y1 > y0 ? (double)kSpatialBins / (y1 - y0) : 0.0;
    }
}

template <class R>
__global__ void __launch_bounds__(256) k_spatial_count(const SpatialArgs<R> A, long long chunk) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (blockIdx.x >= A.nblocks[bm]) return;
    const SliceInfo *info = A.info[bm];
    __shared__ long long st[kMaxSlices];
    __shared__ double bb[kMaxSlices][4];
    const int ns = info->ns;
    for (int t = threadIdx.x; t < ns; t += blockDim.x) st[t] = info->start[t];
    load_spatial_boxes(A.box[bm], ns, bb);
    __syncthreads();
    const long long lo = (long long)blockIdx.x * chunk, hi = min(A.n[bm], lo + chunk);
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const int s = slice_at(A.dest[bm][i], st, ns);
        const int bin = spatial_bin((double)A.c[bm][0][i], (double)A.c[bm][2][i], bb[s]);
        atomicAdd(&A.cursor[bm][s * kSpatialCells + bin], 1);
    }
}

// Exclusive scan of each slice's bin counts into write cursors starting at the slice's start.
// grid (max slices, 2), 1024 threads: four consecutive bins per thread.
template <class R>
__global__ void __launch_bounds__(1024) k_spatial_scan(const SpatialArgs<R> A) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.y, s = blockIdx.x;
    const SliceInfo *info = A.info[bm];
    if (s >= info->ns) return;
    __shared__ int wsum[32];
    int *cnt = A.cursor[bm] + s * kSpatialCells;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int v[4], tot = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) { v[k] = cnt[4 * t + k]; tot += v[k]; }
    int incl = tot;
    for (int o = 1; o < 32; o <<= 1) {
        const int w = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += w;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int x = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int w = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += w;
        }
        wsum[lane] = x;
    }
    __syncthreads();
    long long base = info->start[s] + (warp ? wsum[warp - 1] : 0) + incl - tot;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        cnt[4 * t + k] = (int)base;
        base += v[k];
    }
}

template <class R>
__global__ void __launch_bounds__(256) k_spatial_scatter(const SpatialArgs<R> A, long long chunk) {
    pdl_wait();
    pdl_release();
    const int bm = blockIdx.z;
    if (blockIdx.x >= A.nblocks[bm]) return;
    const SliceInfo *info = A.info[bm];
    __shared__ long long st[kMaxSlices];
    __shared__ double bb[kMaxSlices][4];
    const int ns = info->ns;
    for (int t = threadIdx.x; t < ns; t += blockDim.x) st[t] = info->start[t];
    load_spatial_boxes(A.box[bm], ns, bb);
    __syncthreads();
    const long long lo = (long long)blockIdx.x * chunk, hi = min(A.n[bm], lo + chunk);
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        R v[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = A.c[bm][k][i];
        const int s = slice_at(A.dest[bm][i], st, ns);
        const int bin = spatial_bin((double)v[0], (double)v[2], bb[s]);
        const int pos = atomicAdd(&A.cursor[bm][s * kSpatialCells + bin], 1);
        A.dest[bm][i] = pos;
#pragma unroll
        for (int k = 0; k < 6; ++k) A.t[bm][k][pos] = v[k];
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
