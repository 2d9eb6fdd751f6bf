// Beam moment rows as the moment observer records them (src/tasks/BeamObservers.jl:1000-1060, 1254-1271):
// the means of the six coordinates, then central moments mean(prod_d (c_d - <c_d>)^p_d) of the requested
// power rows, over the live particles (all six coordinates finite) when lost particles are masked, else
// over all particles (one non-finite particle then makes the row NaN).
//
// Two passes over the beam, as the definition needs the means first: k_moment_sums (six sums and the live
// count), then k_moment_pairs (all 21 second-order sums from one read of each particle) and, for rows of
// order 3 and more, k_moment_general in chunks.  Each writes per-block partials (a fixed block count)
// that a fold block sums in a fixed order, so a row is deterministic for a given beam size; the folds write
// the row into device memory, so observing a turn never synchronises the host.
#pragma once
#include "octo_internal.cuh"

namespace octo {

constexpr int kMomentBlocks = 1184;     // partial-sum blocks (a fixed count: fold order independent of the GPU)
constexpr int kMomentThreads = 256;
constexpr int kMomentWarps = kMomentThreads / 32;
constexpr int kMomentChunk = 8;         // rows of order >= 3 per generic pass (accumulators held in registers)
constexpr int kMomentPairs = 21;        // second-order rows: the products of deviations (i <= j)
constexpr int kMomentsMax = 256;

// Rows of order >= 3 of one generic pass.
struct MomentPowers {
    int n;
    unsigned char p[kMomentChunk][6];
    unsigned char slot[kMomentChunk];   // each row's position among the row's moments
};
// Second-order rows: which of the 21 pair sums (pair index of (i, j), i <= j, row-major over the upper
// triangle) goes to which slot.
struct MomentPairRows {
    int n;
    unsigned char pair[kMomentPairs], slot[kMomentPairs];
};
// The order-1 entries of a row: row slot and coordinate of each mean.
struct MomentHead {
    int n;
    unsigned char slot[6], coord[6];
};

__device__ __forceinline__ bool live6(const double (&c)[6]) {
    return isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2]) && isfinite(c[3]) && isfinite(c[4]) && isfinite(c[5]);
}

// Block sums of N per-thread values in a fixed order: a shuffle tree inside each warp, then the warps' sums
// in warp order by thread k < N; partial[blockIdx.x * N + k] receives sum k.
template <int N>
__device__ __forceinline__ void block_sums(double (&v)[N], double *red /* N * kMomentWarps */, double *partial) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        double t = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) red[k * kMomentWarps + warp] = t;
    }
    __syncthreads();
    if ((int)threadIdx.x < N) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kMomentWarps; ++w) t += red[threadIdx.x * kMomentWarps + w];
        partial[blockIdx.x * N + threadIdx.x] = t;
    }
}

template <class R>
__device__ __forceinline__ void load6(double (&c)[6], const R *x, const R *px, const R *y, const R *py, const R *z,
                                      const R *pz, long long i) {
    c[0] = (double)x[i];
    c[1] = (double)px[i];
    c[2] = (double)y[i];
    c[3] = (double)py[i];
    c[4] = (double)z[i];
    c[5] = (double)pz[i];
}

template <class R>
__global__ void __launch_bounds__(kMomentThreads) k_moment_sums(const R *__restrict__ x, const R *__restrict__ px,
                                                                  const R *__restrict__ y, const R *__restrict__ py,
                                                                  const R *__restrict__ z, const R *__restrict__ pz,
                                                                  long long n, int mask, double *partial) {
    pdl_wait();
    pdl_release();
    __shared__ double red[7 * kMomentWarps];
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double c[6];
        load6(c, x, px, y, py, z, pz, i);
        if (mask && !live6(c)) continue;
#pragma unroll
        for (int d = 0; d < 6; ++d) s[d] += c[d];
        s[6] += 1.0;
    }
    block_sums<7>(s, red, partial);
}

// Fixed-order sum of partial[b * stride + k] over b < nb by one block of kMomentThreads threads: thread t
// takes b = t, t + kMomentThreads, ... in order, then the block's fixed shuffle/warp tree.
__device__ __forceinline__ double fold_partials(const double *partial, int nb, int stride, int k) {
    __shared__ double red[kMomentWarps];
    double t = 0.0;
    for (int b = threadIdx.x; b < nb; b += kMomentThreads) t += partial[(size_t)b * stride + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kMomentWarps; ++w) s += red[w];
    return s;
}

// The live count means[6] and means[0..5]; block k folds partial column k (7 blocks).
__global__ void __launch_bounds__(kMomentThreads) k_moment_means(const double *partial, int nb, double *sums) {
    pdl_wait();
    pdl_release();
    const double s = fold_partials(partial, nb, 7, blockIdx.x);
    if (threadIdx.x == 0) sums[blockIdx.x] = s;
}
__global__ void k_moment_divide(double *means) {
    pdl_wait();
    pdl_release();
    if (threadIdx.x < 6) means[8 + threadIdx.x] = means[threadIdx.x] / means[6];
}

// All 21 second-order sums: (c_i - <c_i>) (c_j - <c_j>) for i < j, (c_i - <c_i>)^2 for i = j (the reference's
// term 1.0 * d_i * d_j, and d_i^2 = d_i * d_i).
template <class R>
__global__ void __launch_bounds__(kMomentThreads) k_moment_pairs(const R *__restrict__ x, const R *__restrict__ px,
                                                                   const R *__restrict__ y, const R *__restrict__ py,
                                                                   const R *__restrict__ z, const R *__restrict__ pz,
                                                                   long long n, int mask, const double *means,
                                                                   double *partial) {
    pdl_wait();
    pdl_release();
    __shared__ double red[kMomentPairs * kMomentWarps];
    double mu[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) mu[d] = means[8 + d];
    double acc[kMomentPairs];
#pragma unroll
    for (int k = 0; k < kMomentPairs; ++k) acc[k] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double c[6];
        load6(c, x, px, y, py, z, pz, i);
        if (mask && !live6(c)) continue;
        double dv[6];
#pragma unroll
        for (int d = 0; d < 6; ++d) dv[d] = c[d] - mu[d];
        int k = 0;
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int b = a; b < 6; ++b) acc[k++] += dv[a] * dv[b];
    }
    block_sums<kMomentPairs>(acc, red, partial);
}

__device__ __noinline__ double ipow(double v, int p) {
    double r = v;
    for (int k = 1; k < p; ++k) r *= v;
    return r;
}

// Rows of order >= 3: term = 1.0 * prod_d (c_d - <c_d>)^p_d in coordinate order, the power by repeated
// products.
template <class R>
__global__ void __launch_bounds__(kMomentThreads, 2) k_moment_general(const R *__restrict__ x, const R *__restrict__ px,
                                                                     const R *__restrict__ y, const R *__restrict__ py,
                                                                     const R *__restrict__ z, const R *__restrict__ pz,
                                                                     long long n, int mask, const double *means,
                                                                     const __grid_constant__ MomentPowers P,
                                                                     double *partial) {
    pdl_wait();
    pdl_release();
    __shared__ double red[kMomentChunk * kMomentWarps];
    double mu[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) mu[d] = means[8 + d];
    double acc[kMomentChunk];
#pragma unroll
    for (int k = 0; k < kMomentChunk; ++k) acc[k] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double c[6];
        load6(c, x, px, y, py, z, pz, i);
        if (mask && !live6(c)) continue;
        double dv[6];
#pragma unroll
        for (int d = 0; d < 6; ++d) dv[d] = c[d] - mu[d];
#pragma unroll
        for (int k = 0; k < kMomentChunk; ++k) {
            double term = 1.0;
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                const int p = P.p[k][d];
                if (p) term *= ipow(dv[d], p);
            }
            acc[k] += k < P.n ? term : 0.0;
        }
    }
    block_sums<kMomentChunk>(acc, red, partial);
}

// Folds of the block partials (fixed order), divided by the live count (0 / 0 = NaN for a beam without
// live particles, as the reference reports it).  Block k folds requested row k.
__global__ void __launch_bounds__(kMomentThreads) k_moment_fold_pairs(const double *partial, int nb,
                                                                        const double *means, MomentPairRows Q,
                                                                        double *row) {
    pdl_wait();
    pdl_release();
    const int k = blockIdx.x;
    const double s = fold_partials(partial, nb, kMomentPairs, Q.pair[k]);
    if (threadIdx.x == 0) row[1 + Q.slot[k]] = s / means[6];
}
__global__ void __launch_bounds__(kMomentThreads) k_moment_fold(const double *partial, int nb, const double *means,
                                                                  MomentPowers P, double *row) {
    pdl_wait();
    pdl_release();
    const int k = blockIdx.x;
    const double s = fold_partials(partial, nb, kMomentChunk, k);
    if (threadIdx.x == 0) row[1 + P.slot[k]] = s / means[6];
}

// row[0] = turn and the order-1 entries (the means; NaN for a beam without live particles).
__global__ void k_moment_row_head(const double *means, double turn, MomentHead head, double *row) {
    pdl_wait();
    pdl_release();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    row[0] = turn;
    for (int k = 0; k < head.n; ++k) row[1 + head.slot[k]] = means[8 + head.coord[k]];
}

}  // namespace octo
