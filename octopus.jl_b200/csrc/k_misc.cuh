// One-turn map and seeded beam construction on the device.
#pragma once
#include "octo_internal.cuh"

namespace octo {

struct Mat6 {
    double m[36];
};

// Linear 6D map (linear6d.jl:110-121), applied `turns` times in FP64 to coordinates of element type R.
template <class R>
__global__ void __launch_bounds__(256) k_linear6d(R *x, R *px, R *y, R *py, R *z, R *pz, long long n, Mat6 M, int turns) {
    pdl_wait();
    pdl_release();
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = x[i], b = px[i], c = y[i], d = py[i], e = z[i], f = pz[i];
    const double *m = M.m;
    for (int t = 0; t < turns; ++t) {
        double x1 = m[0] * a + m[1] * b + m[2] * c + m[3] * d + m[4] * e + m[5] * f;
        double px1 = m[6] * a + m[7] * b + m[8] * c + m[9] * d + m[10] * e + m[11] * f;
        double y1 = m[12] * a + m[13] * b + m[14] * c + m[15] * d + m[16] * e + m[17] * f;
        double py1 = m[18] * a + m[19] * b + m[20] * c + m[21] * d + m[22] * e + m[23] * f;
        double z1 = m[24] * a + m[25] * b + m[26] * c + m[27] * d + m[28] * e + m[29] * f;
        double pz1 = m[30] * a + m[31] * b + m[32] * c + m[33] * d + m[34] * e + m[35] * f;
        a = x1; b = px1; c = y1; d = py1; e = z1; f = pz1;
    }
    x[i] = (R)a; px[i] = (R)b; y[i] = (R)c; py[i] = (R)d; z[i] = (R)e; pz[i] = (R)f;
}

// ---------------------------------------------------------------- counter RNG (counter_rng.jl)
__device__ __forceinline__ unsigned long long d_splitmix64(unsigned long long x) {
    unsigned long long z = x + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Philox4x32-10 block (counter_rng.jl:224-233) with the SplitMix key mix (:187-215).
__device__ __forceinline__ unsigned long long d_counter_u64(unsigned long long seed, unsigned long long turn,
                                                            unsigned long long rng_id, unsigned long long particle,
                                                            unsigned long long comp) {
    unsigned c0 = (unsigned)particle, c1 = (unsigned)(particle >> 32), c2 = (unsigned)turn, c3 = (unsigned)(turn >> 32);
    unsigned long long key = d_splitmix64(seed) ^ d_splitmix64(rng_id + 0x9e3779b97f4a7c15ull) ^
                             d_splitmix64(comp + 0xbf58476d1ce4e5b9ull);
    unsigned k0 = (unsigned)key, k1 = (unsigned)(key >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        unsigned hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        unsigned hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        unsigned n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return ((unsigned long long)c0 << 32) | (unsigned long long)c1;
}

__device__ __forceinline__ double d_uniform_open01(unsigned long long v) {
    return ((double)(v >> 12) + 0.5) * 2.220446049250313e-16;
}

// octopus_normal (counter_rng.jl:168-173): Box-Muller pair, odd component -> cos branch.
__global__ void k_beam_normals(double *out, long long n, unsigned long long seed, unsigned long long rng_id, int comp,
                               double cutoff) {
    pdl_wait();
    pdl_release();
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long particle = (unsigned long long)(i + 1);
    unsigned long long pair = (unsigned long long)((comp + 1) / 2);
    double u1 = d_uniform_open01(d_counter_u64(seed, 0, rng_id, particle, 2 * pair - 1));
    double u2 = d_uniform_open01(d_counter_u64(seed, 0, rng_id, particle, 2 * pair));
    double r = sqrt(-2.0 * log(u1));
    double theta = 6.283185307179586476925286766559 * u2;
    double g = (comp & 1) ? r * cos(theta) : r * sin(theta);
    if (isfinite(cutoff)) g = jclamp(g, -cutoff, cutoff);
    out[i] = g;
}

// Deterministic block partial sums of v (pow = 1) or (v - mu)^2 (pow = 2).
__global__ void __launch_bounds__(256) k_partial_sum(const double *v, long long n, const double *mu, int pow2,
                                                     double *partial) {
    pdl_wait();
    pdl_release();
    __shared__ double red[256];
    double m = pow2 ? *mu : 0.0;
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double a = v[i];
        acc += pow2 ? (a - m) * (a - m) : a;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void k_fold_partials(const double *partial, int nb, long long n, int stage, double *stats) {
    pdl_wait();
    pdl_release();
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += partial[b];
    if (stage == 0) stats[0] = s / (double)n;
    else stats[1] = sqrt(fmax(s / (double)n, 0.0));
}

// Beam.jl:148-160 (standardise) followed by the sigma/Twiss normalisation of Beam.jl:545-553.
__global__ void k_standardize(double *v, long long n, const double *stats) {
    pdl_wait();
    pdl_release();
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double mu = stats[0], s = stats[1];
    double a = v[i] - mu;
    v[i] = s == 0.0 ? 0.0 : a / s;
}

__global__ void k_twiss(double *q, double *p, long long n, double sigma, double beta, double alpha) {
    pdl_wait();
    pdl_release();
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double f = sigma / beta;
    double a = q[i];
    p[i] = f * (p[i] - alpha * a);
    q[i] = a * sigma;
}

}  // namespace octo
