// The soft-Gaussian strong-strong solver (GaussianPoissonSolver, src/tasks/strongstrong/gaussian.jl): every
// slice pair kicks each slice with the Bassetti-Erskine field of a Gaussian carrying the other slice's
// transverse moments, drifted to each particle's collision point.  Runs on the slice-sorted coordinates of
// the collide path, one wavefront of conflict-free pairs at a time:
//   k_gauss_sums    shifted first and second sums of every slice of the front (relative to the slice's
//                   first particle, as slicing.jl:670-770 sums), per block of kGaussChunk particles;
//   k_gauss_moments one block per slice: the block partials in a fixed order -> the moment set;
//   k_gauss_kick    drift in, kick, longitudinal term, drift out for every particle of both directions,
//                   and the luminosity density of the sampled direction per block;
//   k_gauss_lum     one block per pair: its density partials in a fixed order -> the pair's luminosity.
#pragma once
#include "be_device.cuh"
#include "k_pic.cuh"
#include "octo_internal.cuh"

namespace octo {

constexpr int kGaussChunk = 8192;    // particles per partial-sum / kick block
constexpr int kGaussThreads = 256;
constexpr int kGaussSums = 14;        // dx, dpx, dy, dpy, dx^2, dpx^2, dy^2, dpy^2, dx dpx, dy dpy, and the
                                      // coupled dx dy, dx dpy, dpx dy, dpx dpy

// One slice of one beam whose moments a front needs.
struct GSlice {
    long long start, n;     // range in the beam's slice-sorted arrays
    int beam;
    int task;               // a kick task whose source this slice is (error reports)
};
// The moment set of a slice (the uncoupled StrongTransverseMoments plus the centroid the kick subtracts).
// One direction of one pair: the field slice kicked by the Gaussian of the source slice.
struct GTask {
    long long fld_start, fld_n;
    int fld_beam, mom;      // mom: the source slice's GMoments index
    int pair, lum;          // lum: this direction samples the pair's luminosity
    double center;          // source slice centre (the virtual drift's reference)
    double kbb;             // weight of the source slice x kbb of the field beam
    double klum;            // weight of the source slice x luminosity scale of the field beam
};
struct GaussArgs {
    void *c[2][6];          // slice-sorted coordinates of both beams, element type R of the kernels
    const GSlice *slices;
    GMoments *mom;
    const GTask *tasks;
    const int2 *blockmap;   // (slice or task index, first particle offset) per block
    double *partial;        // per block
    double *lum_partial;    // per kick block
    double *lum_parts;      // per pair (collision-order index)
    DevStatus *status;
    double min_sigma;
    int ignore_centroid[2];
    int longitudinal;
    int drift;              // virtual drift with the longitudinal kick: 0 Hirata, 1 chromatic, 2 exact
    int coupled;            // include_sigma_xy: the full transverse covariance
};

// The virtual drifts to and from the collision point (strong_beam.jl:517-606): forward returns S.  Without the
// longitudinal kick the solver uses the frozen-longitudinal paraxial drift (gaussian.jl:148-150).
__device__ __forceinline__ double drift_forward(int kind, bool lk, double &x, double px, double &y, double py,
                                                double &z, double &pz, double zo) {
    if (!lk || kind == 0) {
        const double S = 0.5 * (z - zo);
        x += S * px;
        y += S * py;
        if (lk) pz -= 0.25 * (px * px + py * py);
        return S;
    }
    if (kind == 1) {  // ChromaticDrift
        const double S = 0.5 * (z - zo);
        const double phi = sqrt(1 - 0.5 * (px * px + py * py) / ((1 + pz) * (1 + pz))) - 1;
        x += S * px / (1 + pz);
        y += S * py / (1 + pz);
        z += 2 * S * phi;
        pz += (1 + pz) * phi;
        return S;
    }
    // ExactHamiltonianDrift
    const double ps = sqrt((1 + pz) * (1 + pz) - px * px - py * py);
    const double H = 1 + pz - ps;
    const double rr = 0.5 * H / ps;
    const double z2 = (z + rr * zo) / (1 + rr);
    const double S = 0.5 * (z2 - zo);
    z -= H / ps * S;
    pz -= 0.5 * H;
    x += px / ps * S;
    y += py / ps * S;
    return S;
}
__device__ __forceinline__ void drift_reverse(int kind, bool lk, double &x, double px, double &y, double py, double &z,
                                              double &pz, double zo) {
    const double S = 0.5 * (z - zo);
    if (!lk || kind == 0) {
        x -= S * px;
        y -= S * py;
        if (lk) pz += 0.25 * (px * px + py * py);
        return;
    }
    if (kind == 1) {
        const double psi = sqrt(1 + 0.5 * (px * px + py * py) / ((1 + pz) * (1 + pz))) - 1;
        x -= S * px / (1 + pz);
        y -= S * py / (1 + pz);
        z += 2 * S * psi;
        pz += (1 + pz) * psi;
        return;
    }
    const double H0 = 0.5 * (px * px + py * py) / (1 + pz);
    const double ps0 = 1 + pz - 0.5 * H0;
    pz += 0.5 * H0;
    x -= px / ps0 * S;
    y -= py / ps0 * S;
    z += H0 / ps0 * S;
}

// R: the beams' element type.  float32 beams (the precision form) are read and written in float and computed in
// FP64, as the reference promotes a Float32 beam's coordinates against the solver's Float64 moments and scales
// (gaussian.jl:64-70) and rounds them once on store.
template <class R>
__device__ __forceinline__ R *gcol(const GaussArgs &A, int beam, int k) { return static_cast<R *>(A.c[beam][k]); }

template <class R>
__global__ void __launch_bounds__(kGaussThreads) k_gauss_sums(GaussArgs A) {
    pdl_wait();
    pdl_release();
    const int2 bm = A.blockmap[blockIdx.x];
    const GSlice S = A.slices[bm.x];
    const R *c[4] = {gcol<R>(A, S.beam, 0), gcol<R>(A, S.beam, 1), gcol<R>(A, S.beam, 2), gcol<R>(A, S.beam, 3)};
    const double x0 = c[0][S.start], px0 = c[1][S.start], y0 = c[2][S.start], py0 = c[3][S.start];
    double s[kGaussSums] = {};
    const long long end = min(S.n, (long long)bm.y + kGaussChunk);
    for (long long k = bm.y + threadIdx.x; k < end; k += kGaussThreads) {
        const long long i = S.start + k;
        const double dx = (double)c[0][i] - x0, dpx = (double)c[1][i] - px0, dy = (double)c[2][i] - y0,
                     dpy = (double)c[3][i] - py0;
        s[0] += dx; s[1] += dpx; s[2] += dy; s[3] += dpy;
        s[4] += dx * dx; s[5] += dpx * dpx; s[6] += dy * dy; s[7] += dpy * dpy;
        s[8] += dx * dpx; s[9] += dy * dpy;
        if (A.coupled) { s[10] += dx * dy; s[11] += dx * dpy; s[12] += dpx * dy; s[13] += dpx * dpy; }
    }
    __shared__ double red[kGaussSums][kGaussThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kGaussSums; ++q) {
        double t = s[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) red[q][warp] = t;
    }
    __syncthreads();
    if ((int)threadIdx.x < kGaussSums) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kGaussThreads / 32; ++w) t += red[threadIdx.x][w];
        A.partial[(size_t)blockIdx.x * kGaussSums + threadIdx.x] = t;
    }
}

// Block b0 .. b0 + nb - 1 of k_gauss_sums belong to slice blockIdx.x (first block index in first[]).
template <class R>
__global__ void k_gauss_moments(GaussArgs A, const int *first, const int *count) {
    pdl_wait();
    pdl_release();
    if (threadIdx.x != 0) return;
    const int si = blockIdx.x;
    const GSlice S = A.slices[si];
    GMoments M{};
    const double floor2 = A.min_sigma * A.min_sigma;
    if (S.n == 0) {
        // slicing.jl:679-687: an empty slice is a centred Gaussian of the floor size
        M.a0 = floor2;
        M.d0 = floor2;
        A.mom[si] = M;
        return;
    }
    double s[kGaussSums] = {};
    for (int b = first[si]; b < first[si] + count[si]; ++b)
#pragma unroll
        for (int q = 0; q < kGaussSums; ++q) s[q] += A.partial[(size_t)b * kGaussSums + q];
    const double x0 = gcol<R>(A, S.beam, 0)[S.start], px0 = gcol<R>(A, S.beam, 1)[S.start],
                 y0 = gcol<R>(A, S.beam, 2)[S.start], py0 = gcol<R>(A, S.beam, 3)[S.start];
    // slicing.jl:739-770: means from the shifted sums, variances muladd(-m, m, sum2 / n), floors
    const double invn = 1.0 / (double)S.n;
    const double dmx = s[0] * invn, dmpx = s[1] * invn, dmy = s[2] * invn, dmpy = s[3] * invn;
    const double sx2 = fma(-dmx, dmx, s[4] * invn), spx2 = fma(-dmpx, dmpx, s[5] * invn);
    const double sy2 = fma(-dmy, dmy, s[6] * invn), spy2 = fma(-dmpy, dmpy, s[7] * invn);
    const double covxpx = fma(-dmx, dmpx, s[8] * invn), covypy = fma(-dmy, dmpy, s[9] * invn);
    M.a0 = fmax(sx2, floor2);
    M.d0 = fmax(sy2, floor2);
    M.bxx = covxpx;
    M.bypy = covypy;
    M.qxx = fmax(spx2, 0.0);
    M.qyy = fmax(spy2, 0.0);
    if (A.coupled) {
        M.b0 = fma(-dmx, dmy, s[10] * invn);
        M.bxpy = fma(-dmx, dmpy, s[11] * invn);
        M.bypx = fma(-dmpx, dmy, s[12] * invn);
        M.qxy = fma(-dmpx, dmpy, s[13] * invn);
    }
    if (!A.ignore_centroid[S.beam]) {
        M.mx = x0 + dmx;
        M.mpx = px0 + dmpx;
        M.my = y0 + dmy;
        M.mpy = py0 + dmpy;
    }
    // non-finite chokepoint (gaussian.jl:33-42): the reduction saw every transverse coordinate of the slice
    const double chk = M.mx + M.mpx + M.my + M.mpy + sx2 + sy2 + spx2 + spy2 + covxpx + covypy + (x0 + px0 + y0 + py0);
    if (!isfinite(chk)) record_error(A.status, S.task, OCTO_ERR_NONFINITE, 1);
    A.mom[si] = M;
}

// _apply_slice_kick_one! (gaussian.jl:152-185) with the uncoupled _cp_covariance_kick (strong_beam.jl:619-632)
// between the virtual drifts above.
// Three blocks per SM (at most 85 registers): the Bassetti-Erskine response is an FP64 latency chain, and
// occupancy hides it better than registers do (measured: 10.6 ms per production collide at one block per
// SM, 9.4 at two, 9.0 at three).
template <class R>
__global__ void __launch_bounds__(kGaussThreads, 3) k_gauss_kick(GaussArgs A) {
    pdl_wait();
    pdl_release();
    const int2 bm = A.blockmap[blockIdx.x];
    const GTask T = A.tasks[bm.x];
    const GMoments M = A.mom[T.mom];
    R *c[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) c[q] = gcol<R>(A, T.fld_beam, q);
    const bool lk = A.longitudinal != 0;
    const double twopi = 6.283185307179586476925286766559005768394338;
    double dens = 0.0;
    const long long end = min(T.fld_n, (long long)bm.y + kGaussChunk);
    for (long long k = bm.y + threadIdx.x; k < end; k += kGaussThreads) {
        const long long i = T.fld_start + k;
        double x = c[0][i], px = c[1][i], y = c[2][i], py = c[3][i], z = c[4][i], pz = c[5][i];
        const double S = drift_forward(A.drift, lk, x, px, y, py, z, pz, T.center);
        const double xx = x - M.mx + M.mpx * S;
        const double yy = y - M.my + M.mpy * S;
        const double px0 = px, py0 = py, pz0 = pz;
        // _transport_transverse_moments (strong_beam.jl:679-687), uncoupled
        const double a = M.a0 - 2 * S * M.bxx + S * S * M.qxx;
        const double d = M.d0 - 2 * S * M.bypy + S * S * M.qyy;
        const double au = 2 * (M.bxx - S * M.qxx);
        const double du = 2 * (M.bypy - S * M.qyy);
        double density = 0.0;
        if (A.coupled) coupled_kick(M, T.kbb, S, xx, yy, px, py, pz, density);
        else if (!(a <= 0 || d <= 0)) {
            const double sigx = sqrt(a), sigy = sqrt(d);
            double Kx, Ky, Hxx, Hyy;
            be_response(T.kbb, sigx, sigy, xx, yy, Kx, Ky, Hxx, Hyy);
            const double expterm = exp(-0.5 * (xx * xx / (sigx * sigx) + yy * yy / (sigy * sigy)));
            px += Kx * T.kbb;
            py += Ky * T.kbb;
            pz += 0.25 * (Hxx * au + Hyy * du);
            density = expterm / twopi / sigx / sigy;
        }
        if (lk) pz += 0.5 * ((px - px0) * M.mpx + (py - py0) * M.mpy);
        else pz = pz0;
        drift_reverse(A.drift, lk, x, px, y, py, z, pz, T.center);
        c[0][i] = (R)x;
        c[1][i] = (R)px;
        c[2][i] = (R)y;
        c[3][i] = (R)py;
        c[4][i] = (R)z;
        c[5][i] = (R)pz;
        dens += density * twopi;
    }
    if (!T.lum) return;
    __shared__ double red[kGaussThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dens += __shfl_xor_sync(0xffffffffu, dens, o);
    if (lane == 0) red[warp] = dens;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kGaussThreads / 32; ++w) t += red[w];
        A.lum_partial[blockIdx.x] = t;
    }
}

// Pair luminosity (gaussian.jl:64-108): sum of density * 2 pi over the sampled slice / 2 pi * klum.
// One thread per sampling task; its kick blocks' partials in block order.
__global__ void k_gauss_lum(GaussArgs A, const int *lum_task, const int *first, const int *count, int nlum) {
    pdl_wait();
    pdl_release();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlum) return;
    const GTask T = A.tasks[lum_task[k]];
    double s = 0.0;
    for (int b = first[k]; b < first[k] + count[k]; ++b) s += A.lum_partial[b];
    const double twopi = 6.283185307179586476925286766559005768394338;
    A.lum_parts[T.pair] = s / twopi * T.klum;
}

}  // namespace octo
