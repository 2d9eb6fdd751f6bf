// Line tracking between collisions: a sequence of zero-length elements applied to each particle in
// registers, `turns` times, in one pass over the beam (fusedTrack with a TrackingContext,
// src/track/fused_track.jl:53-77; the CUDA loop of src/track/phase6d_track.jl:197-212).
//
// The element list arrives as a kernel parameter (LineProgram, < 4 KB): every thread of a warp runs the
// same element at the same time, so the switch over element kinds is uniform and the parameters are
// read through the constant bank.  Coordinates of either storage type are widened to FP64 on load and
// rounded once on store; all element arithmetic is FP64.
//
// Per-element constants that the reference evaluates per particle but that depend only on parameters
// (cos / sin / tan of the boost angle, 1/sqrt of the coupling determinant, the crab harmonics' i kcc,
// the Philox keys of the six radiation components) are evaluated once on the host with the same
// operations, so they are identical to the reference's values.
#pragma once
#include "octo_internal.cuh"
#include "k_misc.cuh"

namespace octo {

enum : int {
    kElemLinear6D = 1,
    kElemCrab = 2,
    kElemBoost = 3,
    kElemRevBoost = 4,
    kElemChrom = 5,
    kElemRad = 6,
    kElemCrabDisp = 7,
    kElemMomDisp = 8,
    kElemXY = 9,
};
constexpr int kLineOpsPerLaunch = 10;  // LineProgram stays under the classic 4 KB kernel-parameter limit
constexpr int kRadDamping = 1, kRadExcitation = 2;
// Frame transforms whose coefficients are all zero: the identity on finite coordinates (up to the sign of a
// zero result), so they are skipped for particles whose six coordinates are finite; a particle with a
// non-finite coordinate runs them, spreading NaN exactly as the reference's arithmetic does.
constexpr int kZeroZeta = 4, kZeroEta = 8, kZeroR = 16;
// Thin crab cavity: some harmonics had zero strengths in both planes and were dropped on the host.
constexpr int kCrabDropped = 1;

// One compiled element.  a[] layout per kind:
//   Linear6D   a[0..35] row-major matrix
//   crab       a[h] i kcc, a[8+h] strengthX, a[16+h] strengthY, a[24+h] phase (h < n)
//   boost      a[0] cos, a[1] sin, a[2] tan of the half crossing angle
//   chrom      a[0..1] xi, a[2..3] beta, a[4..5] alpha, a[6..7] gamma, a[8..11] zeta, a[12..15] eta,
//              a[16..19] R, a[20] 1/sqrt(1 + r1 r4 - r2 r3)
//   rad        a[0..2] damping, a[3..11] excitation, a[12..15] zeta, a[16..19] eta, a[20..23] R, a[24] g;
//              flags: kRadDamping | kRadExcitation (effective components); key[c]: component c+1's key
//   crab disp  a[0..3] zeta;  mom disp a[0..3] eta;  xy a[0..3] r, a[4] g, n = mode
struct LineOp {
    int kind, n, flags, pad;
    double a[36];
    unsigned long long key[6];
};
struct LineProgram {
    int nops, rng, turns, pad;
    long long turn0;
    LineOp op[kLineOpsPerLaunch];
};
static_assert(sizeof(LineProgram) + 64 <= 4096, "LineProgram and the pointers must fit the 4 KB kernel-parameter space");

struct Coords {
    double x, px, y, py, z, pz;
};

// CrabDispersion, MomentumDispersion and XYCoupling (mode A) forward maps (linear_maps.jl:125-132, 213-220,
// 355-373) and their inverses (chromaticity_kick.jl:151-186).
__device__ __forceinline__ void crab_disp(Coords &c, const double *zt) {
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py, z0 = c.z, pz0 = c.pz;
    c.pz = pz0 + zt[1] * x0 - zt[0] * px0 + zt[3] * y0 - zt[2] * py0;
    c.x = x0 + zt[0] * z0;
    c.px = px0 + zt[1] * z0;
    c.y = y0 + zt[2] * z0;
    c.py = py0 + zt[3] * z0;
}
__device__ __forceinline__ void crab_disp_inv(Coords &c, const double *zt) {
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py, z0 = c.z, pz0 = c.pz;
    c.pz = pz0 - zt[1] * x0 + zt[0] * px0 - zt[3] * y0 + zt[2] * py0;
    c.x = x0 - zt[0] * z0;
    c.px = px0 - zt[1] * z0;
    c.y = y0 - zt[2] * z0;
    c.py = py0 - zt[3] * z0;
}
__device__ __forceinline__ void mom_disp(Coords &c, const double *et) {
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py, z0 = c.z, pz0 = c.pz;
    c.z = z0 - et[1] * x0 + et[0] * px0 - et[3] * y0 + et[2] * py0;
    c.x = x0 + et[0] * pz0;
    c.px = px0 + et[1] * pz0;
    c.y = y0 + et[2] * pz0;
    c.py = py0 + et[3] * pz0;
}
__device__ __forceinline__ void mom_disp_inv(Coords &c, const double *et) {
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py, z0 = c.z, pz0 = c.pz;
    c.z = z0 + et[1] * x0 - et[0] * px0 + et[3] * y0 - et[2] * py0;
    c.x = x0 - et[0] * pz0;
    c.px = px0 - et[1] * pz0;
    c.y = y0 - et[2] * pz0;
    c.py = py0 - et[3] * pz0;
}
// mode 0: identity, 1: A, 2: B
__device__ __forceinline__ void xy_coupling(Coords &c, const double *r, double g, int mode) {
    if (mode == 0) return;
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py;
    if (mode == 1) {
        c.x = g * (x0 + r[3] * y0 - r[1] * py0);
        c.px = g * (px0 - r[2] * y0 + r[0] * py0);
        c.y = g * (-r[0] * x0 - r[1] * px0 + y0);
        c.py = g * (-r[2] * x0 - r[3] * px0 + py0);
    } else {
        c.x = g * (r[3] * x0 - r[1] * px0 + y0);
        c.px = g * (-r[2] * x0 + r[0] * px0 + py0);
        c.y = g * (x0 - r[0] * y0 - r[1] * py0);
        c.py = g * (px0 - r[2] * y0 - r[3] * py0);
    }
}
__device__ __forceinline__ void xy_coupling_inv_a(Coords &c, const double *r, double g) {
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py;
    c.x = g * (x0 - r[3] * y0 + r[1] * py0);
    c.px = g * (px0 + r[2] * y0 - r[0] * py0);
    c.y = g * (r[0] * x0 + r[1] * px0 + y0);
    c.py = g * (r[2] * x0 + r[3] * px0 + py0);
}

__device__ __forceinline__ void linear6d(Coords &c, const double *m) {
    const double a = c.x, b = c.px, d = c.y, e = c.py, f = c.z, h = c.pz;
    c.x = m[0] * a + m[1] * b + m[2] * d + m[3] * e + m[4] * f + m[5] * h;
    c.px = m[6] * a + m[7] * b + m[8] * d + m[9] * e + m[10] * f + m[11] * h;
    c.y = m[12] * a + m[13] * b + m[14] * d + m[15] * e + m[16] * f + m[17] * h;
    c.py = m[18] * a + m[19] * b + m[20] * d + m[21] * e + m[22] * f + m[23] * h;
    c.z = m[24] * a + m[25] * b + m[26] * d + m[27] * e + m[28] * f + m[29] * h;
    c.pz = m[30] * a + m[31] * b + m[32] * d + m[33] * e + m[34] * f + m[35] * h;
}

// ThinCrabCavity (crab_cavity.jl:128-144): harmonic sums in harmonic order.  The host keeps only harmonics
// with a nonzero strength; a dropped one would add (0 s)/(i kcc) and (0 x + 0 y) c, which are zeros for finite
// coordinates (and subtracting a zero from these sums never changes them) and NaN when z (or x, y) is not
// finite, which the last three statements reproduce.
__device__ __forceinline__ void crab_cavity(Coords &c, const LineOp &op) {
    double dpx = 0.0, dpy = 0.0, dpz = 0.0;
    for (int h = 0; h < op.n; ++h) {
        const double ikcc = op.a[h];
        double s, co;
        sincos(ikcc * c.z + op.a[24 + h], &s, &co);
        const double sx = op.a[8 + h], sy = op.a[16 + h];
        dpx -= sx * s / ikcc;
        dpy -= sy * s / ikcc;
        dpz -= (sx * c.x + sy * c.y) * co;
    }
    if (op.flags & kCrabDropped) {
        const double zs = 0.0 * c.z;
        dpx -= zs;
        dpy -= zs;
        dpz -= (0.0 * c.x + 0.0 * c.y) + zs;
    }
    c.px += dpx;
    c.py += dpy;
    c.pz += dpz;
}

__device__ __forceinline__ bool all_finite6(const Coords &c) { return isfinite(c.x + c.px + c.y + c.py + c.z + c.pz); }

// LorentzBoost and RevLorentzBoost (lorentz_boost.jl:128-161), Hirata's crossing-angle transformation.
__device__ __forceinline__ void boost(Coords &c, double ca, double sa, double ta) {
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py, z0 = c.z, pz0 = c.pz;
    const double ps0 = sqrt((1.0 + pz0) * (1.0 + pz0) - px0 * px0 - py0 * py0);
    const double h0 = 1.0 + pz0 - ps0;
    const double py1 = py0 / ca;
    const double h1 = h0 / (ca * ca);
    const double px1 = px0 / ca - h1 * sa;
    const double pz1 = pz0 - px1 * sa;
    const double ps1 = 1.0 + pz1 - h1;
    const double ds = x0 * sa;
    c.x = x0 + z0 * ta + px1 / ps1 * ds;
    c.y = y0 + py1 / ps1 * ds;
    c.z = z0 / ca - h1 / ps1 * ds;
    c.px = px1;
    c.py = py1;
    c.pz = pz1;
}
__device__ __forceinline__ void rev_boost(Coords &c, double ca, double sa) {
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py, z0 = c.z, pz0 = c.pz;
    const double ps0 = sqrt((1.0 + pz0) * (1.0 + pz0) - px0 * px0 - py0 * py0);
    const double h0 = 1.0 + pz0 - ps0;
    double x1 = x0 - z0 * sa;
    x1 = x1 / (1.0 + (px0 + h0 * sa) * sa / ps0);
    c.z = (z0 + h0 / ps0 * x1 * sa) * ca;
    c.y = y0 - py0 / ps0 * x1 * sa;
    c.pz = pz0 + px0 * sa;
    c.px = (px0 + h0 * sa) * ca;
    c.py = py0 * ca;
    c.x = x1;
}

// ChromaticityKick (chromaticity_kick.jl:98-136).
__device__ __forceinline__ void chromaticity(Coords &c, const double *a, int flags) {
    const double *zt = a + 8, *et = a + 12, *r = a + 16;
    const double g = a[20];
    const bool full = !all_finite6(c);
    if (full || !(flags & kZeroZeta)) crab_disp_inv(c, zt);
    if (full || !(flags & kZeroEta)) mom_disp_inv(c, et);
    if (full || !(flags & kZeroR)) xy_coupling_inv_a(c, r, g);
    const double x0 = c.x, px0 = c.px, y0 = c.y, py0 = c.py;
    const double xix = a[0], xiy = a[1], betx = a[2], bety = a[3], alfx = a[4], alfy = a[5], gamx = a[6],
                 gamy = a[7];
    const double twopi = 6.283185307179586476925286766559005768394338;
    double sx, cx, sy, cy;
    sincos(twopi * xix * c.pz, &sx, &cx);
    c.x = x0 * (cx + alfx * sx) + px0 * betx * sx;
    c.px = -x0 * sx * gamx + px0 * (cx - alfx * sx);
    sincos(twopi * xiy * c.pz, &sy, &cy);
    c.y = y0 * (cy + alfy * sy) + py0 * bety * sy;
    c.py = -y0 * sy * gamy + py0 * (cy - alfy * sy);
    const double jx = 0.5 * (gamx * x0 * x0 + 2.0 * alfx * x0 * px0 + betx * px0 * px0);
    const double jy = 0.5 * (gamy * y0 * y0 + 2.0 * alfy * y0 * py0 + bety * py0 * py0);
    c.z += twopi * (xix * jx + xiy * jy);
    if (full || !(flags & kZeroR)) xy_coupling(c, r, g, 1);
    if (full || !(flags & kZeroEta)) mom_disp(c, et);
    if (full || !(flags & kZeroZeta)) crab_disp(c, zt);
}

// Uniform on (0, 1) of a component's counter draw (counter_rng.jl:168-176 with the keys precomputed):
// Philox4x32-10 on the counter (particle, turn); SplitMix: the hash of key ^ mix(turn) ^ mix(particle).
__device__ __forceinline__ double line_uniform(int rng, unsigned long long key, unsigned long long particle,
                                               unsigned long long turn, unsigned long long smix_tp) {
    unsigned long long v;
    if (rng == 1) {
        unsigned c0 = (unsigned)particle, c1 = (unsigned)(particle >> 32), c2 = (unsigned)turn,
                 c3 = (unsigned)(turn >> 32);
        unsigned k0 = (unsigned)key, k1 = (unsigned)(key >> 32);
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            // one 32x32 -> 64-bit product gives both halves of each Philox multiply
            const unsigned long long p0 = (unsigned long long)c0 * 0xD2511F53u;
            const unsigned long long p1 = (unsigned long long)c2 * 0xCD9E8D57u;
            const unsigned n0 = (unsigned)(p1 >> 32) ^ c1 ^ k0, n2 = (unsigned)(p0 >> 32) ^ c3 ^ k1;
            c0 = n0;
            c1 = (unsigned)p1;
            c2 = n2;
            c3 = (unsigned)p0;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        v = ((unsigned long long)c0 << 32) | (unsigned long long)c1;
    } else {
        v = d_splitmix64(key ^ smix_tp);
    }
    return d_uniform_open01(v);
}

// One Box-Muller pair (counter_rng.jl:154-166) and its plane's excitation (radiation.jl:220-227).
__device__ __forceinline__ void rad_plane(double &q, double &p, const double *e, unsigned long long k1,
                                          unsigned long long k2, int rng, unsigned long long particle,
                                          unsigned long long turn, unsigned long long smix_tp) {
    const double u1 = line_uniform(rng, k1, particle, turn, smix_tp);
    const double u2 = line_uniform(rng, k2, particle, turn, smix_tp);
    const double rr = sqrt(-2.0 * log(u1));
    double s, co;
    sincos(6.283185307179586476925286766559 * u2, &s, &co);
    const double n1 = rr * co, n2 = rr * s;
    q += e[0] * n1;
    p += e[1] * n2 + e[2] * n1;
}

// LumpedRad (radiation.jl:196-232, context draws :241-279): components 1..6 are (x, px, y, py, z, pz) normals,
// pairs (1,2), (3,4), (5,6) from one Box-Muller transform each.
__device__ __forceinline__ void lumped_rad(Coords &c, const LineOp &op, int rng, unsigned long long particle,
                                           unsigned long long turn, unsigned long long smix_tp) {
    const bool damp = op.flags & kRadDamping, exc = op.flags & kRadExcitation;
    if (!damp && !exc) return;
    const double *a = op.a;
    const double *zt = a + 12, *et = a + 16, *r = a + 20;
    const double g = a[24];
    const bool full = !all_finite6(c);
    if (full || !(op.flags & kZeroZeta)) crab_disp_inv(c, zt);
    if (full || !(op.flags & kZeroEta)) mom_disp_inv(c, et);
    if (full || !(op.flags & kZeroR)) xy_coupling_inv_a(c, r, g);
    if (damp) {
        c.x *= a[0];
        c.px *= a[0];
        c.y *= a[1];
        c.py *= a[1];
        c.z *= a[2];
        c.pz *= a[2];
    }
    if (exc) {
        // pair p feeds plane p only: q += amp n1, p += slope n2 + cross n1 (n1 the cos branch)
        const double *e = a + 3;
        rad_plane(c.x, c.px, e, op.key[0], op.key[1], rng, particle, turn, smix_tp);
        rad_plane(c.y, c.py, e + 3, op.key[2], op.key[3], rng, particle, turn, smix_tp);
        rad_plane(c.z, c.pz, e + 6, op.key[4], op.key[5], rng, particle, turn, smix_tp);
    }
    // a particle that was finite stays finite through damping and excitation
    if (full || !(op.flags & kZeroR)) xy_coupling(c, r, g, 1);
    if (full || !(op.flags & kZeroEta)) mom_disp(c, et);
    if (full || !(op.flags & kZeroZeta)) crab_disp(c, zt);
}

template <class R>
__global__ void __launch_bounds__(256) k_track_line(R *__restrict__ x, R *__restrict__ px, R *__restrict__ y,
                                                    R *__restrict__ py, R *__restrict__ z, R *__restrict__ pz,
                                                    long long n, const __grid_constant__ LineProgram P) {
    pdl_wait();
    pdl_release();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Coords c{(double)x[i], (double)px[i], (double)y[i], (double)py[i], (double)z[i], (double)pz[i]};
        const unsigned long long particle = (unsigned long long)(i + 1);
        // SplitMix's particle mix does not depend on the turn or the component
        const unsigned long long smix_p = P.rng == 2 ? d_splitmix64(particle + 0x94d049bb133111ebull) : 0ull;
        for (int t = 0; t < P.turns; ++t) {
            const unsigned long long turn = (unsigned long long)(P.turn0 + t);
            const unsigned long long smix_tp =
                P.rng == 2 ? (d_splitmix64(turn + 0x9e3779b97f4a7c15ull) ^ smix_p) : 0ull;
            // Unrolled over the program's slots: every parameter address is a compile-time offset into the
            // constant bank, an operand of the arithmetic itself (a loop index would make each parameter an
            // indexed constant load, which throttles on the address-divergence unit).
#pragma unroll
            for (int k = 0; k < kLineOpsPerLaunch; ++k) {
                if (k >= P.nops) break;
                const LineOp &op = P.op[k];
                switch (op.kind) {
                    case kElemLinear6D: linear6d(c, op.a); break;
                    case kElemCrab: crab_cavity(c, op); break;
                    case kElemBoost: boost(c, op.a[0], op.a[1], op.a[2]); break;
                    case kElemRevBoost: rev_boost(c, op.a[0], op.a[1]); break;
                    case kElemChrom: chromaticity(c, op.a, op.flags); break;
                    case kElemRad: lumped_rad(c, op, P.rng, particle, turn, smix_tp); break;
                    case kElemCrabDisp: crab_disp(c, op.a); break;
                    case kElemMomDisp: mom_disp(c, op.a); break;
                    case kElemXY: xy_coupling(c, op.a, op.a[4], op.n); break;
                    default: break;
                }
            }
        }
        x[i] = (R)c.x;
        px[i] = (R)c.px;
        y[i] = (R)c.y;
        py[i] = (R)c.py;
        z[i] = (R)c.z;
        pz[i] = (R)c.pz;
    }
}

}  // namespace octo
