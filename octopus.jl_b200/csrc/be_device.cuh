// Bassetti-Erskine kick of a transverse Gaussian and its potential-Hessian response on the device (FP64),
// for the analytic add-back of the Gaussian-subtracted hybrid (gaussian_pic.jl:818-884).
//
// Regimes follow the reference's response (src/elements/strong_beam.jl:640-1146): exactly round closed
// form; near-round series in eta = (s1^2 - s2^2)/(s1^2 + s2^2) below eta_*/2; quintic blend to the
// elliptic form up to eta_* = (8/3 * 64 * eps)^(1/4); elliptic Bassetti-Erskine through the Faddeeva
// function w(z), with its radial series near the axis.  w(z) is the N = 32 rational approximation of
// J. A. C. Weideman (SIAM J. Numer. Anal. 31, 1994) -- coefficients computed once on the host from the
// paper's construction -- and, far from the origin, the continued fraction of Poppe & Wijers (ACM TOMS
// 680) and the asymptotic i / (sqrt(pi) z) forms, switched where the reference's CUDA path switches
// (src/math/SpecialMath.jl:77-157).
#pragma once
#include "octo_internal.cuh"

namespace octo {

constexpr int kWeidemanN = 32;
__constant__ double c_weideman[kWeidemanN + 1];  // [0] = L, then the coefficients, highest power first

__device__ __forceinline__ void cdiv(double ar, double ai, double br, double bi, double &r, double &i) {
    const double inv = 1.0 / (br * br + bi * bi);
    r = (ar * br + ai * bi) * inv;
    i = (ai * br - ar * bi) * inv;
}

// w(z) for Im z >= 0 (the Bassetti-Erskine arguments are in the first quadrant).
__device__ __noinline__ void faddeeva_upper(double zr, double zi, double &wr, double &wi) {
    constexpr double kInvSqrtPi = 0.56418958354775628695;
    const double x = fabs(zr), y = zi;
    if (y > 7.0 || (x > 6.0 && (y > 0.1 || (x > 8.0 && y > 1e-10) || x > 28.0))) {
        if (x + y > 4000.0) {
            if (x + y > 1e7) {
                if (x > y) {
                    const double yax = y / zr, d = kInvSqrtPi / (zr + yax * y);
                    wr = d * yax; wi = d;
                } else {
                    const double xya = zr / y, d = kInvSqrtPi / (xya * zr + y);
                    wr = d; wi = d * xya;
                }
                return;
            }
            const double dr = zr * zr - y * y - 0.5, di = 2.0 * zr * y;
            const double d = kInvSqrtPi / (dr * dr + di * di);
            wr = d * (zr * di - y * dr);
            wi = d * (zr * dr + y * di);
            return;
        }
        double nu = floor(3.9 + 11.398 / (0.08254 * x + 0.1421 * y + 0.2023));
        double r = zr, i = y;
        nu = 0.5 * (nu - 1.0);
        for (int it = 0; it < 64 && nu > 0.4; ++it) {  // nu < 26 here: at most 13 steps
            const double inv = nu / (r * r + i * i);
            const double nr = zr - r * inv, ni = y + i * inv;
            r = nr; i = ni;
            nu -= 0.5;
        }
        const double inv = kInvSqrtPi / (r * r + i * i);
        wr = inv * i;
        wi = inv * r;
        return;
    }
    const double L = c_weideman[0];
    const double dr = L + zi, di = -zr, nr = L - zi, ni = zr;
    double Zr, Zi;
    cdiv(nr, ni, dr, di, Zr, Zi);
    double pr = 0.0, pi = 0.0;
    // Horner steps with fused multiply-adds (the polynomial's rounding, ~1e-16 relative, is far below the
    // approximation's own 3e-13)
#pragma unroll 8
    for (int k = 0; k < kWeidemanN; ++k) {
        const double tr = fma(pr, Zr, fma(-pi, Zi, c_weideman[1 + k]));
        const double ti = fma(pr, Zi, pi * Zr);
        pr = tr;
        pi = ti;
    }
    const double d2r = dr * dr - di * di, d2i = 2.0 * dr * di;
    double tr, ti, ir, ii;
    cdiv(2.0 * pr, 2.0 * pi, d2r, d2i, tr, ti);
    cdiv(kInvSqrtPi, 0.0, dr, di, ir, ii);
    wr = tr + ir;
    wi = ti + ii;
}

__device__ __forceinline__ void be_eta_bounds(double &inner, double &outer) {
    outer = sqrt(sqrt((8.0 / 3.0) * 64.0 * 2.220446049250313e-16));
    inner = outer / 2.0;
}

// m_k(q) = int_0^1 s^k exp(-q s) ds, k = k0 .. k0 + CNT - 1
template <int CNT>
__device__ __forceinline__ void be_moments(double q, int k0, double *m) {
    if (q <= 2.0) {
#pragma unroll
        for (int c = 0; c < CNT; ++c) m[c] = 0.0;
        double term = 1.0;
        for (int k = 0; k <= 24; ++k) {
#pragma unroll
            for (int c = 0; c < CNT; ++c) m[c] += term / (double)(k + k0 + c + 1);
            term *= -q / (double)(k + 1);
        }
        return;
    }
    const double eq = exp(-q);
    double mk = -expm1(-q) / q;
    for (int k = 0; k < k0 + CNT; ++k) {
        if (k >= k0) m[k - k0] = mk;
        mk = ((double)(k + 1) * mk - eq) / q;
    }
}

// L (optional): L / D of the rotation term, -x y / v^2 (m1 + eta dr m3 + eta^2 (1.5 m3 - q m4 + dr^2 m5 / 2))
// (strong_beam.jl:930-932).
__device__ __noinline__ void be_near_round(double kbb, double v, double eta, double x, double y, double &Kx, double &Ky,
                                           double &H1, double &H2, double *L = nullptr) {
    const double q = (x * x + y * y) / (2.0 * v);
    const double dr = (x * x - y * y) / (2.0 * v);
    double m[7];
    be_moments<7>(q, 0, m);
    const double eta2 = eta * eta, eta3 = eta2 * eta;
    const double u1 = dr * m[1];
    const double u2 = m[1] / 2.0 - q * m[2] + (dr * dr / 2.0) * m[3];
    const double u3 = 1.5 * dr * m[3] - dr * q * m[4] + dr * dr * dr / 6.0 * m[5];
    const double v1 = dr * (q * m[2] - m[1]);
    const double v2 = 1.5 * q * m[2] - (q * q + dr * dr) * m[3] + (q * dr * dr / 2.0) * m[4];
    const double v3 = -1.5 * dr * m[3] + 3.5 * dr * q * m[4] - (dr * q * q + dr * dr * dr / 2.0) * m[5] +
                      dr * dr * dr * q / 6.0 * m[6];
    const double c1x = dr * m[2] - m[1], c1y = dr * m[2] + m[1];
    const double c2x = 1.5 * m[2] + (-dr - q) * m[3] + (dr * dr / 2.0) * m[4];
    const double c2y = 1.5 * m[2] + (dr - q) * m[3] + (dr * dr / 2.0) * m[4];
    const double c3x = -1.5 * m[3] + (2.5 * dr + q) * m[4] + (-dr * q - dr * dr / 2.0) * m[5] + dr * dr * dr / 6.0 * m[6];
    const double c3y = 1.5 * m[3] + (2.5 * dr - q) * m[4] + (-dr * q + dr * dr / 2.0) * m[5] + dr * dr * dr / 6.0 * m[6];
    Kx = x / v * (m[0] + eta * c1x + eta2 * c2x + eta3 * c3x);
    Ky = y / v * (m[0] + eta * c1y + eta2 * c2y + eta3 * c3y);
    const double uv = -exp(-q) + eta * v1 + eta2 * v2 + eta3 * v3;
    const double ueta = u1 + 2.0 * eta * u2 + 3.0 * eta2 * u3;
    H1 = kbb / v * (uv + (1.0 - eta) * ueta);
    H2 = kbb / v * (uv - (1.0 + eta) * ueta);
    if (L) *L = -x * y / (v * v) * (m[1] + eta * dr * m[3] + eta2 * (1.5 * m[3] - q * m[4] + dr * dr / 2.0 * m[5]));
}

__device__ __noinline__ double be_near_round_residual(double v, double eta, double x, double y) {
    const double q = (x * x + y * y) / (2.0 * v);
    const double dr = (x * x - y * y) / (2.0 * v);
    double m[9];
    be_moments<9>(q, 3, m);
    const double m3 = m[0], m4 = m[1], m5 = m[2], m6 = m[3], m7 = m[4], m8 = m[5], m9 = m[6], m10 = m[7], m11 = m[8];
    const double dr2 = dr * dr, q2 = q * q;
    const double u4 = 3.0 / 8.0 * m3 - 1.5 * q * m4 + (5.0 * dr2 + 2.0 * q2) / 4.0 * m5 - dr2 * q / 2.0 * m6 +
                      dr2 * dr2 / 24.0 * m7;
    const double u5 = 15.0 / 8.0 * dr * m5 - 2.5 * dr * q * m6 + dr * (7.0 * dr2 + 6.0 * q2) / 12.0 * m7 -
                      dr * dr2 * q / 6.0 * m8 + dr * dr2 * dr2 / 120.0 * m9;
    const double u6 = 5.0 / 16.0 * m5 - 15.0 / 8.0 * q * m6 + 5.0 * (7.0 * dr2 + 4.0 * q2) / 16.0 * m7 -
                      q * (21.0 * dr2 + 2.0 * q2) / 12.0 * m8 + dr2 * (3.0 * dr2 + 4.0 * q2) / 16.0 * m9 -
                      dr2 * dr2 * q / 24.0 * m10 + dr2 * dr2 * dr2 / 720.0 * m11;
    return eta * eta * eta * eta * (u4 + eta * (u5 + eta * u6));
}

__device__ __forceinline__ bool be_near_axis(double s1, double s2, double x, double y, double eta) {
    const double rho2 = x * x / (s1 * s1) + y * y / (s2 * s2);
    return rho2 * rho2 * rho2 * sqrt(rho2) <= 2.220446049250313e-16 / sqrt(eta);
}

__device__ __forceinline__ void be_axis_series(double kbb, double sa, double sb, double a, double b, double &K,
                                               double &H) {
    const double s = sa + sb, sa2 = sa * sa, sa3 = sa2 * sa, sa5 = sa3 * sa2, sb2 = sb * sb, sb3 = sb2 * sb;
    const double s2 = s * s, s3 = s2 * s;
    const double j00 = 2.0 / (sa * s);
    const double j10 = 2.0 * (2.0 * sa + sb) / (3.0 * sa3 * s2);
    const double j01 = 2.0 / (sa * sb * s2);
    const double j20 = 2.0 * (8.0 * sa2 + 9.0 * sa * sb + 3.0 * sb2) / (15.0 * sa5 * s3);
    const double j11 = 2.0 * (3.0 * sa + sb) / (3.0 * sa3 * sb * s3);
    const double j02 = 2.0 * (sa + 3.0 * sb) / (3.0 * sa * sb3 * s3);
    const double a2 = a * a, b2 = b * b, a4 = a2 * a2, b4 = b2 * b2, a2b2 = a2 * b2;
    const double scale = j00 - (a2 * j10 + b2 * j01) / 2.0 + a4 * j20 / 8.0 + a2b2 * j11 / 4.0 + b4 * j02 / 8.0;
    const double der = j00 - 1.5 * a2 * j10 - b2 * j01 / 2.0 + 0.625 * a4 * j20 + 0.75 * a2b2 * j11 + b4 * j02 / 8.0;
    K = a * scale;
    H = -kbb * der;
}

__device__ __noinline__ void be_elliptic(double s1, double s2, double x, double y, double eta, double &Kx, double &Ky) {
    if (be_near_axis(s1, s2, x, y, eta)) {
        double h;
        be_axis_series(0.0, s1, s2, x, y, Kx, h);
        be_axis_series(0.0, s2, s1, y, x, Ky, h);
        return;
    }
    const bool negx = x < 0, negy = y < 0;
    const double ax = fabs(x), ay = fabs(y);
    const double den = 1.4142135623730951 * sqrt(s1 * s1 - s2 * s2);
    const double A = 2.0 * 1.7724538509055159 / den;
    const double B = exp(-ax * ax / (2.0 * s1 * s1) - ay * ay / (2.0 * s2 * s2));
    double w1r, w1i, w2r, w2i;
    faddeeva_upper(ax / den, ay / den, w1r, w1i);
    faddeeva_upper(s2 / s1 * ax / den, s1 / s2 * ay / den, w2r, w2i);
    const double rr = A * (w1r - B * w2r), ri = A * (w1i - B * w2i);
    Kx = negx ? -ri : ri;
    Ky = negy ? -rr : rr;
}

// Principal-axis response (s1 >= s2): kick and kbb-scaled potential Hessians.
// L (optional): L / D, the rotation term's response (strong_beam.jl:1061-1116).
__device__ __noinline__ void be_response_principal(double kbb, double s1, double s2, double x, double y, double &Kx,
                                                   double &Ky, double &H1, double &H2, double *L = nullptr) {
    const double v = (s1 * s1 + s2 * s2) / 2.0;
    const double eta = (s1 * s1 - s2 * s2) / (2.0 * v);
    if (eta == 0.0) {
        const double r2 = x * x + y * y;
        if (L) {  // the eta -> 0 limit, -x y m1(q) / v^2
            double mm[2];
            be_moments<2>(r2 / (2.0 * v), 0, mm);
            *L = -x * y / (v * v) * mm[1];
        }
        const double u0 = r2 / (2.0 * v);
        const double phi0 = u0 == 0.0 ? 1.0 : -expm1(-u0) / u0;
        Kx = phi0 / v * x;
        Ky = phi0 / v * y;
        const double expterm = exp(-r2 / (2.0 * v));
        const double sg = sqrt(v), sigma2 = sg * sg;
        if (r2 == 0.0) {
            H1 = H2 = -kbb / sigma2;
            return;
        }
        const double u = r2 / (2.0 * sigma2);
        double f, fp;
        if (u < 1.0e-2) {
            const double ph = 1.0 + u * (-1.0 / 2 + u * (1.0 / 6 + u * (-1.0 / 24 + u * (1.0 / 120 + u * (-1.0 / 720 + u * (1.0 / 5040))))));
            const double dph = -1.0 / 2 + u * (1.0 / 3 + u * (-1.0 / 8 + u * (1.0 / 30 + u * (-1.0 / 144 + u * (1.0 / 840 - u * (1.0 / 5760))))));
            const double inv = 1.0 / sigma2;
            f = ph * inv;
            fp = dph * inv * inv / 2;
        } else {
            const double ome = 1 - expterm;
            f = 2 * ome / r2;
            fp = 2 * (expterm * u - ome) / (r2 * r2);
        }
        H1 = -kbb * (f + 2 * x * x * fp);
        H2 = -kbb * (f + 2 * y * y * fp);
        return;
    }
    double inner, outer;
    be_eta_bounds(inner, outer);
    if (eta <= inner) {
        be_near_round(kbb, v, eta, x, y, Kx, Ky, H1, H2, L);
        return;
    }
    double Kex, Key, He1, He2;
    be_elliptic(s1, s2, x, y, eta, Kex, Key);
    const double Le = (Kex * y - Key * x) / (2.0 * v * eta);
    const double expterm = exp(-0.5 * (x * x / (s1 * s1) + y * y / (s2 * s2)));
    if (be_near_axis(s1, s2, x, y, eta)) {
        double k;
        be_axis_series(kbb, s1, s2, x, y, k, He1);
        be_axis_series(kbb, s2, s1, y, x, k, He2);
    } else {
        const double t1 = kbb * (x * Kex + y * Key), t2 = s1 * s1 - s2 * s2, t3 = s2 / s1;
        He1 = (t1 - 2 * kbb * (1 - expterm * t3)) / t2;
        He2 = (-t1 + 2 * kbb * (1 - expterm / t3)) / t2;
    }
    if (eta >= outer) {
        Kx = Kex; Ky = Key; H1 = He1; H2 = He2;
        if (L) *L = Le;
        return;
    }
    const double invw = 1.0 / (outer - inner), t = (eta - inner) * invw;
    const double w = t * t * t * (10.0 + t * (-15.0 + 6.0 * t));
    const double dw = 30.0 * t * t * (t - 1.0) * (t - 1.0) * invw;
    double Ksx, Ksy, Hs1, Hs2, Ls;
    be_near_round(kbb, v, eta, x, y, Ksx, Ksy, Hs1, Hs2, &Ls);
    const double chain = kbb * dw * be_near_round_residual(v, eta, x, y) / v;
    Kx = Ksx + w * (Kex - Ksx);
    Ky = Ksy + w * (Key - Ksy);
    H1 = Hs1 + w * (He1 - Hs1) + (1.0 - eta) * chain;
    H2 = Hs2 + w * (He2 - Hs2) - (1.0 + eta) * chain;
    if (L) *L = Ls + w * (Le - Ls);
}

// Round Gaussian of size sigma: the kick (gaussian_beambeam_kick, strong_beam.jl:1139-1146 with eta = 0) and the
// full potential Hessian (_round_gaussian_hessian, :711-763), for the coupled kick's D = 0 case.
__device__ __noinline__ void be_round(double kbb, double sigma, double x, double y, double expterm, double &Kx,
                                      double &Ky, double &Hxx, double &Hxy, double &Hyy) {
    Kx = Ky = 0.0;
    if (sigma != 0.0) {
        const double v = (sigma * sigma + sigma * sigma) / 2.0;
        const double r2 = x * x + y * y;
        const double u0 = r2 / (2.0 * v);
        const double phi0 = u0 == 0.0 ? 1.0 : -expm1(-u0) / u0;
        Kx = phi0 / v * x;
        Ky = phi0 / v * y;
    }
    const double r2 = x * x + y * y, sigma2 = sigma * sigma;
    if (r2 == 0.0) {
        Hxx = Hyy = -kbb / sigma2;
        Hxy = 0.0;
        return;
    }
    const double u = r2 / (2.0 * sigma2);
    double f, fp;
    if (u < 1.0e-2) {
        const double ph = 1.0 + u * (-1.0 / 2 + u * (1.0 / 6 + u * (-1.0 / 24 + u * (1.0 / 120 + u * (-1.0 / 720 + u * (1.0 / 5040))))));
        const double dph = -1.0 / 2 + u * (1.0 / 3 + u * (-1.0 / 8 + u * (1.0 / 30 + u * (-1.0 / 144 + u * (1.0 / 840 - u * (1.0 / 5760))))));
        const double inv = 1.0 / sigma2;
        f = ph * inv;
        fp = dph * inv * inv / 2;
    } else {
        const double ome = 1 - expterm;
        f = 2 * ome / r2;
        fp = 2 * (expterm * u - ome) / (r2 * r2);
    }
    Hxx = -kbb * (f + 2 * x * x * fp);
    Hxy = -kbb * (2 * x * y * fp);
    Hyy = -kbb * (f + 2 * y * y * fp);
}

__device__ __forceinline__ void be_response(double kbb, double sigx, double sigy, double x, double y, double &Kx,
                                            double &Ky, double &Hx, double &Hy) {
    if (sigx >= sigy) be_response_principal(kbb, sigx, sigy, x, y, Kx, Ky, Hx, Hy);
    else be_response_principal(kbb, sigy, sigx, y, x, Ky, Kx, Hy, Hx);
}

// Transverse moments of a Gaussian: its centroid (unused by the kick) and the covariance entries of
// StrongTransverseMoments (strong_beam.jl:79-90).  Shared by the soft-Gaussian solver and the coupled
// add-back of the Gaussian-subtracted hybrid.
struct GMoments {
    double mx, mpx, my, mpy;            // zero when the beam's centroid is ignored
    double a0, d0, bxx, bypy, qxx, qyy; // var x, var y, cov(x, px), cov(y, py), var px, var py
    double b0, bxpy, bypx, qxy;         // coupled: cov(x, y), cov(x, py), cov(px, y), cov(px, py); else zero
};

// The coupled _cp_covariance_kick (strong_beam.jl:634-682): the transported covariance's principal axes, the
// rotated kick and potential Hessians, the covariance pz term and the rotation term L / D.
__device__ __noinline__ void coupled_kick(const GMoments &M, double kbb, double S, double xx, double yy, double &px,
                                          double &py, double &pz, double &density) {
    const double a = M.a0 - 2 * S * M.bxx + S * S * M.qxx;
    const double b = M.b0 - S * (M.bxpy + M.bypx) + S * S * M.qxy;
    const double d = M.d0 - 2 * S * M.bypy + S * S * M.qyy;
    const double au = 2 * (M.bxx - S * M.qxx);
    const double bu = M.bxpy + M.bypx - 2 * S * M.qxy;
    const double du = 2 * (M.bypy - S * M.qyy);
    const double detA = a * d - b * b;
    const double twopi = 6.283185307179586476925286766559005768394338;
    density = 0.0;
    if (a <= 0 || d <= 0 || detA <= 0) return;
    const double adiff = a - d;
    const double D = hypot(adiff, 2 * b);
    if (D == 0.0) {
        const double sigma = sqrt((a + d) / 2);
        const double expterm = exp(-0.5 * (xx * xx + yy * yy) / (sigma * sigma));
        double Kx, Ky, Hxx, Hxy, Hyy;
        be_round(kbb, sigma, xx, yy, expterm, Kx, Ky, Hxx, Hxy, Hyy);
        px += kbb * Kx;
        py += kbb * Ky;
        pz += 0.25 * (Hxx * au + 2 * Hxy * bu + Hyy * du);
        density = expterm / (twopi * sigma * sigma);
        return;
    }
    const double theta = 0.5 * atan2(2 * b, a - d);
    double sn, cs;
    sincos(theta, &sn, &cs);
    const double lambda1 = (a + d + D) / 2, lambda2 = (a + d - D) / 2;
    const double sig1 = sqrt(lambda1), sig2 = sqrt(lambda2);
    const double xh = cs * xx + sn * yy;
    const double yh = -sn * xx + cs * yy;
    const double eta = D / (a + d);
    double inner, outer;
    be_eta_bounds(inner, outer);
    double Kxh, Kyh, H11, H22, LoD;
    if (eta <= inner) be_near_round(kbb, (a + d) / 2, eta, xh, yh, Kxh, Kyh, H11, H22, &LoD);
    else be_response_principal(kbb, sig1, sig2, xh, yh, Kxh, Kyh, H11, H22, &LoD);
    const double expterm = exp(-0.5 * (xh * xh / lambda1 + yh * yh / lambda2));
    const double Fxh = kbb * Kxh, Fyh = kbb * Kyh;
    px += cs * Fxh - sn * Fyh;
    py += sn * Fxh + cs * Fyh;
    const double Du = (adiff * (au - du) + 4 * b * bu) / D;
    const double traceu = au + du;
    pz += 0.125 * ((H11 + H22) * traceu + (H11 - H22) * Du);
    const double rotation_projection = (adiff * bu - b * (au - du)) / D;
    pz -= 0.5 * kbb * rotation_projection * LoD;
    density = expterm / (twopi * sig1 * sig2);
}

}  // namespace octo
