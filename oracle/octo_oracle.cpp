// FP64 CPU oracle for the strong-strong PIC collision -- TEST INFRASTRUCTURE ONLY.
//
// A plain restatement of the reference's CPU path, used to check the CUDA
// library: tests, the smoke check and the CPU-baseline leg of the benchmark
// call it; the product never links it.  Every function cites the reference
// file:line it follows (paths relative to the Octopus.jl checkout).
//
// Arithmetic is IEEE FP64 with no contraction (built with -ffp-contract=off),
// evaluated in the reference's own left-to-right order, so scalar decisions
// (grid geometry, Green-cache hits) reproduce the reference bit for bit.  The
// FFT is this file's own (the reference calls FFTW 3.3.12), so field values
// agree with the reference to rounding, not bitwise.
#include "oracle.h"
#include "oracle_be.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

struct OracleError : std::runtime_error {
    int code;
    OracleError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Julia's IEEE min/max: NaN-propagating, -0.0 < +0.0 (base/math.jl semantics).
inline double jmin(double a, double b) {
    if (std::isnan(a) || std::isnan(b)) return a - b;
    if (a < b) return a;
    if (b < a) return b;
    return std::signbit(a) ? a : b;
}
inline double jmax(double a, double b) {
    if (std::isnan(a) || std::isnan(b)) return a - b;
    if (a > b) return a;
    if (b > a) return b;
    return std::signbit(a) ? b : a;
}
// Julia clamp(x, lo, hi) = ifelse(x > hi, hi, ifelse(x < lo, lo, x)).
inline double jclamp(double x, double lo, double hi) { return x > hi ? hi : (x < lo ? lo : x); }
inline long jclampi(long v, long lo, long hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------- counter RNG
// counter_rng.jl:187-233, 341-349, 154-166, 410-430.
const uint32_t PH_M0 = 0xD2511F53u, PH_M1 = 0xCD9E8D57u, PH_W0 = 0x9E3779B9u, PH_W1 = 0xBB67AE85u;

inline uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

inline void philox_block(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)PH_M0 * c[0];
        uint64_t p1 = (uint64_t)PH_M1 * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += PH_W0; k1 += PH_W1;
    }
}

inline uint64_t counter_u64(uint64_t seed, uint64_t turn, uint64_t rng_id, uint64_t particle, uint64_t comp) {
    uint32_t c[4] = {(uint32_t)particle, (uint32_t)(particle >> 32), (uint32_t)turn, (uint32_t)(turn >> 32)};
    uint64_t key = splitmix64(seed) ^ splitmix64(rng_id + 0x9e3779b97f4a7c15ULL) ^
                   splitmix64(comp + 0xbf58476d1ce4e5b9ULL);
    philox_block(c, (uint32_t)key, (uint32_t)(key >> 32));
    return ((uint64_t)c[0] << 32) | (uint64_t)c[1];
}

inline double uniform_open01(uint64_t v) {
    uint64_t bits = v >> 12;
    return ((double)bits + 0.5) * 2.220446049250313e-16;
}

inline double counter_normal(uint64_t seed, uint64_t turn, uint64_t rng_id, uint64_t particle, uint64_t comp) {
    uint64_t pair = (comp + 1) / 2;
    double u1 = uniform_open01(counter_u64(seed, turn, rng_id, particle, 2 * pair - 1));
    double u2 = uniform_open01(counter_u64(seed, turn, rng_id, particle, 2 * pair));
    double r = std::sqrt(-2.0 * std::log(u1));
    double theta = 6.283185307179586476925286766559 * u2;
    return (comp & 1) ? r * std::cos(theta) : r * std::sin(theta);
}

// Pairwise sum in the shape of Julia's `sum` (blocks of 1024, split in halves).
double pairwise_sum(const double *v, int64_t n) {
    if (n <= 1024) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += v[i];
        return s;
    }
    int64_t h = n >> 1;
    return pairwise_sum(v, h) + pairwise_sum(v + h, n - h);
}

// Beam.jl:148-160
void standardize(double *v, int64_t n) {
    double mu = pairwise_sum(v, n) / (double)n;
    for (int64_t i = 0; i < n; ++i) v[i] -= mu;
    std::vector<double> sq(n);
    for (int64_t i = 0; i < n; ++i) sq[i] = v[i] * v[i];
    double s2 = pairwise_sum(sq.data(), n) / (double)n;
    double s = std::sqrt(std::max(s2, 0.0));
    if (s == 0.0) {
        for (int64_t i = 0; i < n; ++i) v[i] = 0.0;
    } else {
        for (int64_t i = 0; i < n; ++i) v[i] /= s;
    }
}

// ------------------------------------------------------------------ erfinv
// Inverse error function: Winitzki's closed-form start refined by Halley steps on
// erf (|x| < 0.5) or erfc (|x| >= 0.5).  Replaces SpecialFunctions.erfinv
// (SpecialMath.jl:174), which the reference calls in slicing.jl:425.
double erfinv_impl(double x) {
    if (std::isnan(x) || x < -1.0 || x > 1.0) return NAN;
    if (x == 1.0) return INFINITY;
    if (x == -1.0) return -INFINITY;
    if (x == 0.0) return x;
    double ax = std::fabs(x);
    const double a = 0.147, pi = 3.141592653589793;
    double ln = std::log1p(-ax * ax);
    double t1 = 2.0 / (pi * a) + ln / 2.0;
    double y = std::sqrt(std::sqrt(t1 * t1 - ln / a) - t1);
    const double two_over_sqrtpi = 1.1283791670955126;
    for (int it = 0; it < 4; ++it) {
        double f = (ax < 0.5) ? (std::erf(y) - ax) : ((1.0 - ax) - std::erfc(y));
        double fp = two_over_sqrtpi * std::exp(-y * y);
        double step = f / fp;
        y = y - step / (1.0 + y * step);
    }
    return x < 0 ? -y : y;
}

// ------------------------------------------------------------------ FFT
// Own FFT (replaces FFTW.jl 1.10.0 / FFTW 3.3.12; call sites pic_cpu.jl:1954-1983).
struct Fft1D {
    int n = 0;
    bool pow2 = false;
    std::vector<cplx> w;      // exp(-2 pi i k / n)
    std::vector<int> rev;
    std::vector<cplx> tmp;
    void init(int n_) {
        n = n_;
        w.resize(n);
        for (int k = 0; k < n; ++k) {
            double a = -2.0 * 3.141592653589793238462643 * (double)k / (double)n;
            w[k] = cplx(std::cos(a), std::sin(a));
        }
        pow2 = (n & (n - 1)) == 0;
        if (pow2) {
            rev.resize(n);
            int lg = 0;
            while ((1 << lg) < n) ++lg;
            for (int i = 0; i < n; ++i) {
                int r = 0;
                for (int b = 0; b < lg; ++b)
                    if (i & (1 << b)) r |= 1 << (lg - 1 - b);
                rev[i] = r;
            }
        }
        tmp.resize(n);
    }
    // Recursive mixed-radix DIT for sizes 2^a 3^b 5^c (generic DFT otherwise).
    void rec(const cplx *in, int stride, cplx *out, int m, bool inv) {
        if (m == 1) { out[0] = in[0]; return; }
        int r = (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5 : m;
        int q = m / r;
        for (int p = 0; p < r; ++p) rec(in + p * stride, stride * r, out + p * q, q, inv);
        int step = n / m;
        cplx buf[16];
        std::vector<cplx> big;
        cplx *b = buf;
        if (r > 16) { big.resize(r); b = big.data(); }
        for (int k = 0; k < q; ++k) {
            for (int p = 0; p < r; ++p) {
                int e = (int)(((long)p * k * step) % n);
                cplx tw = inv ? std::conj(w[e]) : w[e];
                b[p] = out[p * q + k] * tw;
            }
            for (int mm = 0; mm < r; ++mm) {
                cplx s = 0;
                for (int p = 0; p < r; ++p) {
                    int e = (int)(((long)p * mm * q * step) % n);
                    cplx tw = inv ? std::conj(w[e]) : w[e];
                    s += b[p] * tw;
                }
                out[mm * q + k] = s;
            }
        }
    }
    void run(cplx *a, bool inv) {
        if (pow2) {
            for (int i = 0; i < n; ++i)
                if (i < rev[i]) std::swap(a[i], a[rev[i]]);
            for (int len = 2; len <= n; len <<= 1) {
                int half = len >> 1, step = n / len;
                for (int i = 0; i < n; i += len)
                    for (int j = 0; j < half; ++j) {
                        cplx tw = inv ? std::conj(w[j * step]) : w[j * step];
                        cplx u = a[i + j], v = a[i + j + half] * tw;
                        a[i + j] = u + v;
                        a[i + j + half] = u - v;
                    }
            }
        } else {
            std::vector<cplx> in(a, a + n);
            rec(in.data(), 1, a, n, inv);
        }
    }
};

struct Fft2D {
    int n1 = 0, n2 = 0;
    Fft1D f1, f2;
    std::vector<cplx> line;
    void init(int a, int b) {
        n1 = a; n2 = b;
        f1.init(a); f2.init(b);
        line.resize(b);
    }
    // Column-major (n1 fastest), unnormalised forward / 1/(n1 n2)-normalised inverse like FFTW's ifft.
    void run(cplx *a, bool inv) {
        for (int j = 0; j < n2; ++j) f1.run(a + (size_t)j * n1, inv);
        for (int i = 0; i < n1; ++i) {
            for (int j = 0; j < n2; ++j) line[j] = a[i + (size_t)j * n1];
            f2.run(line.data(), inv);
            for (int j = 0; j < n2; ++j) a[i + (size_t)j * n1] = line[j];
        }
        if (inv) {
            double s = 1.0 / ((double)n1 * (double)n2);
            for (size_t k = 0; k < (size_t)n1 * n2; ++k) a[k] *= s;
        }
    }
};

// ----------------------------------------------------------- PIC primitives
// pic_cpu.jl:2182-2197
inline void cic_weights(double u, int n, int &base, double w[2]) {
    if (!(0.0 <= u && u <= (double)(n - 1))) { base = 1; w[0] = 0.0; w[1] = 0.0; return; }
    base = (int)jclampi((long)std::floor(u) + 1, 1, n - 1);
    double f = jclamp(u - (double)(base - 1), 0.0, 1.0);
    w[0] = 1.0 - f; w[1] = f;
}

// pic_cpu.jl:2225-2252
inline void tsc_weights(double u, int n, int &base, double w[3]) {
    if (!(0.0 <= u && u <= (double)(n - 1))) { base = 1; w[0] = w[1] = w[2] = 0.0; return; }
    double fl = std::floor(u);
    long ix = (long)fl;
    double f = u - fl;
    long b;
    if (f < 0.5) {
        double t = f * f;
        w[0] = 0.125 + 0.5 * (t - f); w[1] = 0.75 - t; w[2] = 0.125 + 0.5 * (t + f);
        b = ix;
    } else {
        double fr = 1.0 - f;
        double t = fr * fr;
        w[0] = 0.125 + 0.5 * (t + fr); w[1] = 0.75 - t; w[2] = 0.125 + 0.5 * (t - fr);
        b = ix + 1;
    }
    base = (int)jclampi(b, 1, n - 2);
}

// pic_cpu.jl:2254-2272
inline double atan_ratio(double num, double den) {
    if (den == 0) {
        if (num == 0) return 0.0;
        return std::copysign(3.141592653589793 / 2, num);
    }
    return std::atan(num / den);
}
inline double kernel_integral(double x, double y) {
    double r2 = x * x + y * y;
    if (r2 == 0.0) return 0.0;
    return (std::log(r2) - 3) * x * y + atan_ratio(y, x) * x * x + atan_ratio(x, y) * y * y;
}

// pic_cpu.jl:2478-2509 (integrated / standard kernels)
void green_table(int green_type, double fx0, double fy0, double sx0, double sy0, double hx, double hy, int nx, int ny,
                 double *g) {
    double half_hx = hx / 2, half_hy = hy / 2;
    double hxihyi = -0.5 / (hx * hy);
    for (int j = 0; j < 2 * ny; ++j)
        for (int i = 0; i < 2 * nx; ++i) {
            int ii = i < nx ? i : i - 2 * nx;
            int jj = j < ny ? j : j - 2 * ny;
            double x = fx0 - sx0 + (double)ii * hx;
            double y = fy0 - sy0 + (double)jj * hy;
            double val;
            bool integrated = green_type == 0;
            if (!integrated) {
                double r2 = x * x + y * y;
                if (r2 != 0.0) { g[i + (size_t)j * 2 * nx] = -0.5 * std::log(r2); continue; }
            }
            val = kernel_integral(x + half_hx, y + half_hy);
            val += kernel_integral(x - half_hx, y - half_hy);
            val -= kernel_integral(x + half_hx, y - half_hy);
            val -= kernel_integral(x - half_hx, y + half_hy);
            g[i + (size_t)j * 2 * nx] = hxihyi * val;
        }
}

// pic_cpu.jl:2531-2591
void field_from_phi(const double *phi, int nx, int ny, double hx, double hy, bool fourth, double *Ex, double *Ey) {
    auto P = [&](int i, int j) { return phi[(i - 1) + (size_t)(j - 1) * nx]; };
    auto EX = [&](int i, int j) -> double & { return Ex[(i - 1) + (size_t)(j - 1) * nx]; };
    auto EY = [&](int i, int j) -> double & { return Ey[(i - 1) + (size_t)(j - 1) * nx]; };
    double hxi = 1.0 / hx, hyi = 1.0 / hy;
    double c4 = 1.0 / 12.0;
    for (int i = 1; i <= nx; ++i) {
        EY(i, 1) = hyi * (1.5 * P(i, 1) - 2 * P(i, 2) + 0.5 * P(i, 3));
        EY(i, ny) = hyi * (-1.5 * P(i, ny) + 2 * P(i, ny - 1) - 0.5 * P(i, ny - 2));
    }
    if (fourth && ny >= 5) {
        for (int i = 1; i <= nx; ++i) {
            EY(i, 2) = 0.5 * hyi * (P(i, 1) - P(i, 3));
            EY(i, ny - 1) = 0.5 * hyi * (P(i, ny - 2) - P(i, ny));
        }
        for (int j = 3; j <= ny - 2; ++j)
            for (int i = 1; i <= nx; ++i)
                EY(i, j) = c4 * hyi * ((P(i, j + 2) - P(i, j - 2)) + 8 * (P(i, j - 1) - P(i, j + 1)));
    } else {
        for (int j = 2; j <= ny - 1; ++j)
            for (int i = 1; i <= nx; ++i) EY(i, j) = 0.5 * hyi * (P(i, j - 1) - P(i, j + 1));
    }
    for (int j = 1; j <= ny; ++j) {
        EX(1, j) = hxi * (1.5 * P(1, j) - 2 * P(2, j) + 0.5 * P(3, j));
        EX(nx, j) = hxi * (-1.5 * P(nx, j) + 2 * P(nx - 1, j) - 0.5 * P(nx - 2, j));
        if (fourth && nx >= 5) {
            EX(2, j) = 0.5 * hxi * (P(1, j) - P(3, j));
            EX(nx - 1, j) = 0.5 * hxi * (P(nx - 2, j) - P(nx, j));
            for (int i = 3; i <= nx - 2; ++i)
                EX(i, j) = c4 * hxi * ((P(i + 2, j) - P(i - 2, j)) + 8 * (P(i - 1, j) - P(i + 1, j)));
        } else {
            for (int i = 2; i <= nx - 1; ++i) EX(i, j) = 0.5 * hxi * (P(i - 1, j) - P(i + 1, j));
        }
    }
}

// Fixed-point charge scale: every tap is rounded to a multiple of 2^-bits, with bits chosen so the
// full source population fits a cell without overflow: bits = min(40, 62 - bitlength(nsrc)).
inline int fixed_bits(int64_t n) {
    int bl = 0;
    uint64_t v = (uint64_t)(n < 1 ? 1 : n);
    while (v) { ++bl; v >>= 1; }
    int b = 62 - bl;
    return b > 40 ? 40 : b;
}

struct Grid { double x0, y0, width, height; };
struct Bounds { double xmin, xmax, ymin, ymax; };

constexpr int DEPOSIT_CHUNKS = 16;           // interface.jl:663
constexpr int64_t PARALLEL_DEPOSIT_MIN = 4096;  // interface.jl:615
constexpr int64_t DEPOSIT_PER_CELL = 160;    // interface.jl:643
constexpr double TEMPLATE_MARGIN_CELLS = 1.5;  // interface.jl:674
constexpr int SLICE_FOLD_LANES = 4096;       // slicing.jl:223

inline bool deposit_parallel(int64_t n, int nx, int ny) {  // interface.jl:649-651
    return n >= PARALLEL_DEPOSIT_MIN && n >= DEPOSIT_PER_CELL * (int64_t)nx * ny;
}

// One particle's taps into a column-major grid with leading dimension ld (pic_cpu.jl:2129-2146).
template <class Acc>
inline void deposit_point(int method, double u, double v, int nx, int ny, Acc acc) {
    if (method == 0) {
        int ix, iy; double wx[2], wy[2];
        cic_weights(u, nx, ix, wx);
        cic_weights(v, ny, iy, wy);
        for (int m = 0; m < 2; ++m)
            for (int k = 0; k < 2; ++k) acc(ix + m, iy + k, wx[m] * wy[k]);
    } else {
        int ix, iy; double wx[3], wy[3];
        tsc_weights(u, nx, ix, wx);
        tsc_weights(v, ny, iy, wy);
        for (int m = 0; m < 3; ++m)
            for (int k = 0; k < 3; ++k) acc(ix + m, iy + k, wx[m] * wy[k]);
    }
}

// pic_cpu.jl:2015-2146: serial below the chunk threshold, 16 fixed chunk grids above it.
// drift=true deposits x + px*s; otherwise x (px unused).  fixed: int64 fixed-point accumulation.
void deposit_grid(double *charge, int ld, int method, const double *x, const double *px, const double *y,
                  const double *py, int64_t n, bool drift, double s, double x0, double y0, double hx, double hy,
                  int nx, int ny, bool fixed, int64_t *qfix) {
    double hxi = 1.0 / hx, hyi = 1.0 / hy;
    auto pos = [&](int64_t i, double &u, double &v) {
        double xd = drift ? x[i] + px[i] * s : x[i];
        double yd = drift ? y[i] + py[i] * s : y[i];
        u = (xd - x0) * hxi;
        v = (yd - y0) * hyi;
    };
    if (fixed) {
        int bits = fixed_bits(n);
        double scale = std::ldexp(1.0, bits);
        std::vector<int64_t> q((size_t)ld * (ny + 2), 0);
        for (int64_t i = 0; i < n; ++i) {
            double u, v;
            pos(i, u, v);
            deposit_point(method, u, v, nx, ny, [&](int a, int b, double w) {
                q[(a - 1) + (size_t)(b - 1) * ld] += (int64_t)std::nearbyint(w * scale);
            });
        }
        double inv = std::ldexp(1.0, -bits);
        for (int b = 0; b < ny; ++b)
            for (int a = 0; a < nx; ++a) {
                int64_t val = q[a + (size_t)b * ld];
                charge[a + (size_t)b * ld] += (double)val * inv;
                if (qfix) qfix[a + (size_t)b * nx] = val;
            }
        return;
    }
    if (deposit_parallel(n, nx, ny)) {
        std::vector<double> local((size_t)ld * (ny + 2));
        for (int c = 1; c <= DEPOSIT_CHUNKS; ++c) {
            std::fill(local.begin(), local.end(), 0.0);
            int64_t lo = ((int64_t)(c - 1) * n) / DEPOSIT_CHUNKS, hi = ((int64_t)c * n) / DEPOSIT_CHUNKS;
            for (int64_t i = lo; i < hi; ++i) {
                double u, v;
                pos(i, u, v);
                deposit_point(method, u, v, nx, ny,
                              [&](int a, int b, double w) { local[(a - 1) + (size_t)(b - 1) * ld] += w; });
            }
            for (int b = 0; b < ny; ++b)
                for (int a = 0; a < nx; ++a) charge[a + (size_t)b * ld] += local[a + (size_t)b * ld];
        }
        return;
    }
    for (int64_t i = 0; i < n; ++i) {
        double u, v;
        pos(i, u, v);
        deposit_point(method, u, v, nx, ny,
                      [&](int a, int b, double w) { charge[(a - 1) + (size_t)(b - 1) * ld] += w; });
    }
}

struct Coords {
    std::vector<double> x, px, y, py, z, pz;
    size_t size() const { return x.size(); }
    void resize(size_t n) { x.resize(n); px.resize(n); y.resize(n); py.resize(n); z.resize(n); pz.resize(n); }
};

struct Options {
    oo_options o;
    std::vector<double> pos1, pos2;
    int lum_nx() const { return o.lum_nx > 0 ? o.lum_nx : o.nx; }
    int lum_ny() const { return o.lum_ny > 0 ? o.lum_ny : o.ny; }
    int lum_method() const { return o.lum_deposit_method >= 0 ? o.lum_deposit_method : o.deposit_method; }
};

// pic_cpu.jl:1646-1672
void resolve_extent(const Options &O, double xspan, double yspan, double &w, double &h, const char *context) {
    w = jmax(xspan, O.o.min_extent_x);
    h = jmax(yspan, O.o.min_extent_y);
    if (!(std::isfinite(w) && std::isfinite(h) && w > 0 && h > 0)) {
        char buf[256];
        snprintf(buf, sizeof buf, "%s requires finite, positive transverse extents; observed (x=%g, y=%g)", context,
                 xspan, yspan);
        throw OracleError(OO_ERR_EXTENT, buf);
    }
}

// pic_cpu.jl:1877-1905
void align_origins(int green_type, double s0, double f0, double h, double &so, double &fo) {
    double f1 = s0 / h - std::floor(s0 / h);
    double f2 = f0 / h - std::floor(f0 / h);
    double t = (f2 - f1) / 2;
    if (green_type == 1) {
        t += t > 0 ? -0.25 : 0.25;
    } else {
        if (t > 0.5) t -= 0.5;
        else if (t < -0.5) t += 0.5;
    }
    double shift = t * h;
    so = s0 + shift;
    fo = f0 - shift;
}

inline double quantize_extent(double w, double q) {  // pic_cpu.jl:1641-1644
    if (!(q > 0 && std::isfinite(w) && w > 0)) return w;
    return std::exp2(std::ceil(std::log2(w) / q) * q);
}

// pic_cpu.jl:1674-1718
void interaction_grids(const Options &O, double sxmin, double sxmax, double symin, double symax, double fxmin,
                       double fxmax, double fymin, double fymax, Grid &sg, Grid &fg) {
    int nx = O.o.nx, ny = O.o.ny;
    double width, height;
    resolve_extent(O, jmax(sxmax - sxmin, fxmax - fxmin), jmax(symax - symin, fymax - fymin), width, height,
                   "PIC interaction grid");
    double tx = width / (double)(nx - 4);
    double ty = height / (double)(ny - 4);
    width += 3 * tx;
    height += 3 * ty;
    double q = O.o.grid_quantize;
    if (q > 0) {
        width = quantize_extent(width, q);
        height = quantize_extent(height, q);
        double hx = width / (double)(nx - 1), hy = height / (double)(ny - 1);
        double sx0 = std::nearbyint(((sxmin + sxmax) / 2 - width / 2) / hx) * hx;
        double sy0 = std::nearbyint(((symin + symax) / 2 - height / 2) / hy) * hy;
        double fx0 = std::nearbyint(((fxmin + fxmax) / 2 - width / 2) / hx) * hx;
        double fy0 = std::nearbyint(((fymin + fymax) / 2 - height / 2) / hy) * hy;
        align_origins(O.o.green_type, sx0, fx0, hx, sx0, fx0);
        align_origins(O.o.green_type, sy0, fy0, hy, sy0, fy0);
        sg = {sx0, sy0, width, height};
        fg = {fx0, fy0, width, height};
        return;
    }
    double sx0 = sxmin - 1.5 * tx, sy0 = symin - 1.5 * ty;
    double fx0 = fxmin - 1.5 * tx, fy0 = fymin - 1.5 * ty;
    align_origins(O.o.green_type, sx0, fx0, tx, sx0, fx0);
    align_origins(O.o.green_type, sy0, fy0, ty, sy0, fy0);
    sg = {sx0, sy0, width, height};
    fg = {fx0, fy0, width, height};
}

// pic_cpu.jl:1581-1593 and slicing.jl:667-668
inline void axis_extent(int method, double &lo, double &hi, double origin, double ds, double ds2, int64_t n,
                        double k) {
    if (method == 0 || n < 2) return;
    double invn = 1.0 / (double)n;
    double mean_offset = ds * invn;
    double m = origin + mean_offset;
    // muladd(-a, a, b) (slicing.jl:667-668) is fused on FMA-capable hosts.
    double var = jmax(std::fma(-mean_offset, mean_offset, ds2 * invn), 0.0);
    double sd = std::sqrt(var);
    double half = k * sd;
    if (!(half > 0)) return;
    lo = m - half;
    hi = m + half;
}

struct FieldPlanes { std::vector<double> phi, Ex, Ey; void init(int n) { phi.assign(n, 0); Ex.assign(n, 0); Ey.assign(n, 0); } };

// A copy of one field-solve charge grid of a collide, for the bit-exact fixed-point comparison with the
// product's octo_capture_charge_plane: slice pair (i, j), direction, plane (0 = sL, 1 = sR, 2 = third).
struct Capture {
    bool armed = false, taken = false;
    int i = 0, j = 0, dir = 0, kind = 0;
    std::vector<int64_t> q;
    Grid grid{};
    int bits = 0;
};

struct Workspace {
    Capture *cap = nullptr;  // set with cap_kind >= 0 while the captured interaction runs
    int cap_kind = -1;
    int nx = 0, ny = 0;
    std::vector<double> charge;  // (2nx)*(2ny)
    std::vector<cplx> spectral;
    std::vector<double> green;
    Fft2D fft;
    FieldPlanes left, right, mid;
    int64_t dropped = 0;
    std::vector<double> vx[2], vy[2];
    std::vector<double> q1, q2;
    void init(int nx_, int ny_) {
        nx = nx_; ny = ny_;
        charge.assign((size_t)4 * nx * ny, 0.0);
        spectral.assign((size_t)4 * nx * ny, 0.0);
        green.assign((size_t)4 * nx * ny, 0.0);
        fft.init(2 * nx, 2 * ny);
        left.init(nx * ny); right.init(nx * ny); mid.init(nx * ny);
    }
};

struct GreenEntry {
    bool valid = false;
    Grid sg{}, fg{};
    std::vector<cplx> gfft;
    int64_t uses = 0, rebuilds = 0;
};

struct NodeMesh {
    bool valid = false;
    Grid sg{}, fg{};
    std::vector<cplx> gfft;
};

// pic_cpu.jl:1928-1939
void green_fft(const Options &O, Workspace &ws, const Grid &sg, const Grid &fg, std::vector<cplx> &out) {
    int nx = O.o.nx, ny = O.o.ny;
    double hx = sg.width / (double)(nx - 1), hy = sg.height / (double)(ny - 1);
    green_table(O.o.green_type, fg.x0, fg.y0, sg.x0, sg.y0, hx, hy, nx, ny, ws.green.data());
    out.resize((size_t)4 * nx * ny);
    for (size_t k = 0; k < out.size(); ++k) out[k] = cplx(ws.green[k], 0.0);
    ws.fft.run(out.data(), false);
}

// pic_cpu.jl:1965-1990
void solve_drifted(const Options &O, Workspace &ws, FieldPlanes &fp, const Coords &src, double s, const Grid &sg,
                   const std::vector<cplx> &gfft, bool drift = true, int kind = -1) {
    int nx = O.o.nx, ny = O.o.ny;
    double hx = sg.width / (double)(nx - 1), hy = sg.height / (double)(ny - 1);
    std::fill(ws.charge.begin(), ws.charge.end(), 0.0);
    int64_t *qfix = nullptr;
    if (ws.cap && kind >= 0 && kind == ws.cap_kind && O.o.fixed_point_deposit) {
        ws.cap->q.assign((size_t)nx * ny, 0);
        ws.cap->grid = sg;
        ws.cap->bits = fixed_bits((int64_t)src.size());
        ws.cap->taken = true;
        qfix = ws.cap->q.data();
    }
    deposit_grid(ws.charge.data(), 2 * nx, O.o.deposit_method, src.x.data(), src.px.data(), src.y.data(),
                 src.py.data(), (int64_t)src.size(), drift, s, sg.x0, sg.y0, hx, hy, nx, ny,
                 O.o.fixed_point_deposit != 0, qfix);
    for (size_t k = 0; k < ws.charge.size(); ++k) ws.spectral[k] = cplx(ws.charge[k], 0.0);
    ws.fft.run(ws.spectral.data(), false);
    for (size_t k = 0; k < ws.spectral.size(); ++k) ws.spectral[k] *= gfft[k];
    ws.fft.run(ws.spectral.data(), true);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) fp.phi[i + (size_t)j * nx] = ws.spectral[i + (size_t)j * 2 * nx].real();
    field_from_phi(fp.phi.data(), nx, ny, hx, hy, O.o.field_derivative == 4, fp.Ex.data(), fp.Ey.data());
}

// pic_cpu.jl:2596-2619 (two-node) ; the weights use the kick's deposit method
inline void interpolate_kick(const Options &O, const Grid &g, double x, double y, const FieldPlanes &L,
                             const FieldPlanes &R, double zL, double zR, double &Kx, double &Ky, double &Kz) {
    int nx = O.o.nx, ny = O.o.ny;
    double hx = g.width / (double)(nx - 1), hy = g.height / (double)(ny - 1);
    Kx = 0; Ky = 0; Kz = 0;
    auto body = [&](int ii, int jj, double w) {
        size_t k = (ii - 1) + (size_t)(jj - 1) * nx;
        Kx += w * (zL * L.Ex[k] + zR * R.Ex[k]);
        Ky += w * (zL * L.Ey[k] + zR * R.Ey[k]);
        Kz += w * (L.phi[k] - R.phi[k]);
    };
    deposit_point(O.o.deposit_method, (x - g.x0) / hx, (y - g.y0) / hy, nx, ny, body);
}

// pic_cpu.jl:2648-2680 (three-node)
inline void interpolate_kick_quadratic(const Options &O, const Grid &g, double x, double y, const FieldPlanes &L,
                                       const FieldPlanes &M, const FieldPlanes &R, double t, double &Kx,
                                       double &Ky, double &Kz) {
    int nx = O.o.nx, ny = O.o.ny;
    double hx = g.width / (double)(nx - 1), hy = g.height / (double)(ny - 1);
    double t2 = t * t;
    double aL = 2.0 * t2 - 3.0 * t + 1.0, aM = 4.0 * t - 4.0 * t2, aR = 2.0 * t2 - t;
    double bL = 3.0 - 4.0 * t, bM = 8.0 * t - 4.0, bR = 1.0 - 4.0 * t;
    Kx = 0; Ky = 0; Kz = 0;
    auto body = [&](int ii, int jj, double w) {
        size_t k = (ii - 1) + (size_t)(jj - 1) * nx;
        Kx += w * (aL * L.Ex[k] + aM * M.Ex[k] + aR * R.Ex[k]);
        Ky += w * (aL * L.Ey[k] + aM * M.Ey[k] + aR * R.Ey[k]);
        Kz += w * (bL * L.phi[k] + bM * M.phi[k] + bR * R.phi[k]);
    };
    deposit_point(O.o.deposit_method, (x - g.x0) / hx, (y - g.y0) / hy, nx, ny, body);
}

inline void slice_interp_params(double lb, double rb, double &hzi, double &zbias) {  // pic_cpu.jl:1540-1548
    double denom = rb - lb;
    if (!std::isfinite(denom) || denom == 0.0) { hzi = 0.0; zbias = 0.5; return; }
    hzi = 1.0 / denom;
    zbias = rb * hzi;
}

struct SliceParam { double weight, lb, center, rb; };

struct Slices {
    std::vector<double> center, weight, boundary;
    std::vector<std::vector<int64_t>> indices;  // 0-based particle indices, ascending
};

// slicing.jl:226-257
double lane_sum_all(const double *z, int64_t n, double mu, bool square) {
    std::vector<double> acc(SLICE_FOLD_LANES, 0.0);
    for (int64_t i = 0; i < n; ++i) {
        double v = square ? (z[i] - mu) * (z[i] - mu) : z[i];
        acc[i % SLICE_FOLD_LANES] += v;
    }
    double s = 0.0;
    for (int t = 0; t < SLICE_FOLD_LANES; ++t) s += acc[t];
    return s;
}
double lane_indexed_sum(const double *z, const std::vector<int64_t> &idx) {
    std::vector<double> acc(SLICE_FOLD_LANES, 0.0);
    for (size_t k = 0; k < idx.size(); ++k) acc[k % SLICE_FOLD_LANES] += z[idx[k]];
    double s = 0.0;
    for (int t = 0; t < SLICE_FOLD_LANES; ++t) s += acc[t];
    return s;
}

// _slice_bin (slicing.jl:177-181): the 1-based bin of zi, 0 for a coordinate with none.  d lies within the
// live extrema here, so the clamp never meets an overflowing floor.
int64_t slice_bin(double zi, double zmin, double width, int64_t bins) {
    const double d = (zi - zmin) / width;
    if (!(d > -INFINITY && d < INFINITY)) return 0;
    const double f = std::floor(d);
    if (f >= (double)bins) return bins;
    if (f < 0.0) return 1;
    return jclampi((long)f + 1, 1, (long)bins);
}

// Julia's collect(range(start, stop; length = len)) for Float64 endpoints (Base twiceprecision.jl,
// _linspace(start, stop, len)): a reference element of smallest magnitude, a step split into a truncated high
// part and a low part fitted so both endpoints are reproduced, and each element evaluated in double-double
// arithmetic around the reference index.  Julia first tries an exact-rational form when both endpoints are
// ratios of integers below 2^24 (rat / lcm); that branch is not restated: for such endpoints it can differ
// from this one in the last bit of interior elements.
std::vector<double> julia_range(double start, double stop, int64_t len) {
    std::vector<double> out((size_t)len);
    if (len == 1) { out[0] = start; return out; }
    if (start == stop) { std::fill(out.begin(), out.end(), start); return out; }
    auto add12 = [](double x, double y, double &h, double &l) {
        if (std::fabs(y) > std::fabs(x)) std::swap(x, y);
        h = x + y;
        l = (x - h) + y;
    };
    double delta = stop - start;
    int64_t dfac = 1;
    if (!std::isfinite(delta)) { delta = stop / (double)len - start / (double)len; dfac = len; }
    const double tmin = -(start / delta) / (double)dfac;
    int64_t imin = (int64_t)std::nearbyint(tmin * (double)(len - 1) + 1);  // round(Int, x): ties to even
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
    const double m = std::nextafter(std::numeric_limits<double>::max(), 0.0);
    const double k = (double)std::max(imin - 1, len - imin);
    const double lo = jmax(-(m + ref) / k, (-m + ref) / k), hi = jmin((m - ref) / k, (m + ref) / k);
    const double step_pre = jclamp(step, lo, hi);
    // nbitslen(Float64, len, imin) = min(cld(53, 2), top_set_bit(max(imin - 1, len - imin) - 1))
    const uint64_t span = (uint64_t)(std::max(imin - 1, len - imin) - 1);
    int nb = 0;
    for (uint64_t v = span; v; v >>= 1) ++nb;
    nb = std::min(nb, 27);
    uint64_t bits;
    std::memcpy(&bits, &step_pre, 8);
    bits &= (~0ull) << nb;
    double step_hi;
    std::memcpy(&step_hi, &bits, 8);
    double x1h, x1l, x2h, x2l;
    add12((double)(1 - imin) * step_hi, ref, x1h, x1l);
    add12((double)(len - imin) * step_hi, ref, x2h, x2l);
    const double a = (start - x1h) - x1l, b = (stop - x2h) - x2l;
    const double step_lo = (b - a) / (double)(len - 1);
    const double ref_lo = a - (double)(1 - imin) * step_lo;
    for (int64_t i = 1; i <= len; ++i) {
        const double u = (double)(i - imin);
        const double sh = u * step_hi, sl = u * step_lo;
        double xh, xl;
        add12(ref, sh, xh, xl);
        out[(size_t)(i - 1)] = xh + (xl + (sl + ref_lo));
    }
    return out;
}

// slicing.jl:51-75, 405-460, 523-559, the :specified method slicing.jl:393-403, :equal_area slicing.jl:104-156,
// :equal_count slicing.jl:330-365 and :equal_width slicing.jl:367-388
Slices make_slices(int method, int ns, int center_position, const std::vector<double> &positions, const double *z,
                   int64_t n, int resolution = 100) {
    if (ns <= 0) throw OracleError(OO_ERR_ARG, "nslices must be positive");
    if (n <= 0) throw OracleError(OO_ERR_ARG, "longitudinal slicing requires at least one particle");
    double zmin = INFINITY, zmax = -INFINITY;
    for (int64_t i = 0; i < n; ++i) { zmin = jmin(zmin, z[i]); zmax = jmax(zmax, z[i]); }
    double mu = lane_sum_all(z, n, 0.0, false) / (double)n;
    double s2 = lane_sum_all(z, n, mu, true);
    double sigma = std::sqrt(jmax(s2 / (double)n, 0.0));
    std::vector<double> b(ns + 1);
    if (method == 0) {
        if (sigma == 0.0) {
            std::fill(b.begin(), b.end(), mu);
        } else {
            b[0] = zmin; b[ns] = zmax;
            for (int s = 1; s <= ns - 1; ++s) {
                double q = std::sqrt(2.0) * erfinv_impl((double)(2 * s) / (double)ns - 1.0);
                b[s] = jclamp(mu + sigma * q, b[0], b[ns]);
            }
        }
    } else if (method == 1) {
        std::vector<double> internal;
        for (double p : positions) internal.push_back(mu + p * sigma);
        std::stable_sort(internal.begin(), internal.end());
        b.assign(internal.size() + 2, 0.0);
        b[0] = zmin; b[b.size() - 1] = zmax;
        for (size_t i = 0; i < internal.size(); ++i) b[i + 1] = jclamp(internal[i], b[0], b[b.size() - 1]);
        ns = (int)b.size() - 1;
    } else if (method == 2) {  // :equal_area
        if (resolution <= 0) throw OracleError(OO_ERR_ARG, "resolution must be positive");
        const int64_t bins = (int64_t)ns * resolution;
        if (zmin == zmax) {
            std::fill(b.begin(), b.end(), zmin);
        } else {
            const double width = (zmax - zmin) / (double)bins;
            std::vector<int64_t> counts((size_t)bins, 0);
            for (int64_t i = 0; i < n; ++i) {
                const int64_t bin = slice_bin(z[i], zmin, width, bins);
                if (bin) ++counts[(size_t)(bin - 1)];
            }
            std::vector<double> cum((size_t)bins);
            int64_t run = 0;
            for (int64_t k = 0; k < bins; ++k) {
                run += counts[(size_t)k];
                cum[(size_t)k] = (double)run / (double)std::max<int64_t>(n, 1);
            }
            cum[(size_t)(bins - 1)] = 1.0;
            auto center = [&](int64_t i1) { return zmin + ((double)i1 - 0.5) * width; };
            b[0] = zmin;
            b[ns] = zmax;
            int64_t current = 1;
            for (int s = 1; s <= ns - 1; ++s) {
                const double target = (double)s / (double)ns;
                while (current <= bins && cum[(size_t)(current - 1)] <= target) ++current;
                double x1, x2, y1, y2;
                if (current <= 1) { x1 = b[0]; x2 = center(1); y1 = 0.0; y2 = cum[0]; }
                else if (current > bins) { x1 = center(bins); x2 = b[ns]; y1 = cum[(size_t)(bins - 2)]; y2 = 1.0; }
                else { x1 = center(current - 1); x2 = center(current); y1 = cum[(size_t)(current - 2)]; y2 = cum[(size_t)(current - 1)]; }
                b[s] = y2 == y1 ? (x1 + x2) / 2 : x2 * (target - y1) / (y2 - y1) + x1 * (target - y2) / (y1 - y2);
            }
        }
    } else if (method == 3) {  // :equal_count: membership by rank (ties by index), boundaries at rank midpoints
        std::vector<int64_t> order((size_t)n);
        for (int64_t i = 0; i < n; ++i) order[(size_t)i] = i;
        auto key = [&](int64_t i) {  // isless order of doubles (-0.0 < +0.0)
            uint64_t u;
            std::memcpy(&u, &z[i], 8);
            return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
        };
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t c) { return key(a) < key(c); });
        b[0] = zmin;
        b[ns] = zmax;
        for (int s = 1; s <= ns - 1; ++s) {
            const int64_t pos = (int64_t)std::floor((double)((int64_t)s * n) / (double)ns);
            b[s] = pos == 0 ? z[order[0]] : (pos == n ? z[order[(size_t)(n - 1)]]
                                                     : (z[order[(size_t)(pos - 1)]] + z[order[(size_t)pos]]) / 2);
        }
        for (double v : b)
            if (!std::isfinite(v)) throw OracleError(OO_ERR_NONFINITE, "non-finite beam coordinate (longitudinal slicing)");
        Slices S;
        S.boundary = b;
        S.indices.assign(ns, {});
        for (int s = 1; s <= ns; ++s) {
            const int64_t first = (int64_t)std::floor((double)((int64_t)(s - 1) * n) / (double)ns);
            const int64_t last = (int64_t)std::floor((double)((int64_t)s * n) / (double)ns);
            for (int64_t r = first; r < last; ++r) S.indices[s - 1].push_back(order[(size_t)r]);
        }
        S.center.resize(ns);
        S.weight.resize(ns);
        for (int s = 0; s < ns; ++s) {
            const auto &idx = S.indices[s];
            S.weight[s] = (double)idx.size() / (double)n;
            S.center[s] = center_position == 0 && !idx.empty() ? lane_indexed_sum(z, idx) / (double)idx.size()
                                                               : (b[s] + b[s + 1]) / 2;
        }
        return S;
    } else if (method == 4) {  // :equal_width
        if (!(std::isfinite(zmin) && std::isfinite(zmax)))
            throw OracleError(OO_ERR_NONFINITE, "non-finite beam coordinate (longitudinal slicing)");
        b = julia_range(zmin, zmax, ns + 1);
        Slices S;
        S.boundary = b;
        S.indices.assign(ns, {});
        if (zmin == zmax) {
            for (int64_t i = 0; i < n; ++i) S.indices[0].push_back(i);
        } else {
            const double width = (zmax - zmin) / (double)ns;
            for (int64_t i = 0; i < n; ++i) {
                const int64_t bin = slice_bin(z[i], zmin, width, ns);
                if (bin) S.indices[(size_t)(bin - 1)].push_back(i);
            }
        }
        S.center.resize(ns);
        S.weight.resize(ns);
        for (int s = 0; s < ns; ++s) {
            const auto &idx = S.indices[s];
            S.weight[s] = (double)idx.size() / (double)n;
            S.center[s] = center_position == 0 && !idx.empty() ? lane_indexed_sum(z, idx) / (double)idx.size()
                                                               : (b[s] + b[s + 1]) / 2;
        }
        return S;
    } else {
        throw OracleError(OO_ERR_UNSUPPORTED, "unsupported slicing method");
    }
    for (double v : b)
        if (!std::isfinite(v)) throw OracleError(OO_ERR_NONFINITE, "non-finite beam coordinate (longitudinal slicing)");
    Slices S;
    S.boundary = b;
    S.indices.assign(ns, {});
    if (b[0] == b[ns]) {
        for (int64_t i = 0; i < n; ++i) S.indices[0].push_back(i);
    } else {
        for (int64_t i = 0; i < n; ++i) {
            // searchsortedlast(b, z) clamped to [1, ns]
            int k = (int)(std::upper_bound(b.begin(), b.end(), z[i]) - b.begin());  // count of b <= z
            int s = (int)jclampi(k, 1, ns);
            S.indices[s - 1].push_back(i);
        }
    }
    S.center.resize(ns);
    S.weight.resize(ns);
    for (int s = 0; s < ns; ++s) {
        const auto &idx = S.indices[s];
        S.weight[s] = (double)idx.size() / (double)n;
        if (center_position == 0)
            S.center[s] = idx.empty() ? (b[s] + b[s + 1]) / 2 : lane_indexed_sum(z, idx) / (double)idx.size();
        else
            S.center[s] = (b[s] + b[s + 1]) / 2;
    }
    return S;
}

struct OrderEntry { double t; int i, j; };

// slicing.jl:561-568 (stable sort by collision time)
std::vector<OrderEntry> collision_order(const std::vector<double> &c1, const std::vector<double> &c2) {
    std::vector<OrderEntry> o;
    for (size_t i = 0; i < c1.size(); ++i)
        for (size_t j = 0; j < c2.size(); ++j) o.push_back({-(c1[i] + c2[j]) / 2, (int)i + 1, (int)j + 1});
    std::stable_sort(o.begin(), o.end(), [](const OrderEntry &a, const OrderEntry &b) { return a.t < b.t; });
    return o;
}

// slicing.jl:601-647
std::vector<std::vector<OrderEntry>> pair_batches(const std::vector<double> &c1, const std::vector<double> &c2) {
    auto pairs = collision_order(c1, c2);
    std::vector<std::vector<OrderEntry>> batches;
    int ns1 = (int)c1.size(), ns2 = (int)c2.size();
    std::vector<std::vector<int>> by_i(ns1 + 1), by_j(ns2 + 1);
    for (size_t k = 0; k < pairs.size(); ++k) {
        by_i[pairs[k].i].push_back((int)k);
        by_j[pairs[k].j].push_back((int)k);
    }
    std::vector<size_t> next_i(ns1 + 1, 0), next_j(ns2 + 1, 0);
    std::vector<char> done(pairs.size(), 0);
    size_t remaining = pairs.size();
    while (remaining > 0) {
        std::vector<OrderEntry> cur;
        std::vector<char> used_i(ns1 + 1, 0), used_j(ns2 + 1, 0);
        for (size_t k = 0; k < pairs.size(); ++k) {
            if (done[k]) continue;
            const auto &p = pairs[k];
            if (used_i[p.i] || used_j[p.j]) continue;
            bool ri = next_i[p.i] < by_i[p.i].size() && by_i[p.i][next_i[p.i]] == (int)k;
            bool rj = next_j[p.j] < by_j[p.j].size() && by_j[p.j][next_j[p.j]] == (int)k;
            if (ri && rj) {
                cur.push_back(p);
                used_i[p.i] = 1; used_j[p.j] = 1; done[k] = 1;
                next_i[p.i]++; next_j[p.j]++;
                --remaining;
            }
        }
        if (cur.empty()) throw OracleError(OO_ERR_ARG, "internal collision scheduler error");
        batches.push_back(cur);
    }
    return batches;
}

struct Ctx {
    Options O;
    int ns1 = 0, ns2 = 0;
    std::vector<GreenEntry> cache;  // [(dir-1)][i-1][j-1]
    int64_t hits = 0, misses = 0, rebuilds = 0;
    int64_t dropped = 0;
    std::vector<int> trace_i, trace_j;
    std::vector<double> trace_lum;
    std::string err;
    Capture cap;
    GreenEntry &entry(int i, int j, int dir) { return cache[((size_t)(dir - 1) * ns1 + (i - 1)) * ns2 + (j - 1)]; }
};

std::string pair_ctx(int i, int j, int dir) {
    char b[96];
    snprintf(b, sizeof b, "slice pair (%d, %d), direction %d", i, j, dir);
    return b;
}

[[noreturn]] void nonfinite(const char *role, const Coords &c, const std::string &where) {
    int64_t first = -1;
    for (size_t k = 0; k < c.size(); ++k)
        if (!std::isfinite(c.x[k]) || !std::isfinite(c.px[k]) || !std::isfinite(c.y[k]) || !std::isfinite(c.py[k]) ||
            !std::isfinite(c.z[k])) { first = (int64_t)k + 1; break; }
    char b[256];
    snprintf(b, sizeof b, "non-finite %s coordinate at slice particle %lld (%s)", role, (long long)first,
             where.c_str());
    throw OracleError(OO_ERR_NONFINITE, b);
}

// pic_cpu.jl:1780-1808
bool grid_size_usable(const Grid &c, const Grid &r, double mr) {
    return c.width >= r.width && c.height >= r.height && r.width >= mr * c.width && r.height >= mr * c.height;
}
bool grid_covers(const Options &O, const Grid &g, const Bounds &b) {
    double hx = g.width / (double)(O.o.nx - 1), hy = g.height / (double)(O.o.ny - 1);
    double m = TEMPLATE_MARGIN_CELLS;
    return g.x0 + m * hx <= b.xmin && g.x0 + g.width - m * hx >= b.xmax && g.y0 + m * hy <= b.ymin &&
           g.y0 + g.height - m * hy >= b.ymax;
}
Grid expand_grid(const Grid &g, double factor) {  // pic_cpu.jl:1810-1821
    if (factor <= 1.0) return g;
    double nw = g.width * factor, nh = g.height * factor;
    return {g.x0 - (nw - g.width) / 2, g.y0 - (nh - g.height) / 2, nw, nh};
}

// pic_cpu.jl:1729-1778 ; returns (sg, fg, green)
const std::vector<cplx> &slice_pair_green(Ctx &C, Workspace &ws, int i, int j, int dir, Grid &sg, Grid &fg,
                                          const Bounds &sb, const Bounds &fb, std::vector<cplx> &own,
                                          int64_t counters[3]) {
    const Options &O = C.O;
    if (O.o.green_cache == 1) {
        GreenEntry &e = C.entry(i, j, dir);
        bool usable = e.valid && grid_size_usable(e.sg, sg, O.o.green_min_ratio) &&
                      grid_size_usable(e.fg, fg, O.o.green_min_ratio) && grid_covers(O, e.sg, sb) &&
                      grid_covers(O, e.fg, fb);
        if (usable) {
            counters[0]++;
            e.uses++;
            sg = e.sg; fg = e.fg;
            return e.gfft;
        }
        Grid es = expand_grid(sg, 1.0 + O.o.green_growth);
        Grid ef = expand_grid(fg, 1.0 + O.o.green_growth);
        if (O.o.green_type != 0) {  // pic_cpu.jl:1853-1862
            double hx = es.width / (double)(O.o.nx - 1), hy = es.height / (double)(O.o.ny - 1);
            double sx0, fx0, sy0, fy0;
            align_origins(O.o.green_type, es.x0, ef.x0, hx, sx0, fx0);
            align_origins(O.o.green_type, es.y0, ef.y0, hy, sy0, fy0);
            es.x0 = sx0; ef.x0 = fx0; es.y0 = sy0; ef.y0 = fy0;
        }
        green_fft(O, ws, es, ef, e.gfft);
        if (!e.valid) { counters[1]++; e.rebuilds = 0; }
        else { counters[2]++; e.rebuilds++; }
        e.valid = true; e.uses = 1; e.sg = es; e.fg = ef;
        sg = es; fg = ef;
        return e.gfft;
    }
    green_fft(O, ws, sg, fg, own);
    return own;
}

int64_t count_outside(const std::vector<double> &xs, const std::vector<double> &ys, double xlo, double xhi,
                      double ylo, double yhi) {
    int64_t c = 0;
    for (size_t i = 0; i < xs.size(); ++i) {
        double x = xs[i], y = ys[i];
        if (!(std::isfinite(x) && xlo <= x && x <= xhi && std::isfinite(y) && ylo <= y && y <= yhi)) ++c;
    }
    return c;
}
int64_t count_outside_drifted(const Coords &s, double sL, double sR, double xlo, double xhi, double ylo,
                              double yhi) {
    int64_t c = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        double xl = s.x[i] + s.px[i] * sL, yl = s.y[i] + s.py[i] * sL;
        double xr = s.x[i] + s.px[i] * sR, yr = s.y[i] + s.py[i] * sR;
        if (!(std::isfinite(xl) && xlo <= xl && xl <= xhi && std::isfinite(yl) && ylo <= yl && yl <= yhi &&
              std::isfinite(xr) && xlo <= xr && xr <= xhi && std::isfinite(yr) && ylo <= yr && yr <= yhi))
            ++c;
    }
    return c;
}

void virtual_positions(const Coords &src, double sM, std::vector<double> &vx, std::vector<double> &vy) {
    vx.resize(src.size());
    vy.resize(src.size());
    for (size_t i = 0; i < src.size(); ++i) {
        vx[i] = src.x[i] + src.px[i] * sM;
        vy[i] = src.y[i] + src.py[i] * sM;
    }
}

// pic_cpu.jl:954-1144
// interaction_grid = :source_slice (pic_cpu.jl:610-712): the mesh of every pair of a (source slice, direction)
// is sized from one union box taken at the slice's first use -- the source drifted across the partner beam's
// whole longitudinal range, every partner particle drifted to its collision point -- while the Green cache's
// coverage test still sees this pair's own bounds.
struct UnionBounds {
    bool valid = false;
    Bounds sb{}, fb{};
};

// _pic_union_bounds, the states form the collide loop uses (pic_cpu.jl:665-692), and its source tail
// (pic_cpu.jl:697-712).  The partner's z range and collision-point extrema come from its CURRENT slice states,
// so the box depends on how much of the turn has been applied; the source is bounded at its two extreme drifts
// (the drift is affine in s).  Invalid -- no override, per-pair sizing -- when the partner has no finite z.
UnionBounds union_bounds(const Coords &source, double center, const std::vector<Coords> &partner) {
    UnionBounds u;
    const double c = center;
    double zmin = INFINITY, zmax = -INFINITY;
    double fxmin = INFINITY, fxmax = -INFINITY, fymin = INFINITY, fymax = -INFINITY;
    for (const Coords &fc : partner)
        for (size_t k = 0; k < fc.size(); ++k) {
            const double zi = fc.z[k];
            zmin = jmin(zmin, zi); zmax = jmax(zmax, zi);
            const double s = 0.5 * (zi - c);
            const double xv = fc.x[k] + s * fc.px[k], yv = fc.y[k] + s * fc.py[k];
            fxmin = jmin(fxmin, xv); fxmax = jmax(fxmax, xv);
            fymin = jmin(fymin, yv); fymax = jmax(fymax, yv);
        }
    if (std::isnan(zmin) || !(std::isfinite(fxmin) && std::isfinite(fxmax) && std::isfinite(fymin) &&
                              std::isfinite(fymax)))
        for (const Coords &fc : partner)
            for (size_t k = 0; k < fc.size(); ++k)
                if (!std::isfinite(fc.z[k]) || !std::isfinite(fc.x[k]) || !std::isfinite(fc.px[k]) ||
                    !std::isfinite(fc.y[k]) || !std::isfinite(fc.py[k]))
                    nonfinite("field", fc, "source-slice union bounds");
    if (!std::isfinite(zmin)) return u;
    const double sA = 0.5 * (c - zmax), sB = 0.5 * (c - zmin);
    double sxmin = INFINITY, sxmax = -INFINITY, symin = INFINITY, symax = -INFINITY;
    for (size_t k = 0; k < source.size(); ++k) {
        const double xa = source.x[k] + source.px[k] * sA, xb = source.x[k] + source.px[k] * sB;
        const double ya = source.y[k] + source.py[k] * sA, yb = source.y[k] + source.py[k] * sB;
        sxmin = jmin(jmin(sxmin, xa), xb); sxmax = jmax(jmax(sxmax, xa), xb);
        symin = jmin(jmin(symin, ya), yb); symax = jmax(jmax(symax, ya), yb);
    }
    if (!(std::isfinite(sxmin) && std::isfinite(sxmax) && std::isfinite(symin) && std::isfinite(symax)))
        nonfinite("source", source, "source-slice union bounds");
    u.valid = true;
    u.sb = {sxmin, sxmax, symin, symax};
    u.fb = {fxmin, fxmax, fymin, fymax};
    return u;
}

void interaction(Ctx &C, Workspace &ws, const Coords &source, const SliceParam &ps, Coords &field,
                 const SliceParam &pf, double kbb, int i, int j, int dir, int vslot, int64_t counters[3],
                 const UnionBounds *over = nullptr) {
    const Options &O = C.O;
    const int nsource = (int)source.size(), nfield = (int)field.size();
    double sL = 0.5 * (ps.center - pf.lb);
    double sR = 0.5 * (ps.center - pf.rb);
    double sxl = source.x[0] + source.px[0] * sL, syl = source.y[0] + source.py[0] * sL;
    double sxr = source.x[0] + source.px[0] * sR, syr = source.y[0] + source.py[0] * sR;
    double sxmin = jmin(sxl, sxr), sxmax = jmax(sxl, sxr), symin = jmin(syl, syr), symax = jmax(syl, syr);
    int ge = O.o.grid_extent;
    double sx0 = sxl, sy0 = syl;
    double sxs = 0, sxs2 = 0, sys = 0, sys2 = 0;
    for (int k = 0; k < nsource; ++k) {
        double xl = source.x[k] + source.px[k] * sL, yl = source.y[k] + source.py[k] * sL;
        double xr = source.x[k] + source.px[k] * sR, yr = source.y[k] + source.py[k] * sR;
        sxmin = jmin(jmin(sxmin, xl), xr); sxmax = jmax(jmax(sxmax, xl), xr);
        symin = jmin(jmin(symin, yl), yr); symax = jmax(jmax(symax, yl), yr);
        if (ge != 0) {
            double dxl = xl - sx0, dxr = xr - sx0, dyl = yl - sy0, dyr = yr - sy0;
            sxs += dxl + dxr; sxs2 += dxl * dxl + dxr * dxr;
            sys += dyl + dyr; sys2 += dyl * dyl + dyr * dyr;
        }
    }
    double kext = O.o.grid_extent_sigma;
    axis_extent(ge, sxmin, sxmax, sx0, sxs, sxs2, 2 * (int64_t)nsource, kext);
    axis_extent(ge, symin, symax, sy0, sys, sys2, 2 * (int64_t)nsource, kext);
    if (!(std::isfinite(sxmin) && std::isfinite(sxmax) && std::isfinite(symin) && std::isfinite(symax)))
        nonfinite("source", source, pair_ctx(i, j, dir));

    double fxmin = field.x[0] + 0.5 * (field.z[0] - ps.center) * field.px[0];
    double fxmax = fxmin;
    double fymin = field.y[0] + 0.5 * (field.z[0] - ps.center) * field.py[0];
    double fymax = fymin;
    double fx0 = fxmin, fy0 = fymin;
    double fxs = 0, fxs2 = 0, fys = 0, fys2 = 0;
    for (int k = 0; k < nfield; ++k) {
        double s = 0.5 * (field.z[k] - ps.center);
        field.x[k] += s * field.px[k];
        field.y[k] += s * field.py[k];
        if (O.o.longitudinal_kick) field.pz[k] -= 0.25 * (field.px[k] * field.px[k] + field.py[k] * field.py[k]);
        fxmin = jmin(fxmin, field.x[k]); fxmax = jmax(fxmax, field.x[k]);
        fymin = jmin(fymin, field.y[k]); fymax = jmax(fymax, field.y[k]);
        if (ge != 0) {
            double dx = field.x[k] - fx0, dy = field.y[k] - fy0;
            fxs += dx; fxs2 += dx * dx; fys += dy; fys2 += dy * dy;
        }
    }
    axis_extent(ge, fxmin, fxmax, fx0, fxs, fxs2, nfield, kext);
    axis_extent(ge, fymin, fymax, fy0, fys, fys2, nfield, kext);
    if (!(std::isfinite(fxmin) && std::isfinite(fxmax) && std::isfinite(fymin) && std::isfinite(fymax)))
        nonfinite("field", field, pair_ctx(i, j, dir));

    Grid sg, fg;
    if (over && over->valid)
        interaction_grids(O, over->sb.xmin, over->sb.xmax, over->sb.ymin, over->sb.ymax, over->fb.xmin, over->fb.xmax,
                          over->fb.ymin, over->fb.ymax, sg, fg);
    else
        interaction_grids(O, sxmin, sxmax, symin, symax, fxmin, fxmax, fymin, fymax, sg, fg);
    Bounds sb{sxmin, sxmax, symin, symax}, fb{fxmin, fxmax, fymin, fymax};
    std::vector<cplx> own;
    // :source_slice caches one mesh per (source slice, direction) -- the keys (i, 0, 1) and (j, 0, 2) of
    // pic_cpu.jl:372-373 -- held in the slot of partner slice 1
    const bool shared = O.o.interaction_grid == 1;
    const std::vector<cplx> &gfft = slice_pair_green(C, ws, shared && dir == 2 ? 1 : i, shared && dir == 1 ? 1 : j,
                                                     dir, sg, fg, sb, fb, own, counters);
    if (ge != 0 || O.o.interaction_grid == 1) {
        ws.dropped += count_outside(field.x, field.y, fg.x0, fg.x0 + fg.width, fg.y0, fg.y0 + fg.height);
        ws.dropped += count_outside_drifted(source, sL, sR, sg.x0, sg.x0 + sg.width, sg.y0, sg.y0 + sg.height);
    }
    solve_drifted(O, ws, ws.left, source, sL, sg, gfft, true, 0);
    solve_drifted(O, ws, ws.right, source, sR, sg, gfft, true, 1);
    double ks = 2.0 * kbb;
    double hzi, zbias;
    slice_interp_params(pf.lb, pf.rb, hzi, zbias);
    bool lk = O.o.longitudinal_kick != 0;
    if (O.o.slice_interpolation == 1) {
        double smid = 0.5 * (sL + sR);
        solve_drifted(O, ws, ws.mid, source, smid, sg, gfft, true, 2);
        for (int k = 0; k < nfield; ++k) {
            double zL = jclamp(-field.z[k] * hzi + zbias, 0.0, 1.0);
            double Kx, Ky, Kz;
            interpolate_kick_quadratic(O, fg, field.x[k], field.y[k], ws.left, ws.mid, ws.right, 1.0 - zL, Kx, Ky,
                                       Kz);
            field.px[k] += ks * Kx;
            field.py[k] += ks * Ky;
            if (lk) field.pz[k] += ks * Kz * hzi;
            double s = 0.5 * (ps.center - field.z[k]);
            field.x[k] += s * field.px[k];
            field.y[k] += s * field.py[k];
            if (lk) field.pz[k] += 0.25 * (field.px[k] * field.px[k] + field.py[k] * field.py[k]);
        }
    } else {
        for (int k = 0; k < nfield; ++k) {
            double zL = jclamp(-field.z[k] * hzi + zbias, 0.0, 1.0);
            double zR = 1.0 - zL;
            double Kx, Ky, Kz;
            interpolate_kick(O, fg, field.x[k], field.y[k], ws.left, ws.right, zL, zR, Kx, Ky, Kz);
            field.px[k] += ks * Kx;
            field.py[k] += ks * Ky;
            if (lk) field.pz[k] += ks * Kz * hzi;
            double s = 0.5 * (ps.center - field.z[k]);
            field.x[k] += s * field.px[k];
            field.y[k] += s * field.py[k];
            if (lk) field.pz[k] += 0.25 * (field.px[k] * field.px[k] + field.py[k] * field.py[k]);
        }
    }
    double sM = 0.5 * (ps.center - pf.center);
    virtual_positions(source, sM, ws.vx[vslot], ws.vy[vslot]);
}

// pic_cpu.jl:1448-1538
// ---------------------------------------------------------------- Gaussian-subtracted hybrid
// GaussianPICPoissonSolver (gaussian_pic.jl): the uncoupled subtraction (coupling_tol = Inf, the default) and
// the coupled (rotated) subtraction above a finite coupling_tol.

// Node-centred erf-integrated profile of a unit 1D Gaussian against the CIC / TSC assignment function
// (gaussian_pic.jl:206-237); node i sits at x0 + i h.
void gaussian_profile(int method, double x0, double h, double mu, double s, int n, double *g) {
    const double invroot = 1.0 / (s * std::sqrt(2.0));
    const double norm = 1.0 / (s * std::sqrt(2.0 * be::kPi));
    auto pdf = [&](double x) { return norm * std::exp(-((x - mu) * (x - mu)) / (2.0 * s * s)); };
    auto m0 = [&](double A, double B) { return 0.5 * (std::erf((B - mu) * invroot) - std::erf((A - mu) * invroot)); };
    auto m1 = [&](double A, double B, double xi) { return (mu - xi) * m0(A, B) - s * s * (pdf(B) - pdf(A)); };
    auto m2 = [&](double A, double B, double xi) {
        return (s * s + (mu - xi) * (mu - xi)) * m0(A, B) - s * s * ((B - mu) * pdf(B) - (A - mu) * pdf(A)) -
               2.0 * (mu - xi) * s * s * (pdf(B) - pdf(A));
    };
    const double half = h / 2.0;
    for (int i = 0; i < n; ++i) {
        const double xi = x0 + (double)i * h;
        if (method == 0) {
            g[i] = m0(xi - h, xi + h) + (m1(xi - h, xi, xi) - m1(xi, xi + h, xi)) / h;
        } else {
            const double cL = xi - half, cR = xi + half;
            const double lL = xi - 3.0 * half, lR = xi - half, rL = xi + half, rR = xi + 3.0 * half;
            g[i] = 0.75 * m0(cL, cR) - m2(cL, cR, xi) / (h * h) + 1.125 * (m0(lL, lR) + m0(rL, rR)) +
                   1.5 * (m1(lL, lR, xi) - m1(rL, rR, xi)) / h + 0.5 * (m2(lL, lR, xi) + m2(rL, rR, xi)) / (h * h);
        }
    }
}

// Central moments c_k = int_A^B (x - mu)^k G(x) dx, k = 0..4, of the normalised Gaussian by the integration-
// by-parts recursion (gaussian_pic.jl:274-287).
void central_moments(double A, double B, double mu, double s, double c[5]) {
    const double invroot = 1.0 / (s * std::sqrt(2.0));
    const double norm = 1.0 / (s * std::sqrt(2.0 * be::kPi));
    const double a = A - mu, b = B - mu;
    const double GA = norm * std::exp(-(a * a) / (2.0 * s * s));
    const double GB = norm * std::exp(-(b * b) / (2.0 * s * s));
    const double s2 = s * s;
    c[0] = 0.5 * (std::erf(b * invroot) - std::erf(a * invroot));
    c[1] = -s2 * (GB - GA);
    c[2] = -s2 * (b * GB - a * GA) + s2 * c[0];
    c[3] = -s2 * (b * b * GB - a * a * GA) + 2.0 * s2 * c[1];
    c[4] = -s2 * (b * b * b * GB - a * a * a * GA) + 3.0 * s2 * c[2];
}
// Node-centred moments about xi from the central ones, d = mu - xi (gaussian_pic.jl:291-299).
void shift_moments(const double c[5], double d, double m[5]) {
    const double d2 = d * d, d3 = d2 * d, d4 = d3 * d;
    m[0] = c[0];
    m[1] = c[1] + d * c[0];
    m[2] = c[2] + 2.0 * d * c[1] + d2 * c[0];
    m[3] = c[3] + 3.0 * d * c[2] + 3.0 * d2 * c[1] + d3 * c[0];
    m[4] = c[4] + 4.0 * d * c[3] + 6.0 * d2 * c[2] + 4.0 * d3 * c[1] + d4 * c[0];
}
void cell_moments(double A, double B, double mu, double s, double xi, double m[5]) {
    double c[5];
    central_moments(A, B, mu, s, c);
    shift_moments(c, mu - xi, m);
}
// Assignment-weighted moments W_k = int (x - xi)^k G W(x - xi) dx, k = 0, 1, 2 (gaussian_pic.jl:304-324).
void weighted_moments(double xi, double h, double mu, double s, int method, double W[3]) {
    if (method == 0) {
        double L[5], R[5];
        cell_moments(xi - h, xi, mu, s, xi, L);
        cell_moments(xi, xi + h, mu, s, xi, R);
        for (int k = 0; k < 3; ++k) W[k] = (L[k] + L[k + 1] / h) + (R[k] - R[k + 1] / h);
        return;
    }
    const double half = h / 2.0;
    double C[5], Lw[5], Rw[5];
    cell_moments(xi - half, xi + half, mu, s, xi, C);
    cell_moments(xi - 3.0 * half, xi - half, mu, s, xi, Lw);
    cell_moments(xi + half, xi + 3.0 * half, mu, s, xi, Rw);
    auto core = [&](const double *M, int k) { return 0.75 * M[k] - M[k + 2] / (h * h); };
    auto wing = [&](const double *M, int k, double sgn) {
        return 1.125 * M[k] + sgn * 1.5 * M[k + 1] / h + 0.5 * M[k + 2] / (h * h);
    };
    for (int k = 0; k < 3; ++k) W[k] = core(C, k) + wing(Lw, k, 1.0) + wing(Rw, k, -1.0);
}
// Mean-derivatives g' and g'' of the 1D node profile (gaussian_pic.jl:330-348).
void profile_mean_derivs(double yj, double h, double mu, double s, int method, double &dg, double &ddg) {
    const double invroot = 1.0 / (s * std::sqrt(2.0));
    const double norm = 1.0 / (s * std::sqrt(2.0 * be::kPi));
    auto pdf = [&](double y) { return norm * std::exp(-((y - mu) * (y - mu)) / (2.0 * s * s)); };
    auto m0 = [&](double A, double B) { return 0.5 * (std::erf((B - mu) * invroot) - std::erf((A - mu) * invroot)); };
    if (method == 0) {
        dg = (m0(yj - h, yj) - m0(yj, yj + h)) / h;
        ddg = (pdf(yj - h) - 2.0 * pdf(yj) + pdf(yj + h)) / h;
        return;
    }
    const double half = h / 2.0;
    double C[5], Lw[5], Rw[5];
    cell_moments(yj - half, yj + half, mu, s, yj, C);
    cell_moments(yj - 3.0 * half, yj - half, mu, s, yj, Lw);
    cell_moments(yj + half, yj + 3.0 * half, mu, s, yj, Rw);
    dg = -2.0 * C[1] / (h * h) + (1.5 * Lw[0] + Lw[1] / h) / h + (-1.5 * Rw[0] + Rw[1] / h) / h;
    ddg = (-2.0 * m0(yj - half, yj + half) + m0(yj - 3.0 * half, yj - half) + m0(yj + half, yj + 3.0 * half)) / (h * h);
}
// The six node profiles of the coupled subtraction (gaussian_pic.jl:350-370): x moments about mux, the
// conditional y profile (sigma = sigc) and its two mean-derivatives.
void coupled_profiles(int method, double x0, double hx, double mux, double sigx, int nx, double y0, double hy,
                      double muy, double sigc, int ny, double *gx, double *m1x, double *m2x, double *gy, double *dgy,
                      double *ddgy) {
    for (int i = 0; i < nx; ++i) {
        const double xi = x0 + (double)i * hx;
        double W[3];
        weighted_moments(xi, hx, mux, sigx, method, W);
        const double d = mux - xi;
        gx[i] = W[0];
        m1x[i] = W[1] - d * W[0];
        m2x[i] = W[2] - 2.0 * d * W[1] + d * d * W[0];
    }
    gaussian_profile(method, y0, hy, muy, sigc, ny, gy);
    for (int j = 0; j < ny; ++j) profile_mean_derivs(y0 + (double)j * hy, hy, muy, sigc, method, dgy[j], ddgy[j]);
}

// Full transverse covariance in StrongTransverseMoments order (strong_beam.jl:79-90).
struct CovMoments {
    double a0, b0, d0, bxx, bxpy, bypx, bypy, qxx, qxy, qyy;
};
// _cp_covariance_kick, coupled (strong_beam.jl:634-682): adds the kick of the covariance transported by S to
// px, py and its pz terms to pz; returns the density at (xx, yy) (0 for a degenerate covariance).
double coupled_covariance_kick(const CovMoments &m, double kbb, double S, double xx, double yy, double &px, double &py,
                               double &pz) {
    const double twopi_c = 6.283185307179586476925286766559005768394338;
    const double a = m.a0 - 2 * S * m.bxx + S * S * m.qxx;
    const double bb = m.b0 - S * (m.bxpy + m.bypx) + S * S * m.qxy;
    const double d = m.d0 - 2 * S * m.bypy + S * S * m.qyy;
    const double au = 2 * (m.bxx - S * m.qxx);
    const double bu = m.bxpy + m.bypx - 2 * S * m.qxy;
    const double du = 2 * (m.bypy - S * m.qyy);
    const double detA = a * d - bb * bb;
    if (a <= 0 || d <= 0 || detA <= 0) return 0.0;
    const double adiff = a - d;
    const double D = std::hypot(adiff, 2 * bb);
    if (D == 0.0) {
        const double sigma = std::sqrt((a + d) / 2);
        const double expterm = std::exp(-0.5 * (xx * xx + yy * yy) / (sigma * sigma));
        double Kx, Ky, Hxx, Hxy, Hyy;
        be::round_kick_hessian(kbb, sigma, xx, yy, expterm, Kx, Ky, Hxx, Hxy, Hyy);
        px += kbb * Kx;
        py += kbb * Ky;
        pz += 0.25 * (Hxx * au + 2 * Hxy * bu + Hyy * du);
        return expterm / (twopi_c * sigma * sigma);
    }
    const double theta = 0.5 * std::atan2(2 * bb, a - d);
    const double c = std::cos(theta), sn = std::sin(theta);
    const double lambda1 = (a + d + D) / 2, lambda2 = (a + d - D) / 2;
    const double sig1 = std::sqrt(lambda1), sig2 = std::sqrt(lambda2);
    const double xh = c * xx + sn * yy, yh = -sn * xx + c * yy;
    const double eta = D / (a + d);
    double inner, outer;
    be::eta_bounds(inner, outer);
    double Kxh, Kyh, H11, H22, LoD;
    if (eta <= inner) be::near_round_series(kbb, (a + d) / 2, eta, xh, yh, Kxh, Kyh, H11, H22, &LoD);
    else be::response_principal(kbb, sig1, sig2, xh, yh, Kxh, Kyh, H11, H22, &LoD);
    const double expterm = std::exp(-0.5 * (xh * xh / lambda1 + yh * yh / lambda2));
    const double Fxh = kbb * Kxh, Fyh = kbb * Kyh;
    px += c * Fxh - sn * Fyh;
    py += sn * Fxh + c * Fyh;
    const double Du = (adiff * (au - du) + 4 * bb * bu) / D;
    const double traceu = au + du;
    pz += 0.125 * ((H11 + H22) * traceu + (H11 - H22) * Du);
    const double rotation_projection = (adiff * bu - bb * (au - du)) / D;
    pz -= 0.5 * kbb * rotation_projection * LoD;
    return expterm / (twopi_c * sig1 * sig2);
}

// Transverse moments of the source slice from sums relative to its first particle (gaussian_pic.jl:432-486).
// coupled: also the four cross-plane sums (only the coupled subtraction reads them).
struct SourceMoments {
    int64_t n;
    double mx, mpx, varx, cxpx, varpx, my, mpy, vary, cypy, varpy;
    double cxy, cxpy, cypx, cpxpy;
};
SourceMoments source_moments(const Coords &s, bool coupled = false) {
    SourceMoments m{};
    const size_t n = s.size();
    m.n = (int64_t)n;
    const double x0 = s.x[0], px0 = s.px[0], y0 = s.y[0], py0 = s.py[0];
    double sx = 0, spx = 0, sy = 0, spy = 0, sxx = 0, spxpx = 0, syy = 0, spypy = 0, sxpx = 0, sypy = 0;
    double sxy = 0, sxpy = 0, sypx = 0, spxpy = 0;
    for (size_t i = 0; i < n; ++i) {
        const double dx = s.x[i] - x0, dpx = s.px[i] - px0, dy = s.y[i] - y0, dpy = s.py[i] - py0;
        sx += dx; spx += dpx; sy += dy; spy += dpy;
        sxx += dx * dx; spxpx += dpx * dpx;
        syy += dy * dy; spypy += dpy * dpy;
        sxpx += dx * dpx; sypy += dy * dpy;
        if (coupled) { sxy += dx * dy; sxpy += dx * dpy; sypx += dy * dpx; spxpy += dpx * dpy; }
    }
    const double invn = 1.0 / (double)n;
    const double dmx = sx * invn, dmpx = spx * invn, dmy = sy * invn, dmpy = spy * invn;
    m.mx = x0 + dmx; m.mpx = px0 + dmpx; m.my = y0 + dmy; m.mpy = py0 + dmpy;
    // muladd(-a, b, c) of slicing.jl:664-668, fused on FMA hosts
    m.varx = jmax(std::fma(-dmx, dmx, sxx * invn), 0.0);
    m.vary = jmax(std::fma(-dmy, dmy, syy * invn), 0.0);
    m.cxpx = std::fma(-dmx, dmpx, sxpx * invn);
    m.varpx = jmax(std::fma(-dmpx, dmpx, spxpx * invn), 0.0);
    m.cypy = std::fma(-dmy, dmpy, sypy * invn);
    m.varpy = jmax(std::fma(-dmpy, dmpy, spypy * invn), 0.0);
    if (coupled) {
        m.cxy = std::fma(-dmx, dmy, sxy * invn);
        m.cxpy = std::fma(-dmx, dmpy, sxpy * invn);
        m.cypx = std::fma(-dmy, dmpx, sypx * invn);
        m.cpxpy = std::fma(-dmpx, dmpy, spxpy * invn);
    }
    return m;
}
CovMoments coupled_moments(const SourceMoments &m) {  // _gpic_coupled_moments (gaussian_pic.jl:436-447)
    return CovMoments{m.varx, m.cxy, m.vary, m.cxpx, m.cxpy, m.cypx, m.cypy, m.varpx, m.cpxpy, m.varpy};
}

// Drifted reference Gaussian at a slice boundary (gaussian_pic.jl:496-540, uncoupled).
// coupled: also the drifted covariance (a, b, d), its correlation, whether it is resolved (full rank to the
// precision-derived tolerance), the conditional slope lambda = b / a and sigma sigc (gaussian_pic.jl:456-523).
struct Boundary {
    double mux, muy, sigx, sigy, rx, ry, s;
    double a, b, d, rxy, lam, sigc;
    bool resolved;
};
Boundary boundary(const SourceMoments &m, double s, bool coupled = false) {
    Boundary b{};
    b.s = s;
    b.mux = m.mx + m.mpx * s;
    b.muy = m.my + m.mpy * s;
    const double varx = m.varx + 2.0 * s * m.cxpx + s * s * m.varpx;
    const double vary = m.vary + 2.0 * s * m.cypy + s * s * m.varpy;
    b.sigx = std::sqrt(jmax(varx, 0.0));
    b.sigy = std::sqrt(jmax(vary, 0.0));
    b.rx = 2.0 * (m.cxpx + s * m.varpx);
    b.ry = 2.0 * (m.cypy + s * m.varpy);
    if (!coupled) return b;
    const CovMoments c = coupled_moments(m);
    const double S = -s;  // _transport_transverse_moments with the field-particle convention
    b.a = c.a0 - 2 * S * c.bxx + S * S * c.qxx;
    b.b = c.b0 - S * (c.bxpy + c.bypx) + S * S * c.qxy;
    b.d = c.d0 - 2 * S * c.bypy + S * S * c.qyy;
    b.rxy = (b.a <= 0 || b.d <= 0) ? 0.0 : (b.b / std::sqrt(b.a)) / std::sqrt(b.d);
    bool ok = std::isfinite(b.a) && std::isfinite(b.b) && std::isfinite(b.d) && b.a > 0 && b.d > 0;
    if (ok) {
        const double rho = (b.b / std::sqrt(b.a)) / std::sqrt(b.d);
        ok = std::isfinite(rho) && std::fma(-rho, rho, 1.0) > std::sqrt(2.220446049250313e-16);
    }
    b.resolved = ok;
    b.lam = ok ? b.b / b.a : 0.0;
    const double rcv = ok ? jmax(std::fma(-b.rxy, b.rxy, 1.0), 0.0) : 0.0;
    b.sigc = ok ? std::sqrt(b.d * rcv) : 0.0;
    return b;
}

bool boundary_resolved(int64_t n, const Boundary &L, const Boundary &R) {  // gaussian_pic.jl:525-530
    return n >= 2 && std::isfinite(L.sigx) && std::isfinite(L.sigy) && std::isfinite(R.sigx) &&
           std::isfinite(R.sigy) && L.sigx > 0 && L.sigy > 0 && R.sigx > 0 && R.sigy > 0;
}
// _gpic_control_variate_mode (gaussian_pic.jl:525-536): 0 plain PIC, 1 uncoupled, 2 coupled.
int control_variate_mode(int64_t n, double tol, const Boundary &L, const Boundary &R) {
    if (!boundary_resolved(n, L, R)) return 0;
    const bool requested = std::isfinite(tol) && jmax(std::fabs(L.rxy), std::fabs(R.rxy)) > tol;
    if (!requested) return 1;
    return L.resolved && R.resolved ? 2 : 0;
}

// Deposit, subtract the (neutralised) erf-integrated reference Gaussian -- separable, or the tilted one as three
// outer products when coupled -- and solve (gaussian_pic.jl:559-640).
void solve_drifted_gaussian(const Options &O, Workspace &ws, FieldPlanes &fp, const Coords &src, double s,
                            const Grid &sg, const std::vector<cplx> &gfft, const Boundary &b, bool coupled) {
    const int nx = O.o.nx, ny = O.o.ny;
    const double hx = sg.width / (double)(nx - 1), hy = sg.height / (double)(ny - 1);
    std::fill(ws.charge.begin(), ws.charge.end(), 0.0);
    deposit_grid(ws.charge.data(), 2 * nx, O.o.deposit_method, src.x.data(), src.px.data(), src.y.data(),
                 src.py.data(), (int64_t)src.size(), true, s, sg.x0, sg.y0, hx, hy, nx, ny,
                 O.o.fixed_point_deposit != 0, nullptr);
    std::vector<double> gx(nx), gy(ny);
    double qsum = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) qsum += ws.charge[i + (size_t)j * 2 * nx];
    if (coupled) {  // the tilted Gaussian to second order in lambda (gaussian_pic.jl:597-630)
        std::vector<double> m1x(nx), m2x(nx), dgy(ny), ddgy(ny);
        coupled_profiles(O.o.deposit_method, sg.x0, hx, b.mux, std::sqrt(b.a), nx, sg.y0, hy, b.muy, b.sigc, ny,
                         gx.data(), m1x.data(), m2x.data(), gy.data(), dgy.data(), ddgy.data());
        const double lam = b.lam, half_lam2 = 0.5 * lam * lam;
        auto sum = [](const std::vector<double> &v) { double t = 0; for (double e : v) t += e; return t; };
        const double sgm = sum(gx) * sum(gy) + lam * sum(m1x) * sum(dgy) + half_lam2 * sum(m2x) * sum(ddgy);
        const double amp = (O.o.neutralize && sgm != 0.0) ? qsum / sgm : (double)src.size();
        for (int j = 0; j < ny; ++j) {
            const double gj = amp * gy[j], dj = amp * lam * dgy[j], ddj = amp * half_lam2 * ddgy[j];
            for (int i = 0; i < nx; ++i) ws.charge[i + (size_t)j * 2 * nx] -= gx[i] * gj + m1x[i] * dj + m2x[i] * ddj;
        }
    } else {
        gaussian_profile(O.o.deposit_method, sg.x0, hx, b.mux, b.sigx, nx, gx.data());
        gaussian_profile(O.o.deposit_method, sg.y0, hy, b.muy, b.sigy, ny, gy.data());
        double sgx = 0, sgy = 0;
        for (double v : gx) sgx += v;
        for (double v : gy) sgy += v;
        double amp = (double)src.size();
        if (O.o.neutralize && sgx * sgy > 0.0) amp = qsum / (sgx * sgy);
        for (int j = 0; j < ny; ++j) {
            const double gj = amp * gy[j];
            for (int i = 0; i < nx; ++i) ws.charge[i + (size_t)j * 2 * nx] -= gx[i] * gj;
        }
    }
    for (size_t k = 0; k < ws.charge.size(); ++k) ws.spectral[k] = cplx(ws.charge[k], 0.0);
    ws.fft.run(ws.spectral.data(), false);
    for (size_t k = 0; k < ws.spectral.size(); ++k) ws.spectral[k] *= gfft[k];
    ws.fft.run(ws.spectral.data(), true);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) fp.phi[i + (size_t)j * nx] = ws.spectral[i + (size_t)j * 2 * nx].real();
    field_from_phi(fp.phi.data(), nx, ny, hx, hy, O.o.field_derivative == 4, fp.Ex.data(), fp.Ey.data());
}

// One directed Gaussian-subtracted interaction (gaussian_pic.jl:604-810); falls back to plain PIC when
// the drifted source moments are degenerate (gaussian_pic.jl:542-553, 634-637).
void interaction_gaussian(Ctx &C, Workspace &ws, const Coords &source, const SliceParam &ps, Coords &field,
                          const SliceParam &pf, double kbb, int i, int j, int dir, int vslot, int64_t counters[3]) {
    const Options &O = C.O;
    const int nsource = (int)source.size(), nfield = (int)field.size();
    const double sL = 0.5 * (ps.center - pf.lb);
    const double sR = 0.5 * (ps.center - pf.rb);
    const bool gate = std::isfinite(O.o.coupling_tol);  // the cross-plane sums only when they can be read
    const SourceMoments mom = source_moments(source, gate);
    const Boundary bL = boundary(mom, sL, gate), bR = boundary(mom, sR, gate);
    const int mode = control_variate_mode(mom.n, O.o.coupling_tol, bL, bR);
    if (mode == 0) {
        interaction(C, ws, source, ps, field, pf, kbb, i, j, dir, vslot, counters);
        return;
    }
    const bool use_coupled = mode == 2;
    const CovMoments cmom = coupled_moments(mom);
    const double margin = O.o.margin_sigma;
    double sxl = source.x[0] + source.px[0] * sL, syl = source.y[0] + source.py[0] * sL;
    double sxr = source.x[0] + source.px[0] * sR, syr = source.y[0] + source.py[0] * sR;
    double sxmin = jmin(sxl, sxr), sxmax = jmax(sxl, sxr), symin = jmin(syl, syr), symax = jmax(syl, syr);
    for (int k = 1; k < nsource; ++k) {
        const double xl = source.x[k] + source.px[k] * sL, yl = source.y[k] + source.py[k] * sL;
        const double xr = source.x[k] + source.px[k] * sR, yr = source.y[k] + source.py[k] * sR;
        sxmin = jmin(jmin(sxmin, xl), xr); sxmax = jmax(jmax(sxmax, xl), xr);
        symin = jmin(jmin(symin, yl), yr); symax = jmax(jmax(symax, yl), yr);
    }
    if (margin > 0) {
        const double gxlo = jmin(bL.mux - margin * bL.sigx, bR.mux - margin * bR.sigx);
        const double gxhi = jmax(bL.mux + margin * bL.sigx, bR.mux + margin * bR.sigx);
        const double gylo = jmin(bL.muy - margin * bL.sigy, bR.muy - margin * bR.sigy);
        const double gyhi = jmax(bL.muy + margin * bL.sigy, bR.muy + margin * bR.sigy);
        sxmin = jmin(sxmin, gxlo); sxmax = jmax(sxmax, gxhi);
        symin = jmin(symin, gylo); symax = jmax(symax, gyhi);
    }
    if (!(std::isfinite(sxmin) && std::isfinite(sxmax) && std::isfinite(symin) && std::isfinite(symax)))
        nonfinite("source", source, pair_ctx(i, j, dir));
    double fxmin = field.x[0] + 0.5 * (field.z[0] - ps.center) * field.px[0];
    double fxmax = fxmin;
    double fymin = field.y[0] + 0.5 * (field.z[0] - ps.center) * field.py[0];
    double fymax = fymin;
    const bool lk = O.o.longitudinal_kick != 0;
    for (int k = 0; k < nfield; ++k) {
        const double s = 0.5 * (field.z[k] - ps.center);
        field.x[k] += s * field.px[k];
        field.y[k] += s * field.py[k];
        if (lk) field.pz[k] -= 0.25 * (field.px[k] * field.px[k] + field.py[k] * field.py[k]);
        fxmin = jmin(fxmin, field.x[k]); fxmax = jmax(fxmax, field.x[k]);
        fymin = jmin(fymin, field.y[k]); fymax = jmax(fymax, field.y[k]);
    }
    if (!(std::isfinite(fxmin) && std::isfinite(fxmax) && std::isfinite(fymin) && std::isfinite(fymax)))
        nonfinite("field", field, pair_ctx(i, j, dir));
    Grid sg, fg;
    interaction_grids(O, sxmin, sxmax, symin, symax, fxmin, fxmax, fymin, fymax, sg, fg);
    Bounds sb{sxmin, sxmax, symin, symax}, fb{fxmin, fxmax, fymin, fymax};
    std::vector<cplx> own;
    const std::vector<cplx> &gfft = slice_pair_green(C, ws, i, j, dir, sg, fg, sb, fb, own, counters);
    solve_drifted_gaussian(O, ws, ws.left, source, sL, sg, gfft, bL, use_coupled);
    solve_drifted_gaussian(O, ws, ws.right, source, sR, sg, gfft, bR, use_coupled);

    const double ks = 2.0 * kbb;
    const double half_ns = 0.5 * (double)nsource;
    const double kbb_eff = ks * half_ns;
    double hzi, zbias;
    slice_interp_params(pf.lb, pf.rb, hzi, zbias);
    for (int k = 0; k < nfield; ++k) {
        const double x = field.x[k], y = field.y[k];
        const double zL = jclamp(-field.z[k] * hzi + zbias, 0.0, 1.0);
        const double zR = 1.0 - zL;
        double Kxd, Kyd, Kzd;
        interpolate_kick(O, fg, x, y, ws.left, ws.right, zL, zR, Kxd, Kyd, Kzd);
        if (use_coupled) {  // rotated analytic add-back through _cp_covariance_kick (gaussian_pic.jl:837-854)
            double pxL = 0, pyL = 0, pzL = 0, pxR = 0, pyR = 0, pzR = 0;
            coupled_covariance_kick(cmom, kbb_eff, -bL.s, x - bL.mux, y - bL.muy, pxL, pyL, pzL);
            coupled_covariance_kick(cmom, kbb_eff, -bR.s, x - bR.mux, y - bR.muy, pxR, pyR, pzR);
            const double dpxa = zL * pxL + zR * pxR;
            const double dpya = zL * pyL + zR * pyR;
            field.px[k] += ks * Kxd + dpxa;
            field.py[k] += ks * Kyd + dpya;
            if (lk) {
                field.pz[k] += ks * Kzd * hzi;
                field.pz[k] += zL * pzL + zR * pzR;
                field.pz[k] += 0.5 * (dpxa * mom.mpx + dpya * mom.mpy);
            }
            const double s = 0.5 * (ps.center - field.z[k]);
            field.x[k] += s * field.px[k];
            field.y[k] += s * field.py[k];
            if (lk) field.pz[k] += 0.25 * (field.px[k] * field.px[k] + field.py[k] * field.py[k]);
            continue;
        }
        double bLx, bLy, HxL = 0, HyL = 0, bRx, bRy, HxR = 0, HyR = 0;
        if (lk) {
            be::response(kbb_eff, bL.sigx, bL.sigy, x - bL.mux, y - bL.muy, bLx, bLy, HxL, HyL);
            be::response(kbb_eff, bR.sigx, bR.sigy, x - bR.mux, y - bR.muy, bRx, bRy, HxR, HyR);
        } else {
            be::kick(bL.sigx, bL.sigy, x - bL.mux, y - bL.muy, bLx, bLy);
            be::kick(bR.sigx, bR.sigy, x - bR.mux, y - bR.muy, bRx, bRy);
        }
        const double Kxa = half_ns * (zL * bLx + zR * bRx);
        const double Kya = half_ns * (zL * bLy + zR * bRy);
        const double dpxa = ks * Kxa, dpya = ks * Kya;
        field.px[k] += ks * Kxd + dpxa;
        field.py[k] += ks * Kyd + dpya;
        if (lk) {
            const double covL = (HxL * bL.rx + HyL * bL.ry) / 4.0;
            const double covR = (HxR * bR.rx + HyR * bR.ry) / 4.0;
            field.pz[k] += ks * Kzd * hzi;
            field.pz[k] += zL * covL + zR * covR;
            field.pz[k] += 0.5 * (dpxa * mom.mpx + dpya * mom.mpy);
        }
        const double s = 0.5 * (ps.center - field.z[k]);
        field.x[k] += s * field.px[k];
        field.y[k] += s * field.py[k];
        if (lk) field.pz[k] += 0.25 * (field.px[k] * field.px[k] + field.py[k] * field.py[k]);
    }
    const double sM = 0.5 * (ps.center - pf.center);
    virtual_positions(source, sM, ws.vx[vslot], ws.vy[vslot]);
}

void interaction_node(Ctx &C, Workspace &ws, const Coords &source, const SliceParam &ps, Coords &field,
                      const SliceParam &pf, double kbb, const NodeMesh &gL, const NodeMesh &gR, int vslot) {
    const Options &O = C.O;
    bool lk = O.o.longitudinal_kick != 0;
    double sL = 0.5 * (ps.center - pf.lb);
    double sR = 0.5 * (ps.center - pf.rb);
    int nfield = (int)field.size();
    for (int k = 0; k < nfield; ++k) {
        double s = 0.5 * (field.z[k] - ps.center);
        field.x[k] += s * field.px[k];
        field.y[k] += s * field.py[k];
        if (lk) field.pz[k] -= 0.25 * (field.px[k] * field.px[k] + field.py[k] * field.py[k]);
    }
    ws.dropped += count_outside_drifted(source, sL, sL, gL.sg.x0, gL.sg.x0 + gL.sg.width, gL.sg.y0,
                                        gL.sg.y0 + gL.sg.height);
    ws.dropped += count_outside_drifted(source, sR, sR, gR.sg.x0, gR.sg.x0 + gR.sg.width, gR.sg.y0,
                                        gR.sg.y0 + gR.sg.height);
    ws.dropped += count_outside(field.x, field.y, gL.fg.x0, gL.fg.x0 + gL.fg.width, gL.fg.y0, gL.fg.y0 + gL.fg.height);
    solve_drifted(O, ws, ws.left, source, sL, gL.sg, gL.gfft, true, 0);
    solve_drifted(O, ws, ws.right, source, sR, gR.sg, gR.gfft, true, 1);
    if (lk) solve_drifted(O, ws, ws.mid, source, sR, gL.sg, gL.gfft, true, 2);
    double ks = 2.0 * kbb;
    double hzi, zbias;
    slice_interp_params(pf.lb, pf.rb, hzi, zbias);
    for (int k = 0; k < nfield; ++k) {
        double zL = jclamp(-field.z[k] * hzi + zbias, 0.0, 1.0);
        double zR = 1.0 - zL;
        double x = field.x[k], y = field.y[k];
        double KxL, KyL, KzL, KxR, KyR, KzR;
        interpolate_kick(O, gL.fg, x, y, ws.left, ws.left, 1.0, 0.0, KxL, KyL, KzL);
        interpolate_kick(O, gR.fg, x, y, ws.right, ws.right, 1.0, 0.0, KxR, KyR, KzR);
        field.px[k] += ks * (zL * KxL + zR * KxR);
        field.py[k] += ks * (zL * KyL + zR * KyR);
        if (lk) {
            double a, b, Kz;
            // phiZ paired with the L transverse planes (pic_cpu.jl:1522-1523)
            interpolate_kick(O, gL.fg, x, y, ws.left, ws.mid, 1.0, 0.0, a, b, Kz);
            field.pz[k] += ks * Kz * hzi;
        }
        double s = 0.5 * (ps.center - field.z[k]);
        field.x[k] += s * field.px[k];
        field.y[k] += s * field.py[k];
        if (lk) field.pz[k] += 0.25 * (field.px[k] * field.px[k] + field.py[k] * field.py[k]);
    }
    double sM = 0.5 * (ps.center - pf.center);
    virtual_positions(source, sM, ws.vx[vslot], ws.vy[vslot]);
}

// pic_cpu.jl:1317-1382 : all node meshes of one (source slice, direction)
void build_node_meshes(Ctx &C, Workspace &ws, const Coords &src, double center, const double *fb[6],
                       const Slices &fs, std::vector<NodeMesh> &out) {
    const Options &O = C.O;
    int nb = (int)fs.boundary.size(), ns = nb - 1;
    double c = center;
    std::vector<double> drifts(nb);
    for (int b = 0; b < nb; ++b) drifts[b] = 0.5 * (c - fs.boundary[b]);
    std::vector<double> sxlo(nb, INFINITY), sxhi(nb, -INFINITY), sylo(nb, INFINITY), syhi(nb, -INFINITY);
    for (size_t k = 0; k < src.size(); ++k) {
        double x = src.x[k], px = src.px[k], y = src.y[k], py = src.py[k];
        for (int b = 0; b < nb; ++b) {
            double d = drifts[b];
            double xv = x + px * d, yv = y + py * d;
            sxlo[b] = jmin(sxlo[b], xv); sxhi[b] = jmax(sxhi[b], xv);
            sylo[b] = jmin(sylo[b], yv); syhi[b] = jmax(syhi[b], yv);
        }
    }
    std::vector<double> fxlo(ns, INFINITY), fxhi(ns, -INFINITY), fylo(ns, INFINITY), fyhi(ns, -INFINITY);
    for (int sl = 0; sl < ns; ++sl)
        for (int64_t i : fs.indices[sl]) {
            double sh = 0.5 * (fb[4][i] - c);
            double xv = fb[0][i] + sh * fb[1][i], yv = fb[2][i] + sh * fb[3][i];
            fxlo[sl] = jmin(fxlo[sl], xv); fxhi[sl] = jmax(fxhi[sl], xv);
            fylo[sl] = jmin(fylo[sl], yv); fyhi[sl] = jmax(fyhi[sl], yv);
        }
    for (int b = 0; b < nb; ++b)
        if (std::isnan(sxlo[b]) || std::isnan(sxhi[b]) || std::isnan(sylo[b]) || std::isnan(syhi[b]))
            throw OracleError(OO_ERR_NONFINITE, "non-finite source coordinate (node-mesh build)");
    for (int b = 0; b < ns; ++b)
        if (std::isnan(fxlo[b]) || std::isnan(fxhi[b]) || std::isnan(fylo[b]) || std::isnan(fyhi[b]))
            throw OracleError(OO_ERR_NONFINITE, "non-finite field coordinate (node-mesh build)");
    out.assign(nb, NodeMesh());
    for (int b = 1; b <= nb; ++b) {
        int bn = std::min(b + 1, nb);
        double sxmin = jmin(sxlo[b - 1], sxlo[bn - 1]), sxmax = jmax(sxhi[b - 1], sxhi[bn - 1]);
        double symin = jmin(sylo[b - 1], sylo[bn - 1]), symax = jmax(syhi[b - 1], syhi[bn - 1]);
        double fxmin = INFINITY, fxmax = -INFINITY, fymin = INFINITY, fymax = -INFINITY;
        for (int adj = b - 1; adj <= b; ++adj) {
            if (!(1 <= adj && adj <= ns)) continue;
            if (!std::isfinite(fxlo[adj - 1])) continue;
            fxmin = jmin(fxmin, fxlo[adj - 1]); fxmax = jmax(fxmax, fxhi[adj - 1]);
            fymin = jmin(fymin, fylo[adj - 1]); fymax = jmax(fymax, fyhi[adj - 1]);
        }
        if (!std::isfinite(fxmin)) continue;
        NodeMesh &m = out[b - 1];
        interaction_grids(O, sxmin, sxmax, symin, symax, fxmin, fxmax, fymin, fymax, m.sg, m.fg);
        green_fft(O, ws, m.sg, m.fg, m.gfft);
        m.valid = true;
    }
}

// pic_cpu.jl:2700-2736
double luminosity(const Options &O, const std::vector<double> &x1, const std::vector<double> &y1,
                  const std::vector<double> &x2, const std::vector<double> &y2, double klum, Workspace &ws) {
    int nx = O.lum_nx(), ny = O.lum_ny();
    double xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY;
    double a = INFINITY, b = -INFINITY, c = INFINITY, d = -INFINITY;
    for (double v : x1) { a = jmin(a, v); b = jmax(b, v); }
    for (double v : y1) { c = jmin(c, v); d = jmax(d, v); }
    double a2 = INFINITY, b2 = -INFINITY, c2 = INFINITY, d2 = -INFINITY;
    for (double v : x2) { a2 = jmin(a2, v); b2 = jmax(b2, v); }
    for (double v : y2) { c2 = jmin(c2, v); d2 = jmax(d2, v); }
    xmin = jmin(a, a2); xmax = jmax(b, b2); ymin = jmin(c, c2); ymax = jmax(d, d2);
    double width, height;
    resolve_extent(O, xmax - xmin, ymax - ymin, width, height, "PIC luminosity grid");
    double tx = width / ((double)nx - 1.1);
    double ty = height / ((double)ny - 1.1);
    width += 0.1 * tx;
    height += 0.1 * ty;
    xmin -= 0.05 * tx;
    ymin -= 0.05 * ty;
    double hx = width / (double)(nx - 1), hy = height / (double)(ny - 1);
    double hxi = 1.0 / hx, hyi = 1.0 / hy;
    int ld = nx + 1;
    ws.q1.assign((size_t)(nx + 1) * (ny + 1), 0.0);
    ws.q2.assign((size_t)(nx + 1) * (ny + 1), 0.0);
    int method = O.lum_method();
    bool fixed = O.o.fixed_point_deposit != 0;
    deposit_grid(ws.q1.data(), ld, method, x1.data(), nullptr, y1.data(), nullptr, (int64_t)x1.size(), false, 0.0,
                 xmin, ymin, hx, hy, nx + 1, ny + 1, fixed, nullptr);
    deposit_grid(ws.q2.data(), ld, method, x2.data(), nullptr, y2.data(), nullptr, (int64_t)x2.size(), false, 0.0,
                 xmin, ymin, hx, hy, nx + 1, ny + 1, fixed, nullptr);
    double lum = 0.0;
    for (int j = 0; j < ny + 1; ++j)
        for (int i = 0; i < nx + 1; ++i) lum += ws.q1[i + (size_t)j * ld] * ws.q2[i + (size_t)j * ld];
    return lum * klum * hxi * hyi;
}

void gather(const double *b[6], const std::vector<int64_t> &idx, Coords &c) {
    c.resize(idx.size());
    for (size_t k = 0; k < idx.size(); ++k) {
        int64_t i = idx[k];
        c.x[k] = b[0][i]; c.px[k] = b[1][i]; c.y[k] = b[2][i];
        c.py[k] = b[3][i]; c.z[k] = b[4][i]; c.pz[k] = b[5][i];
    }
}

void validate(const Options &O) {
    const oo_options &o = O.o;
    if (o.nx < 5 || o.ny < 5) throw OracleError(OO_ERR_ARG, "PICPoissonSolver grid must be at least (5, 5)");
    if (o.deposit_method < 0 || o.deposit_method > 1) throw OracleError(OO_ERR_ARG, "deposit_method");
    if (o.green_type < 0 || o.green_type > 1) throw OracleError(OO_ERR_UNSUPPORTED, "green_type");
    if (o.interaction_grid < 0 || o.interaction_grid > 2) throw OracleError(OO_ERR_UNSUPPORTED, "interaction_grid");
    if (o.interaction_grid != 0 && o.grid_extent != 0)
        throw OracleError(OO_ERR_UNSUPPORTED, "grid_extent != :extrema with interaction_grid != :slice_pair");
    if (o.interaction_grid == 2 && o.slice_interpolation != 0)
        throw OracleError(OO_ERR_UNSUPPORTED, "slice_interpolation = :quadratic with interaction_grid = :node");
    if (o.gaussian && (o.slice_interpolation != 0 || o.interaction_grid != 0 || o.grid_extent != 0))
        throw OracleError(OO_ERR_UNSUPPORTED, "GaussianPICPoissonSolver needs linear slice interpolation on the "
                                              ":slice_pair grid with grid_extent = :extrema");
    if (o.gaussian && !(o.margin_sigma >= 0)) throw OracleError(OO_ERR_ARG, "margin_sigma must be non-negative");
    if (o.gaussian && !(o.coupling_tol >= 0)) throw OracleError(OO_ERR_ARG, "coupling_tol must be non-negative");
}

int nslices_of(const oo_options &o, int which) {
    int method = which == 1 ? o.slicing_method1 : o.slicing_method2;
    int ns = which == 1 ? o.nslices1 : o.nslices2;
    return method == 1 ? ns : ns;  // :specified uses nslices-1 positions (interface.jl:828-829)
}

// pic_cpu.jl:82-275
double collide(Ctx &C, double *b1[6], int64_t n1, double *b2[6], int64_t n2, const oo_beam_params &p1,
               const oo_beam_params &p2, bool compute_lum) {
    Options &O = C.O;
    validate(O);
    Slices s1 = make_slices(O.o.slicing_method1, O.o.nslices1, O.o.center_position1, O.pos1, b1[4], n1,
                            O.o.resolution1 > 0 ? O.o.resolution1 : 100);
    Slices s2 = make_slices(O.o.slicing_method2, O.o.nslices2, O.o.center_position2, O.pos2, b2[4], n2,
                            O.o.resolution2 > 0 ? O.o.resolution2 : 100);
    int ns1 = (int)s1.center.size(), ns2 = (int)s2.center.size();
    if (C.cache.empty() || ns1 != C.ns1 || ns2 != C.ns2) {
        C.ns1 = ns1; C.ns2 = ns2;
        C.cache.assign((size_t)2 * ns1 * ns2, GreenEntry());
    }
    // slicing.jl:77-91 and pic_cpu.jl:821-829
    double kbb1p = O.o.has_kbb1 ? O.o.kbb1 : p1.charge * p2.charge * p1.r0 * p2.npart * p1.mc2 / p1.E0;
    double kbb2p = O.o.has_kbb2 ? O.o.kbb2 : p1.charge * p2.charge * p2.r0 * p1.npart * p2.mc2 / p2.E0;
    if (!O.o.has_kbb1 && !(std::isfinite(p1.E0) && p1.E0 != 0))
        throw OracleError(OO_ERR_ARG, "beam1 E0 must be finite and nonzero when kbb1 is not specified");
    if (!O.o.has_kbb2 && !(std::isfinite(p2.E0) && p2.E0 != 0))
        throw OracleError(OO_ERR_ARG, "beam2 E0 must be finite and nonzero when kbb2 is not specified");
    double kbb1 = kbb1p / (double)n2;
    double kbb2 = kbb2p / (double)n1;
    double klum = O.o.has_lum_scale ? O.o.lum_scale : p1.npart * p2.npart / (double)(n1 * n2);

    int nx = O.o.nx, ny = O.o.ny;
    bool node = O.o.interaction_grid == 2;
    int nthreads = O.o.nthreads > 0 ? O.o.nthreads : 1;
    std::vector<Workspace> wss(nthreads);
    for (auto &w : wss) w.init(nx, ny);

    std::vector<Coords> state1(ns1), state2(ns2), scratch2(ns2);
    const double *cb1[6] = {b1[0], b1[1], b1[2], b1[3], b1[4], b1[5]};
    const double *cb2[6] = {b2[0], b2[1], b2[2], b2[3], b2[4], b2[5]};
    for (int s = 0; s < ns1; ++s) gather(cb1, s1.indices[s], state1[s]);
    for (int s = 0; s < ns2; ++s) { gather(cb2, s2.indices[s], state2[s]); scratch2[s] = state2[s]; }

    // pic_cpu.jl:1404-1419 : node meshes from the turn-start state
    std::vector<std::vector<NodeMesh>> node1(ns1), node2(ns2);
    std::string first_err;
    int first_code = 0;
    if (node) {
#pragma omp parallel for num_threads(nthreads) schedule(dynamic)
        for (int t = 0; t < ns1 + ns2; ++t) {
            try {
#ifdef _OPENMP
                Workspace &w = wss[omp_get_thread_num()];
#else
                Workspace &w = wss[0];
#endif
                if (t < ns1) {
                    if (!s1.indices[t].empty()) build_node_meshes(C, w, state1[t], s1.center[t], cb2, s2, node1[t]);
                } else {
                    int s = t - ns1;
                    if (!s2.indices[s].empty()) build_node_meshes(C, w, state2[s], s2.center[s], cb1, s1, node2[s]);
                }
            } catch (OracleError &e) {
#pragma omp critical
                if (!first_code) { first_code = e.code; first_err = e.what(); }
            }
        }
        if (first_code) throw OracleError(first_code, first_err);
    }

    auto order = collision_order(s1.center, s2.center);
    size_t npairs = order.size();
    std::vector<int> pos_of((size_t)ns1 * ns2);
    for (size_t p = 0; p < npairs; ++p) pos_of[(size_t)(order[p].i - 1) * ns2 + (order[p].j - 1)] = (int)p;
    std::vector<double> lum_parts(npairs, 0.0);
    std::vector<char> ran(npairs, 0);
    // :source_slice runs the pairs one at a time in collision order (pic_cpu.jl:54, 240-248): its union boxes are
    // taken at each source slice's first use, from the states as that pair finds them
    const bool shared = O.o.interaction_grid == 1;
    std::vector<std::vector<OrderEntry>> batches;
    if (shared)
        for (const OrderEntry &e : order) batches.push_back({e});
    else
        batches = pair_batches(s1.center, s2.center);
    std::vector<std::array<int64_t, 3>> counters(npairs, {0, 0, 0});
    std::vector<UnionBounds> ub1(shared ? ns1 : 0), ub2(shared ? ns2 : 0);
    std::vector<char> ub1_done(shared ? ns1 : 0, 0), ub2_done(shared ? ns2 : 0, 0);

    for (auto &batch : batches) {
#pragma omp parallel for num_threads(nthreads) schedule(dynamic)
        for (int q = 0; q < (int)batch.size(); ++q) {
#ifdef _OPENMP
            Workspace &ws = wss[omp_get_thread_num()];
#else
            Workspace &ws = wss[0];
#endif
            int i = batch[q].i, j = batch[q].j;
            int p = pos_of[(size_t)(i - 1) * ns2 + (j - 1)];
            try {
                if (s1.indices[i - 1].empty() || s2.indices[j - 1].empty()) continue;
                SliceParam pa1{s1.weight[i - 1], s1.boundary[i - 1], s1.center[i - 1], s1.boundary[i]};
                SliceParam pa2{s2.weight[j - 1], s2.boundary[j - 1], s2.center[j - 1], s2.boundary[j]};
                Coords &coord1 = state1[i - 1];
                Coords &coord2 = state2[j - 1];
                Coords &field2 = scratch2[j - 1];
                field2 = coord2;
                // the armed charge-grid capture, if it is one of this pair's interactions
                auto arm = [&](int dir) {
                    const bool hit = C.cap.armed && !C.cap.taken && C.cap.i == i && C.cap.j == j && C.cap.dir == dir;
                    ws.cap = hit ? &C.cap : nullptr;
                    ws.cap_kind = hit ? C.cap.kind : -1;
                };
                arm(1);
                if (node) {
                    auto &nc1 = node1[i - 1];
                    auto &nc2 = node2[j - 1];
                    if (nc1.empty() || nc2.empty()) throw OracleError(OO_ERR_ARG, "node mesh cache missing");
                    const NodeMesh &gL1 = nc1[j - 1], &gR1 = nc1[j], &gL2 = nc2[i - 1], &gR2 = nc2[i];
                    if (!gL1.valid || !gR1.valid || !gL2.valid || !gR2.valid) continue;
                    interaction_node(C, ws, coord1, pa1, field2, pa2, kbb2, gL1, gR1, 0);
                    arm(2);
                    interaction_node(C, ws, coord2, pa2, coord1, pa1, kbb1, gL2, gR2, 1);
                } else if (O.o.gaussian) {
                    interaction_gaussian(C, ws, coord1, pa1, field2, pa2, kbb2, i, j, 1, 0, counters[p].data());
                    interaction_gaussian(C, ws, coord2, pa2, coord1, pa1, kbb1, i, j, 2, 1, counters[p].data());
                } else {
                    const UnionBounds *ov1 = nullptr, *ov2 = nullptr;
                    if (shared) {  // both boxes before either direction kicks (pic_cpu.jl:368-371)
                        if (!ub1_done[i - 1]) { ub1[i - 1] = union_bounds(coord1, pa1.center, state2); ub1_done[i - 1] = 1; }
                        if (!ub2_done[j - 1]) { ub2[j - 1] = union_bounds(coord2, pa2.center, state1); ub2_done[j - 1] = 1; }
                        ov1 = &ub1[i - 1];
                        ov2 = &ub2[j - 1];
                    }
                    interaction(C, ws, coord1, pa1, field2, pa2, kbb2, i, j, 1, 0, counters[p].data(), ov1);
                    arm(2);
                    interaction(C, ws, coord2, pa2, coord1, pa1, kbb1, i, j, 2, 1, counters[p].data(), ov2);
                }
                ws.cap = nullptr;
                ws.cap_kind = -1;
                std::swap(state2[j - 1], scratch2[j - 1]);
                if (compute_lum) lum_parts[p] = luminosity(O, ws.vx[0], ws.vy[0], ws.vx[1], ws.vy[1], klum, ws);
                ran[p] = 1;
            } catch (OracleError &e) {
#pragma omp critical
                if (!first_code) { first_code = e.code; first_err = e.what(); }
            }
        }
        if (first_code) throw OracleError(first_code, first_err);
    }
    for (auto &c : counters) { C.hits += c[0]; C.misses += c[1]; C.rebuilds += c[2]; }

    // scatter back (pic_cpu.jl:255-256)
    for (int s = 0; s < ns1; ++s)
        for (size_t k = 0; k < s1.indices[s].size(); ++k) {
            int64_t i = s1.indices[s][k];
            const Coords &c = state1[s];
            b1[0][i] = c.x[k]; b1[1][i] = c.px[k]; b1[2][i] = c.y[k]; b1[3][i] = c.py[k]; b1[4][i] = c.z[k]; b1[5][i] = c.pz[k];
        }
    for (int s = 0; s < ns2; ++s)
        for (size_t k = 0; k < s2.indices[s].size(); ++k) {
            int64_t i = s2.indices[s][k];
            const Coords &c = state2[s];
            b2[0][i] = c.x[k]; b2[1][i] = c.px[k]; b2[2][i] = c.y[k]; b2[3][i] = c.py[k]; b2[4][i] = c.z[k]; b2[5][i] = c.pz[k];
        }
    C.dropped = 0;
    for (auto &w : wss) C.dropped += w.dropped;
    C.trace_i.clear(); C.trace_j.clear(); C.trace_lum.clear();
    double lum = NAN;
    if (compute_lum) {
        lum = 0.0;
        for (size_t p = 0; p < npairs; ++p) {
            if (!ran[p]) continue;
            lum += lum_parts[p];
            C.trace_i.push_back(order[p].i);
            C.trace_j.push_back(order[p].j);
            C.trace_lum.push_back(lum_parts[p]);
        }
    }
    return lum;
}

Options make_options(const oo_options *o) {
    Options O;
    O.o = *o;
    if (o->slicing_method1 == 1 && o->positions1) O.pos1.assign(o->positions1, o->positions1 + (o->nslices1 - 1));
    if (o->slicing_method2 == 1 && o->positions2) O.pos2.assign(o->positions2, o->positions2 + (o->nslices2 - 1));
    O.o.positions1 = nullptr;
    O.o.positions2 = nullptr;
    return O;
}

}  // namespace

extern "C" {

void oo_philox4x32_block(const uint32_t c[4], const uint32_t k[2], uint32_t out[4]) {
    uint32_t w[4] = {c[0], c[1], c[2], c[3]};
    philox_block(w, k[0], k[1]);
    for (int i = 0; i < 4; ++i) out[i] = w[i];
}
uint64_t oo_counter_uint64(uint64_t seed, uint64_t turn, uint64_t rng_id, uint64_t particle, uint64_t component) {
    return counter_u64(seed, turn, rng_id, particle, component);
}
double oo_normal(uint64_t seed, uint64_t turn, uint64_t rng_id, uint64_t particle, uint64_t component) {
    return counter_normal(seed, turn, rng_id, particle, component);
}

// Beam.jl:475-515, 127-181, 545-553 (counter-RNG Gaussian beam, sigma/Twiss normalisation)
void oo_beam_gaussian(int64_t n, uint64_t seed, uint64_t rng_id, const double beta[3], const double alpha[3],
                      const double sigma[3], double cutoff, double *x, double *px, double *y, double *py, double *z,
                      double *pz) {
    double *c[6] = {x, px, y, py, z, pz};
    for (int d = 0; d < 6; ++d) {
        double *v = c[d];
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double g = counter_normal(seed, 0, rng_id, (uint64_t)(i + 1), (uint64_t)(d + 1));
            v[i] = std::isfinite(cutoff) ? jclamp(g, -cutoff, cutoff) : g;
        }
        standardize(v, n);
    }
    for (int a = 0; a < 3; ++a) {
        double *q = c[2 * a], *p = c[2 * a + 1];
        double f = sigma[a] / beta[a];
        for (int64_t i = 0; i < n; ++i) p[i] = f * (p[i] - alpha[a] * q[i]);
        for (int64_t i = 0; i < n; ++i) q[i] *= sigma[a];
    }
}

double oo_erfinv(double x) { return erfinv_impl(x); }
void oo_faddeeva(double zr, double zi, double out[2]) { be::faddeeva(zr, zi, out[0], out[1]); }
void oo_be_response(double kbb, double sigx, double sigy, double x, double y, double out[4]) {
    be::response(kbb, sigx, sigy, x, y, out[0], out[1], out[2], out[3]);
}
void oo_gaussian_profile(int32_t method, double x0, double h, double mu, double sigma, int32_t n, double *g) {
    gaussian_profile(method, x0, h, mu, sigma, n, g);
}
double oo_kernel_integral(double x, double y) { return kernel_integral(x, y); }
double oo_atan_ratio(double num, double den) { return atan_ratio(num, den); }
void oo_cic_weights(double u, int32_t n, int32_t *base, double w[2]) { int b; cic_weights(u, n, b, w); *base = b; }
void oo_tsc_weights(double u, int32_t n, int32_t *base, double w[3]) { int b; tsc_weights(u, n, b, w); *base = b; }
void oo_green_table(int32_t green_type, double fx0, double fy0, double sx0, double sy0, double hx, double hy,
                    int32_t nx, int32_t ny, double *out) {
    green_table(green_type, fx0, fy0, sx0, sy0, hx, hy, nx, ny, out);
}
void oo_fft2(double *re, double *im, int32_t n1, int32_t n2, int32_t inverse) {
    Fft2D f;
    f.init(n1, n2);
    std::vector<cplx> a((size_t)n1 * n2);
    for (size_t k = 0; k < a.size(); ++k) a[k] = cplx(re[k], im[k]);
    f.run(a.data(), inverse != 0);
    for (size_t k = 0; k < a.size(); ++k) { re[k] = a[k].real(); im[k] = a[k].imag(); }
}
void oo_field(const double *phi, int32_t nx, int32_t ny, double hx, double hy, int32_t fourth, double *Ex,
              double *Ey) {
    field_from_phi(phi, nx, ny, hx, hy, fourth != 0, Ex, Ey);
}
int32_t oo_fixed_scale_bits(int64_t nsrc) { return fixed_bits(nsrc); }
void oo_deposit_drifted(int32_t method, const double *x, const double *px, const double *y, const double *py,
                        int64_t n, double s, double x0, double y0, double hx, double hy, int32_t nx, int32_t ny,
                        int32_t fixed, double *charge, int64_t *qfix) {
    deposit_grid(charge, 2 * nx, method, x, px, y, py, n, true, s, x0, y0, hx, hy, nx, ny, fixed != 0, qfix);
}
void oo_solve_field(const oo_options *opt, const double *x, const double *y, int64_t n, double sx0, double sy0,
                    double sw, double sh, double fx0, double fy0, double *phi, double *Ex, double *Ey) {
    Options O = make_options(opt);
    Workspace ws;
    ws.init(O.o.nx, O.o.ny);
    Grid sg{sx0, sy0, sw, sh}, fg{fx0, fy0, sw, sh};
    std::vector<cplx> g;
    green_fft(O, ws, sg, fg, g);
    Coords src;
    src.x.assign(x, x + n); src.y.assign(y, y + n);
    src.px.assign(n, 0.0); src.py.assign(n, 0.0); src.z.assign(n, 0.0); src.pz.assign(n, 0.0);
    solve_drifted(O, ws, ws.left, src, 0.0, sg, g, false);
    size_t m = (size_t)O.o.nx * O.o.ny;
    std::copy(ws.left.phi.begin(), ws.left.phi.begin() + m, phi);
    std::copy(ws.left.Ex.begin(), ws.left.Ex.begin() + m, Ex);
    std::copy(ws.left.Ey.begin(), ws.left.Ey.begin() + m, Ey);
}
void oo_interpolation_grids(const oo_options *opt, const double b[8], double out[8]) {
    Options O = make_options(opt);
    Grid sg, fg;
    interaction_grids(O, b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], sg, fg);
    out[0] = sg.x0; out[1] = sg.y0; out[2] = sg.width; out[3] = sg.height;
    out[4] = fg.x0; out[5] = fg.y0; out[6] = fg.width; out[7] = fg.height;
}

void oo_interpolate(const oo_options *opt, const double grid[4], double x, double y, const double *phiL,
                    const double *ExL, const double *EyL, const double *phiM, const double *ExM, const double *EyM,
                    const double *phiR, const double *ExR, const double *EyR, int32_t quadratic, double param,
                    double out[3]) {
    Options O = make_options(opt);
    size_t m = (size_t)O.o.nx * O.o.ny;
    FieldPlanes L, M, R;
    L.phi.assign(phiL, phiL + m); L.Ex.assign(ExL, ExL + m); L.Ey.assign(EyL, EyL + m);
    R.phi.assign(phiR, phiR + m); R.Ex.assign(ExR, ExR + m); R.Ey.assign(EyR, EyR + m);
    Grid g{grid[0], grid[1], grid[2], grid[3]};
    if (quadratic) {
        M.phi.assign(phiM, phiM + m); M.Ex.assign(ExM, ExM + m); M.Ey.assign(EyM, EyM + m);
        interpolate_kick_quadratic(O, g, x, y, L, M, R, param, out[0], out[1], out[2]);
    } else {
        interpolate_kick(O, g, x, y, L, R, param, 1.0 - param, out[0], out[1], out[2]);
    }
}

double oo_luminosity(const oo_options *opt, const double *x1, const double *y1, int64_t n1, const double *x2,
                     const double *y2, int64_t n2, double klum, double *q1, double *q2) {
    Options O = make_options(opt);
    Workspace ws;
    std::vector<double> a(x1, x1 + n1), b(y1, y1 + n1), c(x2, x2 + n2), d(y2, y2 + n2);
    double lum;
    try {
        lum = luminosity(O, a, b, c, d, klum, ws);
    } catch (OracleError &) {
        return NAN;
    }
    if (q1) std::copy(ws.q1.begin(), ws.q1.end(), q1);
    if (q2) std::copy(ws.q2.begin(), ws.q2.end(), q2);
    return lum;
}

void oo_julia_range(double start, double stop, int64_t len, double *out) {
    const std::vector<double> r = julia_range(start, stop, len);
    std::copy(r.begin(), r.end(), out);
}

int oo_slices(int32_t method, int32_t ns, int32_t center_position, const double *positions, const double *z,
              int64_t n, double *boundary, double *center, double *weight, int64_t *count, int64_t *order,
              int32_t resolution) {
    try {
        std::vector<double> pos;
        if (method == 1 && positions) pos.assign(positions, positions + (ns - 1));
        Slices S = make_slices(method, ns, center_position, pos, z, n, resolution > 0 ? resolution : 100);
        int m = (int)S.center.size();
        for (int s = 0; s <= m; ++s) boundary[s] = S.boundary[s];
        int64_t k = 0;
        for (int s = 0; s < m; ++s) {
            center[s] = S.center[s];
            weight[s] = S.weight[s];
            count[s] = (int64_t)S.indices[s].size();
            for (int64_t i : S.indices[s]) order[k++] = i;
        }
        return OO_OK;
    } catch (OracleError &e) {
        return e.code;
    }
}

int32_t oo_pair_batches(const double *c1, int32_t ns1, const double *c2, int32_t ns2, int32_t *batch_of,
                        int32_t *pi, int32_t *pj, int32_t *order_i, int32_t *order_j) {
    std::vector<double> a(c1, c1 + ns1), b(c2, c2 + ns2);
    auto order = collision_order(a, b);
    for (size_t k = 0; k < order.size(); ++k) { order_i[k] = order[k].i; order_j[k] = order[k].j; }
    auto batches = pair_batches(a, b);
    int k = 0;
    for (size_t bi = 0; bi < batches.size(); ++bi)
        for (auto &p : batches[bi]) { batch_of[k] = (int)bi; pi[k] = p.i; pj[k] = p.j; ++k; }
    return (int32_t)batches.size();
}

int32_t oo_union_bounds(const double *src[4], int64_t ns, double center, const double *part[5], int64_t np,
                        double out[8], int32_t *valid) {
    Coords a, b;
    a.resize((size_t)ns);
    b.resize((size_t)np);
    for (int64_t k = 0; k < ns; ++k) { a.x[k] = src[0][k]; a.px[k] = src[1][k]; a.y[k] = src[2][k]; a.py[k] = src[3][k]; }
    for (int64_t k = 0; k < np; ++k) {
        b.x[k] = part[0][k]; b.px[k] = part[1][k]; b.y[k] = part[2][k]; b.py[k] = part[3][k]; b.z[k] = part[4][k];
    }
    try {
        UnionBounds u = union_bounds(a, center, std::vector<Coords>{b});
        *valid = u.valid;
        const double v[8] = {u.sb.xmin, u.sb.xmax, u.sb.ymin, u.sb.ymax, u.fb.xmin, u.fb.xmax, u.fb.ymin, u.fb.ymax};
        for (int k = 0; k < 8; ++k) out[k] = v[k];
    } catch (OracleError &e) {
        return e.code;
    }
    return OO_OK;
}

void *oo_create(const oo_options *opt) {
    Ctx *c = new Ctx();
    c->O = make_options(opt);
    return c;
}
void oo_destroy(void *ctx) { delete (Ctx *)ctx; }
int oo_collide(void *ctx, double *b1[6], int64_t n1, double *b2[6], int64_t n2, const oo_beam_params *p1,
               const oo_beam_params *p2, int32_t compute_luminosity, double *lum) {
    Ctx &C = *(Ctx *)ctx;
    try {
        double l = collide(C, b1, n1, b2, n2, *p1, *p2, compute_luminosity != 0);
        if (lum) *lum = l;
        C.err.clear();
        return OO_OK;
    } catch (OracleError &e) {
        C.err = e.what();
        return e.code;
    }
}
void oo_cache_stats(void *ctx, int64_t out[3]) {
    Ctx &C = *(Ctx *)ctx;
    out[0] = C.hits; out[1] = C.misses; out[2] = C.rebuilds;
}
int64_t oo_dropped(void *ctx) { return ((Ctx *)ctx)->dropped; }
int64_t oo_pair_trace(void *ctx, int32_t *pi, int32_t *pj, double *lum, int64_t cap) {
    Ctx &C = *(Ctx *)ctx;
    int64_t n = (int64_t)C.trace_lum.size();
    for (int64_t k = 0; k < n && k < cap; ++k) { pi[k] = C.trace_i[k]; pj[k] = C.trace_j[k]; lum[k] = C.trace_lum[k]; }
    return n;
}
const char *oo_last_error(void *ctx) { return ((Ctx *)ctx)->err.c_str(); }
// Arm / read the charge-grid capture (fixed_point_deposit must be on).  Returns 0 when a grid was captured.
void oo_capture_plane(void *ctx, int32_t i, int32_t j, int32_t dir, int32_t kind) {
    Capture &c = ((Ctx *)ctx)->cap;
    c = Capture();
    c.armed = true; c.i = i; c.j = j; c.dir = dir; c.kind = kind;
}
int32_t oo_captured_plane(void *ctx, int64_t *q, double mesh[4], int32_t *bits) {
    Capture &c = ((Ctx *)ctx)->cap;
    if (!c.armed || !c.taken) return OO_ERR_ARG;
    std::copy(c.q.begin(), c.q.end(), q);
    mesh[0] = c.grid.x0; mesh[1] = c.grid.y0; mesh[2] = c.grid.width; mesh[3] = c.grid.height;
    *bits = c.bits;
    c.armed = false;
    return OO_OK;
}

// linear6d.jl:110-121
void oo_linear6d(const double m[36], double *x, double *px, double *y, double *py, double *z, double *pz, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        double a = x[i], b = px[i], c = y[i], d = py[i], e = z[i], f = pz[i];
        x[i] = m[0] * a + m[1] * b + m[2] * c + m[3] * d + m[4] * e + m[5] * f;
        px[i] = m[6] * a + m[7] * b + m[8] * c + m[9] * d + m[10] * e + m[11] * f;
        y[i] = m[12] * a + m[13] * b + m[14] * c + m[15] * d + m[16] * e + m[17] * f;
        py[i] = m[18] * a + m[19] * b + m[20] * c + m[21] * d + m[22] * e + m[23] * f;
        z[i] = m[24] * a + m[25] * b + m[26] * c + m[27] * d + m[28] * e + m[29] * f;
        pz[i] = m[30] * a + m[31] * b + m[32] * c + m[33] * d + m[34] * e + m[35] * f;
    }
}
// linear6d.jl:233-280 with equal Twiss at both ends and no coupling/dispersion: per-plane rotation.
void oo_linear6d_matrix(const double beta[3], const double alpha[3], const double tune[3], double m[36]) {
    for (int k = 0; k < 36; ++k) m[k] = 0.0;
    for (int i = 0; i < 3; ++i) {
        double mu = 2.0 * 3.141592653589793 * tune[i];
        double s = std::sin(mu), c = std::cos(mu);
        double b1 = beta[i], b2 = beta[i], a1 = alpha[i], a2 = alpha[i];
        int r = 2 * i;
        m[r * 6 + r] = std::sqrt(b2 / b1) * (c + a1 * s);
        m[r * 6 + r + 1] = std::sqrt(b2 * b1) * s;
        m[(r + 1) * 6 + r] = (-(1.0 + a1 * a2) * s + (a1 - a2) * c) / std::sqrt(b1 * b2);
        m[(r + 1) * 6 + r + 1] = std::sqrt(b1 / b2) * (c - a2 * s);
    }
}


}  // extern "C"

// ---------------------------------------------------------------- line elements
// Each element restated per particle as the reference evaluates it, constructor constants included.
namespace {

// splitmix_uint64 (counter_rng.jl:284-291)
uint64_t splitmix_u64(uint64_t seed, uint64_t turn, uint64_t rng_id, uint64_t particle, uint64_t comp) {
    uint64_t x = seed;
    x ^= splitmix64(turn + 0x9e3779b97f4a7c15ULL);
    x ^= splitmix64(rng_id + 0xbf58476d1ce4e5b9ULL);
    x ^= splitmix64(particle + 0x94d049bb133111ebULL);
    x ^= splitmix64(comp + 0xD2B74407B1CE6E93ULL);
    return splitmix64(x);
}

// octopus_normal (counter_rng.jl:103-176): method-selected uniform pair, Box-Muller, odd component -> cos.
double octopus_normal(uint64_t seed, int method, uint64_t turn, uint64_t rng_id, uint64_t particle, uint64_t comp) {
    const uint64_t pair = (comp + 1) / 2;
    auto u64 = [&](uint64_t c) {
        return method == 1 ? counter_u64(seed, turn, rng_id, particle, c) : splitmix_u64(seed, turn, rng_id, particle, c);
    };
    const double u1 = uniform_open01(u64(2 * pair - 1));
    const double u2 = uniform_open01(u64(2 * pair));
    const double r = std::sqrt(-2.0 * std::log(u1));
    const double theta = 6.283185307179586476925286766559 * u2;
    return (comp & 1) ? r * std::cos(theta) : r * std::sin(theta);
}

typedef std::array<double, 6> Phase;

// CrabDispersion / MomentumDispersion forward (linear_maps.jl:125-132, 213-220) and inverse
// (chromaticity_kick.jl:151-167).
Phase zeta_fwd(const double *zt, Phase v) {
    const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3], z0 = v[4], pz0 = v[5];
    const double pz1 = pz0 + zt[1] * x0 - zt[0] * px0 + zt[3] * y0 - zt[2] * py0;
    return {x0 + zt[0] * z0, px0 + zt[1] * z0, y0 + zt[2] * z0, py0 + zt[3] * z0, z0, pz1};
}
Phase zeta_inv(const double *zt, Phase v) {
    const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3], z0 = v[4], pz0 = v[5];
    const double pz1 = pz0 - zt[1] * x0 + zt[0] * px0 - zt[3] * y0 + zt[2] * py0;
    return {x0 - zt[0] * z0, px0 - zt[1] * z0, y0 - zt[2] * z0, py0 - zt[3] * z0, z0, pz1};
}
Phase eta_fwd(const double *et, Phase v) {
    const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3], z0 = v[4], pz0 = v[5];
    const double z1 = z0 - et[1] * x0 + et[0] * px0 - et[3] * y0 + et[2] * py0;
    return {x0 + et[0] * pz0, px0 + et[1] * pz0, y0 + et[2] * pz0, py0 + et[3] * pz0, z1, pz0};
}
Phase eta_inv(const double *et, Phase v) {
    const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3], z0 = v[4], pz0 = v[5];
    const double z1 = z0 + et[1] * x0 - et[0] * px0 + et[3] * y0 - et[2] * py0;
    return {x0 - et[0] * pz0, px0 - et[1] * pz0, y0 - et[2] * pz0, py0 - et[3] * pz0, z1, pz0};
}
// XYCoupling (linear_maps.jl:353-372) and its mode-A inverse (chromaticity_kick.jl:179-186).
Phase xy_fwd(const double *r, int mode, Phase v) {
    if (mode == 0) return v;
    const double g = 1.0 / std::sqrt(1 + r[0] * r[3] - r[1] * r[2]);
    const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3];
    if (mode == 1)
        return {g * (x0 + r[3] * y0 - r[1] * py0), g * (px0 - r[2] * y0 + r[0] * py0),
                g * (-r[0] * x0 - r[1] * px0 + y0), g * (-r[2] * x0 - r[3] * px0 + py0), v[4], v[5]};
    return {g * (r[3] * x0 - r[1] * px0 + y0), g * (-r[2] * x0 + r[0] * px0 + py0), g * (x0 - r[0] * y0 - r[1] * py0),
            g * (px0 - r[2] * y0 - r[3] * py0), v[4], v[5]};
}
Phase xy_inv_a(const double *r, Phase v) {
    const double g = 1.0 / std::sqrt(1 + r[0] * r[3] - r[1] * r[2]);
    const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3];
    return {g * (x0 - r[3] * y0 + r[1] * py0), g * (px0 + r[2] * y0 - r[0] * py0), g * (r[0] * x0 + r[1] * px0 + y0),
            g * (r[2] * x0 + r[3] * px0 + py0), v[4], v[5]};
}

Phase track_element(const oo_element &e, Phase v, uint64_t seed, int method, uint64_t turn, uint64_t particle) {
    const double *p = e.p;
    switch (e.kind) {
        case 1: {  // Linear6D (linear6d.jl:110-121)
            Phase o;
            for (int r = 0; r < 6; ++r) {
                const double *m = p + 6 * r;
                o[r] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2] + m[3] * v[3] + m[4] * v[4] + m[5] * v[5];
            }
            return o;
        }
        case 2: {  // ThinCrabCavity (crab_cavity.jl:87-101, 128-144)
            const double kcc = 2.0 * 3.14159265358979323846 * p[0] / 299792458.0;
            double dpx = 0.0, dpy = 0.0, dpz = 0.0;
            for (int i = 1; i <= e.nharm; ++i) {
                const double ikcc = (double)i * kcc;
                const double th = ikcc * v[4] + p[17 + i - 1];
                const double s = std::sin(th), c = std::cos(th);
                const double sx = p[1 + i - 1], sy = p[9 + i - 1];
                dpx -= sx * s / ikcc;
                dpy -= sy * s / ikcc;
                dpz -= (sx * v[0] + sy * v[2]) * c;
            }
            return {v[0], v[1] + dpx, v[2], v[3] + dpy, v[4], v[5] + dpz};
        }
        case 3: {  // LorentzBoost (lorentz_boost.jl:128-143, constants :168-174)
            const double ca = std::cos(p[0]), sa = std::sin(p[0]), ta = sa / ca;
            const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3], z0 = v[4], pz0 = v[5];
            const double ps0 = std::sqrt((1.0 + pz0) * (1.0 + pz0) - px0 * px0 - py0 * py0);
            const double h0 = 1.0 + pz0 - ps0;
            const double py1 = py0 / ca;
            const double h1 = h0 / (ca * ca);
            const double px1 = px0 / ca - h1 * sa;
            const double pz1 = pz0 - px1 * sa;
            const double ps1 = 1.0 + pz1 - h1;
            const double ds = x0 * sa;
            return {x0 + z0 * ta + px1 / ps1 * ds, px1, y0 + py1 / ps1 * ds, py1, z0 / ca - h1 / ps1 * ds, pz1};
        }
        case 4: {  // RevLorentzBoost (lorentz_boost.jl:148-161)
            const double ca = std::cos(p[0]), sa = std::sin(p[0]);
            const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3], z0 = v[4], pz0 = v[5];
            const double ps0 = std::sqrt((1.0 + pz0) * (1.0 + pz0) - px0 * px0 - py0 * py0);
            const double h0 = 1.0 + pz0 - ps0;
            double x1 = x0 - z0 * sa;
            x1 = x1 / (1.0 + (px0 + h0 * sa) * sa / ps0);
            const double z1 = (z0 + h0 / ps0 * x1 * sa) * ca;
            const double y1 = y0 - py0 / ps0 * x1 * sa;
            return {x1, (px0 + h0 * sa) * ca, y1, py0 * ca, z1, pz0 + px0 * sa};
        }
        case 5: {  // ChromaticityKick (chromaticity_kick.jl:74-136)
            const double xix = p[0], xiy = p[1], betx = p[2], bety = p[3], alfx = p[4], alfy = p[5];
            const double gamx = (1.0 + alfx * alfx) / betx, gamy = (1.0 + alfy * alfy) / bety;
            const double *zt = p + 6, *et = p + 10, *r = p + 14;
            v = zeta_inv(zt, v);
            v = eta_inv(et, v);
            v = xy_inv_a(r, v);
            const double x0 = v[0], px0 = v[1], y0 = v[2], py0 = v[3];
            const double twopi = 6.283185307179586476925286766559005768394338;
            const double mux = twopi * xix * v[5];
            const double cx = std::cos(mux), sx = std::sin(mux);
            v[0] = x0 * (cx + alfx * sx) + px0 * betx * sx;
            v[1] = -x0 * sx * gamx + px0 * (cx - alfx * sx);
            const double muy = twopi * xiy * v[5];
            const double cy = std::cos(muy), sy = std::sin(muy);
            v[2] = y0 * (cy + alfy * sy) + py0 * bety * sy;
            v[3] = -y0 * sy * gamy + py0 * (cy - alfy * sy);
            const double jx = 0.5 * (gamx * x0 * x0 + 2 * alfx * x0 * px0 + betx * px0 * px0);
            const double jy = 0.5 * (gamy * y0 * y0 + 2 * alfy * y0 * py0 + bety * py0 * py0);
            v[4] += twopi * (xix * jx + xiy * jy);
            v = xy_fwd(r, 1, v);
            v = eta_fwd(et, v);
            return zeta_fwd(zt, v);
        }
        case 6: {  // LumpedRad (radiation.jl:83-131, 162-171, 196-279, 286-299)
            const bool enabled = p[9] >= 0.0 && p[10] >= 0.0 && p[11] >= 0.0;
            const bool damp = e.is_damping != 0 && e.mode != 2;
            const bool exc = e.is_excitation != 0 && enabled && e.mode != 1;
            if (!damp && !exc) return v;
            double damping[3], excitation[9];
            for (int i = 0; i < 3; ++i) {
                damping[i] = std::exp(-1.0 / p[i]);
                const double scale = std::sqrt(-std::expm1(-2.0 / p[i]));
                for (int k = 0; k < 3; ++k) {
                    const double sigma = p[9 + i];
                    double val;
                    if (sigma < 0.0) val = 0.0;
                    else {
                        const double amp = sigma * scale, slope = amp / p[3 + i];
                        val = k == 0 ? amp : k == 1 ? slope : -slope * p[6 + i];
                    }
                    excitation[3 * i + k] = val;
                }
            }
            double nrm[6] = {0, 0, 0, 0, 0, 0};
            if (exc)
                for (int c = 1; c <= 6; ++c) nrm[c - 1] = octopus_normal(seed, method, turn, e.rng_id, particle, c);
            const double *zt = p + 12, *et = p + 16, *r = p + 20;
            v = zeta_inv(zt, v);
            v = eta_inv(et, v);
            v = xy_inv_a(r, v);
            if (damp) {
                v[0] *= damping[0]; v[1] *= damping[0];
                v[2] *= damping[1]; v[3] *= damping[1];
                v[4] *= damping[2]; v[5] *= damping[2];
            }
            if (exc) {
                v[0] += excitation[0] * nrm[0];
                v[1] += excitation[1] * nrm[1] + excitation[2] * nrm[0];
                v[2] += excitation[3] * nrm[2];
                v[3] += excitation[4] * nrm[3] + excitation[5] * nrm[2];
                v[4] += excitation[6] * nrm[4];
                v[5] += excitation[7] * nrm[5] + excitation[8] * nrm[4];
            }
            v = xy_fwd(r, 1, v);
            v = eta_fwd(et, v);
            return zeta_fwd(zt, v);
        }
        case 7: return zeta_fwd(p, v);
        case 8: return eta_fwd(p, v);
        case 9: return xy_fwd(p, e.mode, v);
        default: return v;
    }
}

}  // namespace

extern "C" {

double oo_octopus_normal(uint64_t seed, int32_t rng_method, uint64_t turn, uint64_t rng_id, uint64_t particle,
                         uint64_t component) {
    return octopus_normal(seed, rng_method, turn, rng_id, particle, component);
}

// track!(rep, elems, turns, policy, ctx) (src/track/phase6d_track.jl:25-35): turn-major, particle i as id i + 1.
void oo_track_line(const oo_element *elems, int32_t n_elems, int64_t turn, int32_t turns, uint64_t seed,
                   int32_t rng_method, double *x, double *px, double *y, double *py, double *z, double *pz,
                   int64_t n) {
    for (int32_t t = 0; t < turns; ++t) {
        const uint64_t tt = (uint64_t)(turn + t);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            Phase v = {x[i], px[i], y[i], py[i], z[i], pz[i]};
            for (int32_t k = 0; k < n_elems; ++k) v = track_element(elems[k], v, seed, rng_method, tt, (uint64_t)(i + 1));
            x[i] = v[0]; px[i] = v[1]; y[i] = v[2]; py[i] = v[3]; z[i] = v[4]; pz[i] = v[5];
        }
    }
}


}  // extern "C"

// ---------------------------------------------------------------- the soft-Gaussian solver (gaussian.jl)
namespace {
std::string g_gauss_error;

const int REDUCTION_CHUNKS = 64;          // interface.jl:664
const int64_t PARALLEL_MOMENT_MIN = 4096; // interface.jl:609
const int64_t PARALLEL_KICK_MIN = 4096;   // interface.jl:610

// _chunk_bounds (slicing.jl:517-521), 0-based half-open
inline void chunk_bounds(int64_t n, int nchunks, int chunk1, int64_t &lo, int64_t &hi) {
    lo = ((int64_t)(chunk1 - 1) * n) / nchunks;
    hi = ((int64_t)chunk1 * n) / nchunks;
}

struct SoftMoments {
    double mx, mpx, my, mpy;                  // after ignore_centroid
    double a0, d0, bxx, bypy, qxx, qyy;       // StrongTransverseMoments
    double b0, bxpy, bypx, qxy;               // its coupled entries (zero when uncoupled)
    double sx, sy, spx, spy, covxpx, covypy;  // for the finiteness check
};
bool g_coupled = false;

// _slice_transverse_moments (slicing.jl:670-770), uncoupled
SoftMoments slice_moments(double *const b[6], const std::vector<int64_t> &idx, bool ignore_centroid, double min_sigma) {
    SoftMoments M{};
    const int64_t n = (int64_t)idx.size();
    const double floor2 = min_sigma * min_sigma;
    if (n == 0) {
        M.a0 = floor2; M.d0 = floor2;
        M.sx = min_sigma; M.sy = min_sigma;
        return M;
    }
    const int64_t f = idx[0];
    const double x0 = b[0][f], px0 = b[1][f], y0 = b[2][f], py0 = b[3][f];
    double s[14] = {};
    auto acc = [&](double *t, int64_t lo, int64_t hi) {
        for (int64_t p = lo; p < hi; ++p) {
            const int64_t i = idx[p];
            const double dx = b[0][i] - x0, dpx = b[1][i] - px0, dy = b[2][i] - y0, dpy = b[3][i] - py0;
            t[0] += dx; t[1] += dpx; t[2] += dy; t[3] += dpy;
            t[4] += dx * dx; t[5] += dpx * dpx; t[6] += dy * dy; t[7] += dpy * dpy;
            t[8] += dx * dpx; t[9] += dy * dpy;
            if (g_coupled) { t[10] += dx * dy; t[11] += dx * dpy; t[12] += dpx * dy; t[13] += dpx * dpy; }
        }
    };
    if (n < PARALLEL_MOMENT_MIN) {
        acc(s, 0, n);
    } else {
        for (int ch = 1; ch <= REDUCTION_CHUNKS; ++ch) {
            double t[14] = {};
            int64_t lo, hi;
            chunk_bounds(n, REDUCTION_CHUNKS, ch, lo, hi);
            acc(t, lo, hi);
            for (int q = 0; q < 14; ++q) s[q] += t[q];
        }
    }
    const double invn = 1.0 / (double)n;
    const double dmx = s[0] * invn, dmpx = s[1] * invn, dmy = s[2] * invn, dmpy = s[3] * invn;
    double mx = x0 + dmx, mpx = px0 + dmpx, my = y0 + dmy, mpy = py0 + dmpy;
    const double sx2 = std::fma(-dmx, dmx, s[4] * invn), spx2 = std::fma(-dmpx, dmpx, s[5] * invn);
    const double sy2 = std::fma(-dmy, dmy, s[6] * invn), spy2 = std::fma(-dmpy, dmpy, s[7] * invn);
    const double covxpx = std::fma(-dmx, dmpx, s[8] * invn), covypy = std::fma(-dmy, dmpy, s[9] * invn);
    const double varx = jmax(sx2, floor2), vary = jmax(sy2, floor2);
    M.a0 = varx; M.d0 = vary; M.bxx = covxpx; M.bypy = covypy;
    M.qxx = jmax(spx2, 0.0); M.qyy = jmax(spy2, 0.0);
    if (g_coupled) {
        M.b0 = std::fma(-dmx, dmy, s[10] * invn);
        M.bxpy = std::fma(-dmx, dmpy, s[11] * invn);
        M.bypx = std::fma(-dmpx, dmy, s[12] * invn);
        M.qxy = std::fma(-dmpx, dmpy, s[13] * invn);
    }
    if (ignore_centroid) { mx = 0; mpx = 0; my = 0; mpy = 0; }
    M.mx = mx; M.mpx = mpx; M.my = my; M.mpy = mpy;
    M.sx = std::sqrt(varx); M.sy = std::sqrt(vary);
    M.spx = std::sqrt(jmax(spx2, 0.0)); M.spy = std::sqrt(jmax(spy2, 0.0));
    M.covxpx = covxpx; M.covypy = covypy;
    return M;
}

// _gaussian_moments_finite (gaussian.jl:126-130)
bool moments_finite(const SoftMoments &m) {
    return std::isfinite(m.mx) && std::isfinite(m.mpx) && std::isfinite(m.my) && std::isfinite(m.mpy) &&
           std::isfinite(m.sx) && std::isfinite(m.sy) && std::isfinite(m.spx) && std::isfinite(m.spy) &&
           std::isfinite(m.covxpx) && std::isfinite(m.covypy);
}

// _apply_slice_kick_one! (gaussian.jl:152-185): Hirata paraxial drift (strong_beam.jl:559-577) or, without the
// longitudinal kick, the frozen-longitudinal paraxial drift (:517-531); _cp_covariance_kick (:619-632)
// The virtual drifts (strong_beam.jl:517-606); without the longitudinal kick the frozen paraxial drift.
double forward_drift(int kind, bool lk, double &x, double px, double &y, double py, double &z, double &pz, double zo) {
    if (!lk || kind == 0) {
        const double S = 0.5 * (z - zo);
        x += S * px;
        y += S * py;
        if (lk) pz -= 0.25 * (px * px + py * py);
        return S;
    }
    if (kind == 1) {
        const double S = 0.5 * (z - zo);
        const double phi = std::sqrt(1 - 0.5 * (px * px + py * py) / ((1 + pz) * (1 + pz))) - 1;
        x += S * px / (1 + pz);
        y += S * py / (1 + pz);
        z += 2 * S * phi;
        pz += (1 + pz) * phi;
        return S;
    }
    const double ps = std::sqrt((1 + pz) * (1 + pz) - px * px - py * py);
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
void reverse_drift(int kind, bool lk, double &x, double px, double &y, double py, double &z, double &pz, double zo) {
    const double S = 0.5 * (z - zo);
    if (!lk || kind == 0) {
        x -= S * px;
        y -= S * py;
        if (lk) pz += 0.25 * (px * px + py * py);
        return;
    }
    if (kind == 1) {
        const double psi = std::sqrt(1 + 0.5 * (px * px + py * py) / ((1 + pz) * (1 + pz))) - 1;
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

int g_drift_kind = 0;

double apply_one(double *const b[6], int64_t i, const SoftMoments &m, double center, double kbb, bool lk,
                 bool compute_lum) {
    double x = b[0][i], px = b[1][i], y = b[2][i], py = b[3][i], z = b[4][i], pz = b[5][i];
    const double S = forward_drift(g_drift_kind, lk, x, px, y, py, z, pz, center);
    const double xx = x - m.mx + m.mpx * S;
    const double yy = y - m.my + m.mpy * S;
    const double px0 = px, py0 = py, pz0 = pz;
    const double twopi_c = 6.283185307179586476925286766559005768394338;
    if (g_coupled) {  // _cp_covariance_kick, coupled (strong_beam.jl:634-682)
        const CovMoments cm{m.a0, m.b0, m.d0, m.bxx, m.bxpy, m.bypx, m.bypy, m.qxx, m.qxy, m.qyy};
        const double density = coupled_covariance_kick(cm, kbb, S, xx, yy, px, py, pz);
        if (lk) pz += 0.5 * ((px - px0) * m.mpx + (py - py0) * m.mpy);
        else pz = pz0;
        reverse_drift(g_drift_kind, lk, x, px, y, py, z, pz, center);
        b[0][i] = x; b[1][i] = px; b[2][i] = y; b[3][i] = py; b[4][i] = z; b[5][i] = pz;
        return compute_lum ? density * twopi_c : 0.0;
    }
    const double a = m.a0 - 2 * S * m.bxx + S * S * m.qxx;
    const double d = m.d0 - 2 * S * m.bypy + S * S * m.qyy;
    const double au = 2 * (m.bxx - S * m.qxx);
    const double du = 2 * (m.bypy - S * m.qyy);
    const double twopi = 6.283185307179586476925286766559005768394338;
    double density = 0.0;
    if (!(a <= 0 || d <= 0)) {
        const double sigx = std::sqrt(a), sigy = std::sqrt(d);
        double Kx, Ky, Hxx, Hyy;
        be::response(kbb, sigx, sigy, xx, yy, Kx, Ky, Hxx, Hyy);
        const double expterm = std::exp(-0.5 * (xx * xx / (sigx * sigx) + yy * yy / (sigy * sigy)));
        px += Kx * kbb;
        py += Ky * kbb;
        pz += 0.25 * (Hxx * au + Hyy * du);
        density = expterm / twopi / sigx / sigy;
    }
    if (lk) pz += 0.5 * ((px - px0) * m.mpx + (py - py0) * m.mpy);
    else pz = pz0;
    reverse_drift(g_drift_kind, lk, x, px, y, py, z, pz, center);
    b[0][i] = x; b[1][i] = px; b[2][i] = y; b[3][i] = py; b[4][i] = z; b[5][i] = pz;
    return compute_lum ? density * twopi : 0.0;
}

// _slice_slice_gaussian_kick! (gaussian.jl:59-108)
double slice_kick(double *const b[6], const std::vector<int64_t> &idx, const SoftMoments &m2, double center2,
                  double kbb_slice, double klum_slice, bool lk, bool compute_lum) {
    const int64_t n = (int64_t)idx.size();
    if (n == 0) return 0.0;
    const double twopi = 6.283185307179586476925286766559005768394338;
    if (n < PARALLEL_KICK_MIN) {
        double lum = 0.0;
        for (int64_t p = 0; p < n; ++p) lum += apply_one(b, idx[p], m2, center2, kbb_slice, lk, compute_lum);
        return lum / twopi * klum_slice;
    }
    double local[REDUCTION_CHUNKS];
#pragma omp parallel for schedule(static)
    for (int ch = 1; ch <= REDUCTION_CHUNKS; ++ch) {
        int64_t lo, hi;
        chunk_bounds(n, REDUCTION_CHUNKS, ch, lo, hi);
        double t = 0.0;
        for (int64_t p = lo; p < hi; ++p) t += apply_one(b, idx[p], m2, center2, kbb_slice, lk, compute_lum);
        local[ch - 1] = t;
    }
    double sum = 0.0;
    for (int ch = 0; ch < REDUCTION_CHUNKS; ++ch) sum += local[ch];
    return sum / twopi * klum_slice;
}

}  // namespace

extern "C" {

// collide!(::GaussianPoissonSolver, beam1, beam2, ::CPUThreadsBackend) (gaussian.jl:7-57); include_sigma_xy selects
// the coupled covariance; virtual_drift 0 :hirata, 1 :chromatic, 2 :exact; opt supplies the slicings, kbb / luminosity-scale overrides and
// longitudinal_kick.
int oo_gaussian_collide(const oo_options *opt, double min_sigma, int32_t gaussian_when_luminosity,
                        int32_t ignore_centroid1, int32_t ignore_centroid2, int32_t virtual_drift,
                        int32_t include_sigma_xy, double *b1[6], int64_t n1, double *b2[6], int64_t n2,
                        const oo_beam_params *p1, const oo_beam_params *p2, double *luminosity) {
    try {
        g_drift_kind = virtual_drift;
        g_coupled = include_sigma_xy != 0;
        std::vector<double> pos1, pos2;
        if (opt->slicing_method1 == 1 && opt->positions1) pos1.assign(opt->positions1, opt->positions1 + opt->nslices1 - 1);
        if (opt->slicing_method2 == 1 && opt->positions2) pos2.assign(opt->positions2, opt->positions2 + opt->nslices2 - 1);
        Slices s1 = make_slices(opt->slicing_method1, opt->nslices1, opt->center_position1, pos1, b1[4], n1,
                                opt->resolution1 > 0 ? opt->resolution1 : 100);
        Slices s2 = make_slices(opt->slicing_method2, opt->nslices2, opt->center_position2, pos2, b2[4], n2,
                                opt->resolution2 > 0 ? opt->resolution2 : 100);
        if (!opt->has_kbb1 && !(std::isfinite(p1->E0) && p1->E0 != 0))
            throw OracleError(OO_ERR_ARG, "beam1 E0 must be finite and nonzero when kbb1 is not specified");
        if (!opt->has_kbb2 && !(std::isfinite(p2->E0) && p2->E0 != 0))
            throw OracleError(OO_ERR_ARG, "beam2 E0 must be finite and nonzero when kbb2 is not specified");
        const double kbb1 = opt->has_kbb1 ? opt->kbb1 : p1->charge * p2->charge * p1->r0 * p2->npart * p1->mc2 / p1->E0;
        const double kbb2 = opt->has_kbb2 ? opt->kbb2 : p1->charge * p2->charge * p2->r0 * p1->npart * p2->mc2 / p2->E0;
        const double klum1 = opt->has_lum_scale ? opt->lum_scale : p1->npart * p2->npart / (double)n1;
        const double klum2 = opt->has_lum_scale ? opt->lum_scale : p1->npart * p2->npart / (double)n2;
        const bool lk = opt->longitudinal_kick != 0;
        const bool sample_beam1 = gaussian_when_luminosity == 1;
        double lum = 0.0;
        for (const OrderEntry &pr : collision_order(s1.center, s2.center)) {
            const int i = pr.i - 1, j = pr.j - 1;
            const SoftMoments m1 = slice_moments(b1, s1.indices[i], ignore_centroid1 != 0, min_sigma);
            const SoftMoments m2 = slice_moments(b2, s2.indices[j], ignore_centroid2 != 0, min_sigma);
            if (!moments_finite(m1))
                throw OracleError(OO_ERR_NONFINITE, "non-finite source coordinate (beam 1, slice " + std::to_string(i + 1) + ")");
            if (!moments_finite(m2))
                throw OracleError(OO_ERR_NONFINITE, "non-finite source coordinate (beam 2, slice " + std::to_string(j + 1) + ")");
            const double lum2 = slice_kick(b1, s1.indices[i], m2, s2.center[j], s2.weight[j] * kbb1, s2.weight[j] * klum1,
                                           lk, !sample_beam1);
            const double lum1 = slice_kick(b2, s2.indices[j], m1, s1.center[i], s1.weight[i] * kbb2, s1.weight[i] * klum2,
                                           lk, sample_beam1);
            lum += sample_beam1 ? lum1 : lum2;
        }
        if (luminosity) *luminosity = lum;
        return OO_OK;
    } catch (OracleError &e) {
        g_gauss_error = e.what();
        return e.code;
    }
}

const char *oo_gaussian_last_error(void) { return g_gauss_error.c_str(); }

// Pieces of the coupled kick's rotation term for the pins: the near-round series (strong_beam.jl:897-933) and
// the principal-axis response (:1061-1116), each with L / D; and the elliptic kick alone (:1139-1146 regime).
void oo_be_near_round_L(double kbb, double v, double eta, double x, double y, double out[5]) {
    be::near_round_series(kbb, v, eta, x, y, out[0], out[1], out[2], out[3], &out[4]);
}
void oo_be_principal_L(double kbb, double s1, double s2, double x, double y, double out[5]) {
    be::response_principal(kbb, s1, s2, x, y, out[0], out[1], out[2], out[3], &out[4]);
}
void oo_be_elliptic(double s1, double s2, double x, double y, double out[2]) {
    const double eta = (s1 * s1 - s2 * s2) / (s1 * s1 + s2 * s2);
    be::elliptic_kick(s1, s2, x, y, eta, out[0], out[1]);
}

}  // extern "C"
