// Internal types and device helpers shared by the libocto_b200 translation units.
//
// Precision contract of this FP64 build: the library is compiled with -fmad=false, so
// every scalar expression below rounds exactly like the reference's (Julia does not
// contract a*b+c).  Grid geometry and Green-cache decisions therefore come out bit-equal
// to the reference's on equal inputs, and fixed-point charge grids bit-equal to the CPU
// restatement's.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

namespace octo {

constexpr int kFoldLanes = 4096;           // slicing.jl:223 (_SLICE_FOLD_LANES)
constexpr int kMaxSlices = 64;
constexpr double kTemplateMarginCells = 1.5;  // interface.jl:674

struct Grid {
    double x0, y0, w, h;
};

// One directed interaction of a slice pair: `src` slice sources the field that kicks `fld`.
// Direction 1: source = beam 1 slice i, field = beam 2 slice j; direction 2 the reverse
// (pic_cpu.jl:364-377).
struct Task {
    int32_t dir, i, j;           // 1-based pair, direction
    int32_t src_beam, fld_beam;  // 0 / 1
    int32_t key;                 // Green-cache slot ((dir-1)*S1 + i-1)*S2 + j-1
    int32_t nodeL, nodeR;        // node-mesh ids (interaction_grid = :node), else -1
    int32_t pair;                // position in collision order
    int32_t front;               // wavefront index
    int32_t plane0, nplanes;     // field-solve planes of this task
    int64_t src_start, src_n, fld_start, fld_n;  // ranges in the slice-sorted arrays
    double c_src, c_fld, lb_fld, rb_fld;
    double sL, sR, sM, ks, hzi, zbias;
    // :node with luminosity: the kick of this task's field slice also reduces that slice's virtual positions
    // for its next pair in the schedule (collision-order index next_pair, whose direction-1 task is
    // next_task, drift next_sM); -1 when the slice has no later pair.
    int32_t next_pair, next_task;
    double next_sM;
    // interaction_grid = :source_slice: the row of this task's (direction, source slice) union box, and 1 when
    // this task is the source slice's first use (it computes the box)
    int32_t ub, ub_first;
};

// One beam's slice table, computed on the device by the slicing kernels and read back once per collide.
struct SliceInfo {
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

// The kick blocks of one wavefront: tasks t0 .. t0+nt-1, block map entries b0 .. b0+cap-1 of kchunk field
// particles each (a captured collide graph's map carries spare entries, task -1, for slices that grow).
struct FrontKick {
    int32_t t0, nt, b0, cap, kchunk, pad;
};

// :source_slice union box rows: partner z, partner x, partner y, source x, source y (min, max each)
constexpr int kUnionRow = 10;
constexpr int kUnionTrig = 1, kUnionBad = 2, kUnionSrcBad = 4;

// :node with luminosity: virtual-position extrema of each slice for its first pair of the collide.
struct FirstLum {
    int64_t start, count;
    double sM;
    int32_t beam, pair, task, pad;
};

// One deposit+solve plane.  kind: 0 = L (sL), 1 = R (sR), 2 = M (midpoint), 3 = Z (:node, sR on gL).
struct Plane {
    int32_t task, kind;
    int32_t geom;        // node mesh id, or -1 to use the task's planned source grid
    int32_t green;       // Green slot (resolved on the device for slice-pair tasks when -1)
    int32_t fixed_bits;  // fixed-point scale of the int64 charge grid
    int32_t count_dropped;
    int32_t src_beam;
    int32_t pad;
    // Precision form only: the plane is transformed as an exact int64 difference of charge grids,
    // q[self] - q[self + other_delta] (self_first = 1) or q[self + other_delta] - q[self] (self_first = 0),
    // so potentials that the kick subtracts are solved without FP32 cancellation.  other_delta = 0: none.
    int32_t other_delta, self_first;
    int64_t src_start, src_n;
    double s;            // drift of the deposit
};

// Planned geometry of a slice-pair task (written by the plan kernel).
struct TaskGeom {
    Grid sg, fg;
    int32_t green;       // Green slot used
    int32_t rebuild;     // 1 when this task (re)builds its Green slot in this front
};

struct CacheEntry {
    Grid sg, fg;
    int32_t valid;
    int32_t rebuilds;
    int64_t uses;
};

struct NodeMesh {
    Grid sg, fg;
    int32_t valid;
    int32_t pad;
};

// Luminosity of one slice pair (pic_cpu.jl:2700-2736).
struct LumJob {
    int32_t pair;
    int32_t bits1, bits2;
    int32_t pad;
    int64_t s1_start, s1_n, s2_start, s2_n;  // beam-1 slice i, beam-2 slice j
    double sM1, sM2;
};

struct LumGeom {
    double x0, y0, hx, hy;
    int32_t ok;
    int32_t pad;
};

// Cumulative device counters and the first error.
struct DevStatus {
    unsigned long long first_bad;   // (task index << 1) | 0 ; ~0ull when none
    int32_t code;
    int32_t role;
    long long hits, misses, rebuilds;
    long long dropped;
};

// ---------------------------------------------------------------- programmatic dependent launch
// Every kernel of the library begins with pdl_wait(); pdl_release().  A kernel launched with programmatic
// stream serialization (launch_pdl) may then begin launching while its predecessor in the stream drains:
// pdl_wait() blocks until the predecessor grid has completed and its memory operations are visible, and
// pdl_release() lets the successor's blocks launch once every block of this grid has executed it.  For a
// kernel launched normally both are no-ops.  Only work that touches no memory another kernel of the
// stream writes comes before the wait (twiddle tables uploaded at context creation, clearing shared
// memory); the wait precedes every other access and every early return, so a grid's completion still
// implies the completion of everything before it in the stream.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---------------------------------------------------------------- ordered doubles
// Monotone map double -> uint64 so integer atomicMin/atomicMax order doubles the way
// Julia's min/max do (-0.0 < +0.0).  NaN never enters: callers flag it separately.
__host__ __device__ inline unsigned long long ord_encode(double v) {
    unsigned long long u;
    memcpy(&u, &v, 8);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ inline double ord_decode(unsigned long long u) {
    u = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
    double v;
    memcpy(&v, &u, 8);
    return v;
}
constexpr unsigned long long kOrdMinInit = 0xffffffffffffffffull;  // decodes to NaN -> "+inf" sentinel
constexpr unsigned long long kOrdMaxInit = 0x0000000000000000ull;

// Julia semantics (base/math.jl): NaN-propagating, -0.0 < +0.0.
__host__ __device__ inline double jmin(double a, double b) {
    if (a != a || b != b) return a - b;
    if (a < b) return a;
    if (b < a) return b;
    return signbit(a) ? a : b;
}
__host__ __device__ inline double jmax(double a, double b) {
    if (a != a || b != b) return a - b;
    if (a > b) return a;
    if (b > a) return b;
    return signbit(a) ? b : a;
}
// Julia clamp(x, lo, hi) = ifelse(x > hi, hi, ifelse(x < lo, lo, x)).
__host__ __device__ inline double jclamp(double x, double lo, double hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}
__host__ __device__ inline float jclamp(float x, float lo, float hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}

// ---------------------------------------------------------------- particle real type
// R is the element type of the particle arrays and the arithmetic type of the particle kernels:
// double for the plain form, float for the precision form (FP32 particles, field planes and FFTs;
// FP64 Green function, slice statistics, grid geometry and luminosity sums; int64 charge grids).
// Every expression is written once for both, so the R = double instantiation is the plain form.
template <class R>
struct RealT;
template <>
struct RealT<double> {
    using C2 = double2;  // complex FFT element
    using FC = double2;  // field-plane vector: a cell is two of them, (phi, Ex), (Ey, 0)
    static constexpr int kCellVec = 2;
};
template <>
struct RealT<float> {
    using C2 = float2;
    using FC = float4;   // a cell is one 16-byte vector (phi, Ex, Ey, 0)
    static constexpr int kCellVec = 1;
};

__device__ __forceinline__ int floor_int(double u) { return __double2int_rd(u); }
__device__ __forceinline__ int floor_int(float u) { return __float2int_rd(u); }
__device__ __forceinline__ long long round_ll(double v) { return __double2ll_rn(v); }
__device__ __forceinline__ long long round_ll(float v) { return __float2ll_rn(v); }

// ---------------------------------------------------------------- weights
// CIC (pic_cpu.jl:2182-2197): 1-based base, zero weights outside [0, n-1] or non-finite.
template <class R>
__device__ __forceinline__ void cic_weights(R u, int n, int &base, R w[2]) {
    if (!(R(0) <= u && u <= (R)(n - 1))) {
        base = 1; w[0] = R(0); w[1] = R(0);
        return;
    }
    int b = floor_int(u) + 1;  // floor(u) + 1; u is in [0, n-1] here
    b = b < 1 ? 1 : (b > n - 1 ? n - 1 : b);
    base = b;
    R f = jclamp(u - (R)(base - 1), R(0), R(1));
    w[0] = R(1) - f;
    w[1] = f;
}

// TSC (pic_cpu.jl:2225-2252).
template <class R>
__device__ __forceinline__ void tsc_weights(R u, int n, int &base, R w[3]) {
    if (!(R(0) <= u && u <= (R)(n - 1))) {
        base = 1; w[0] = R(0); w[1] = R(0); w[2] = R(0);
        return;
    }
    const int ix = floor_int(u);  // floor(u); u is in [0, n-1] here
    R f = u - (R)ix;
    int b;
    if (f < R(0.5)) {
        R t = f * f;
        w[0] = R(0.125) + R(0.5) * (t - f);
        w[1] = R(0.75) - t;
        w[2] = R(0.125) + R(0.5) * (t + f);
        b = ix;
    } else {
        R fr = R(1) - f;
        R t = fr * fr;
        w[0] = R(0.125) + R(0.5) * (t + fr);
        w[1] = R(0.75) - t;
        w[2] = R(0.125) + R(0.5) * (t - fr);
        b = ix + 1;
    }
    b = b < 1 ? 1 : (b > n - 2 ? n - 2 : b);
    base = b;
}

// Fixed-point scale: taps are rounded to multiples of 2^-bits with
// bits = min(40, 62 - bitlength(nsrc)), so a whole slice fits one int64 cell.
__host__ __device__ inline int fixed_bits_for(int64_t n) {
    int bl = 0;
    uint64_t v = (uint64_t)(n < 1 ? 1 : n);
    while (v) { ++bl; v >>= 1; }
    int b = 62 - bl;
    return b > 40 ? 40 : b;
}
// The precision form's scale: bits = min(40, 30 - bitlength(nsrc)), so a whole slice fits one int32 cell of the
// block-private shared grids (its int64 plane grids and every integer sum stay exact).  An FP32 weight carries
// 24 significant bits, so the quanta lose nothing for slices of up to ~64 particles and at most 2^-(bits+1) of a
// particle's charge per tap beyond (2^-13 at 170,000 particles).
__host__ __device__ inline int fixed_bits_for32(int64_t n) {
    int bl = 0;
    uint64_t v = (uint64_t)(n < 1 ? 1 : n);
    while (v) { ++bl; v >>= 1; }
    int b = 30 - bl;
    return b > 40 ? 40 : b;
}

// ---------------------------------------------------------------- options (device copy)
struct DevOptions {
    int nx, ny, method, lum_method, lnx, lny;
    int green_type, green_cache, fourth, quadratic, node, longitudinal_kick;
    int dep_global, lum_global;  // charge / luminosity grid larger than shared memory: global atomics
    int gaussian, neutralize;    // GaussianPICPoissonSolver (Gaussian-subtracted hybrid)
    int dep_rotate;              // rotate each lane's deposit tap order (spatially ordered slices)
    int grid_extent;             // :slice_pair mesh extent: 0 :extrema, 1 :sigma (mean +- extent_k sd)
    int shared_grid;             // interaction_grid = :source_slice: one union-sized mesh per source slice
    double extent_k;             // grid_extent_sigma
    double min_ex, min_ey, quantize, min_ratio, growth;
    double margin;               // hybrid: Gaussian containment half-width in sigmas
    double coupling_tol;         // hybrid: |r_xy| above which the coupled subtraction runs (inf: never)
};

// Gaussian-subtracted hybrid state of one directed task (gaussian_pic.jl:604-705): the drifted reference
// Gaussian of the source slice at the two boundaries of the field slice ([0]: sL, [1]: sR).
struct HybridTask {
    int32_t mode;  // 0: plain PIC (degenerate moments); 1: uncoupled subtraction; 2: coupled (rotated) subtraction
    int32_t pad;
    double half_ns, mpx, mpy;
    double mux[2], muy[2], sigx[2], sigy[2], rx[2], ry[2];
    // coupled (gaussian_pic.jl:493-523): per boundary the drift s, sqrt of the drifted var x, the conditional
    // slope lambda = sigma_xy / sigma_x^2 and sigma sigc; the source's covariance for the rotated add-back
    double s[2], sa[2], lam[2], sigc[2];
    double cov[10];  // a0, b0, d0, bxx, bxpy, bypx, bypy, qxx, qxy, qyy (StrongTransverseMoments order)
};
// sums of dx, dpx, dy, dpy, dx^2, dpx^2, dy^2, dpy^2, dx dpx, dy dpy and, when the coupled subtraction can
// run (finite coupling_tol), the cross-plane dx dy, dx dpy, dy dpx, dpx dpy
constexpr int kMomentSums = 14;
constexpr int kMaxBoundBlocks = 128;  // blocks per slice of the bounds / moments passes

}  // namespace octo
