// PIC wavefront kernels.  Each launch covers every directed interaction (task), deposit plane
// or pair of one collision-time wavefront (slicing.jl:601-647), so the S1*S2 pairs of a turn run
// as 2S-1 batched launch sequences instead of one launch chain per pair.
#pragma once
#include "be_device.cuh"
#include "fft.cuh"
#include "rfft.cuh"
#include "geometry.cuh"
#include "octo_internal.cuh"

namespace octo {

struct SoA {
    void *c[6];  // x, px, y, py, z, pz (slice-sorted), element type R of the collide
};
template <class R>
__device__ __forceinline__ R *col(const SoA &S, int k) { return static_cast<R *>(S.c[k]); }

// Dynamic shared memory, typed per kernel (one declaration serves every template instantiation).
extern __shared__ __align__(16) unsigned char g_smem[];

struct Collide {           // device pointers for one collide (passed by value)
    DevOptions o;
    const Task *tasks;
    const Plane *planes;
    const LumJob *lumjobs;
    TaskGeom *geom;
    CacheEntry *cache;
    const NodeMesh *nodes;
    LumGeom *lumgeom;
    unsigned long long *bnd;   // [task][8]: src xmin,xmax,ymin,ymax ; fld xmin,xmax,ymin,ymax (ordered)
    unsigned long long *lumb;  // [pair][4] (ordered)
    int *nanflag;              // [task] bit0 source, bit1 field ; [ntasks + pair] bit2 luminosity
    DevStatus *status;
    double2 *ghat;             // Green spectra: slot * gstride
    long long gstride;         // (nx+1) * 2ny
    int scratch_green0;        // first scratch Green slot (green_cache = :none)
    long long *qgrid;          // int64 charge grids: plane-in-front * nx*ny
    void *spec;                // spectral scratch (RealT<R>::C2): plane-in-front * (nx+1)*ny
    void *fields;              // field planes (RealT<R>::FC): plane-in-front * kCellVec * nx*ny
    long long *lq;             // luminosity grids: (pair-in-front*2 + side) * (lnx+1)*(lny+1)
    double *lum_parts;         // [pair position]
    double *lum_partial;       // [pair-in-front][kLumSplit] overlap partial sums
    unsigned *lum_tick;        // [pair-in-front] blocks of k_lum_overlap done (reset by the last)
    const double2 *tw_x, *tw_y;  // FP64 twiddles for 2nx and 2ny (Green spectra)
    const void *twr_x, *twr_y;   // the same in RealT<R>::C2 (charge convolution)
    SoA beam[2];
    double klum;
    // Gaussian-subtracted hybrid (C.o.gaussian)
    HybridTask *hyb;             // [task]
    double *hmom;                // [task][kMaxBoundBlocks][kMomentSums] block partial moment sums
    unsigned long long *qtot;    // [plane-in-front] total fixed-point charge of the plane (two's complement)
    double *esum;                // grid_extent = :sigma: [task][kMaxBoundBlocks][8] block partial sums of the drifted
                                 // source (x, x^2, y, y^2 over both drifts) and field (x, x^2, y, y^2) offsets
    double *hprof;               // [plane-in-front][3][nx + ny] reference-Gaussian node profiles (gx | gy, then the
                                 // coupled subtraction's m1x | dgy and m2x | ddgy)
    double *hsum;                // [plane-in-front][2] profile sums
    // interaction_grid = :source_slice: per (direction, source slice) union box, row Task::ub of kUnionRow ordered
    // words (partner z min/max, partner collision-point x and y min/max, source x and y min/max over both extreme
    // drifts), its flags (kUnion*) and both beams' slice ranges slr[beam][slice] = (start, count)
    unsigned long long *ubox;
    int *uflag;
    const long long *slr;
};

// ------------------------------------------------------------------ bounds
__device__ __forceinline__ unsigned long long shfl_min_u64(unsigned long long v) {
    for (int o = 16; o; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long shfl_max_u64(unsigned long long v) {
    for (int o = 16; o; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Extremes of one slice of a pair in all three roles it plays: source of one direction
// (drifted to sL and sR, pic_cpu.jl:961-1003), field of the other (drifted to its collision
// point, pic_cpu.jl:1005-1035) and luminosity source (drifted to sM, pic_cpu.jl:1279-1287).
// Per-thread extrema use the native min/max (NaN is flagged separately; a +-0 tie cannot change any
// geometry built from them), encoded to ordered integers once per block for the atomics.
// grid: (blocks per side, 2 * pairs in front).
template <class R>
__global__ void __launch_bounds__(256) k_pair_bounds(Collide C, int task0) {
    pdl_wait();
    pdl_release();
    const int q = blockIdx.y >> 1, side = blockIdx.y & 1;
    const int t1 = task0 + 2 * q, t2 = t1 + 1;
    const Task &A = C.tasks[t1];  // dir 1: source beam-1 slice i, field beam-2 slice j
    const Task &B = C.tasks[t2];  // dir 2: source beam-2 slice j, field beam-1 slice i
    const Task &src_task = side == 0 ? A : B;  // this slice is the source of src_task
    const Task &fld_task = side == 0 ? B : A;  // ... and the field of fld_task
    const SoA S = C.beam[side];
    const long long st = src_task.src_start, n = src_task.src_n;
    const R sL = (R)src_task.sL, sR = (R)src_task.sR, sM = (R)src_task.sM, cf = (R)fld_task.c_src;
    R mn[6], mx[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) { mn[k] = R(INFINITY); mx[k] = R(-INFINITY); }
    bool nan_s = false, nan_f = false, nan_l = false;
    const R *X = col<R>(S, 0) + st, *PX = col<R>(S, 1) + st, *Y = col<R>(S, 2) + st, *PY = col<R>(S, 3) + st,
            *Z = col<R>(S, 4) + st;
    if (C.o.grid_extent) {
        // grid_extent = :sigma (pic_cpu.jl:954-1010): FP64 sums of the drifted offsets from the slice's first
        // particle -- source at both drifts (2n samples), field at its collision points -- as per-block partials
        // folded in block order by k_plan
        double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (n > 0) {
            const double sx0 = (double)(X[0] + PX[0] * sL), sy0 = (double)(Y[0] + PY[0] * sL);
            const R s0 = R(0.5) * (Z[0] - cf);
            const double fx0 = (double)(X[0] + s0 * PX[0]), fy0 = (double)(Y[0] + s0 * PY[0]);
            for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
                const R x = X[k], px = PX[k], y = Y[k], py = PY[k];
                const double dxl = (double)(x + px * sL) - sx0, dxr = (double)(x + px * sR) - sx0;
                const double dyl = (double)(y + py * sL) - sy0, dyr = (double)(y + py * sR) - sy0;
                e[0] += dxl + dxr; e[1] += dxl * dxl + dxr * dxr;
                e[2] += dyl + dyr; e[3] += dyl * dyl + dyr * dyr;
                const R s = R(0.5) * (Z[k] - cf);
                const double dx = (double)(x + s * px) - fx0, dy = (double)(y + s * py) - fy0;
                e[4] += dx; e[5] += dx * dx; e[6] += dy; e[7] += dy * dy;
            }
        }
        __shared__ double ered[8][8];
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            double v = e[q];
            for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (l == 0) ered[w][q] = v;
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            double v = 0.0;
            for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) v += ered[ww][threadIdx.x];
            // source sums belong to the task this slice sources, field sums to the task it is the field of
            const int task = threadIdx.x < 4 ? (side == 0 ? t1 : t2) : (side == 0 ? t2 : t1);
            C.esum[((long long)task * kMaxBoundBlocks + blockIdx.x) * 8 + threadIdx.x] = v;
        }
    }
#pragma unroll 4
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const R x = X[k], px = PX[k], y = Y[k], py = PY[k];
        const R lx = x + px * sM, ly = y + py * sM;
        nan_l |= (lx != lx) | (ly != ly);
        mn[4] = fmin(mn[4], lx); mx[4] = fmax(mx[4], lx);
        mn[5] = fmin(mn[5], ly); mx[5] = fmax(mx[5], ly);
        const R z = Z[k];
        const R a = x + px * sL, b = x + px * sR, c = y + py * sL, d = y + py * sR;
        const R s = R(0.5) * (z - cf);
        const R fx = x + s * px, fy = y + s * py;
        nan_s |= (a != a) | (b != b) | (c != c) | (d != d);
        nan_f |= (fx != fx) | (fy != fy);
        mn[0] = fmin(mn[0], fmin(a, b)); mx[0] = fmax(mx[0], fmax(a, b));
        mn[1] = fmin(mn[1], fmin(c, d)); mx[1] = fmax(mx[1], fmax(c, d));
        mn[2] = fmin(mn[2], fx); mx[2] = fmax(mx[2], fx);
        mn[3] = fmin(mn[3], fy); mx[3] = fmax(mx[3], fy);
    }
    __shared__ unsigned long long red[8][12];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        unsigned long long a = shfl_min_u64(mn[k] == R(INFINITY) ? kOrdMinInit : ord_encode((double)mn[k]));
        unsigned long long b = shfl_max_u64(mx[k] == R(-INFINITY) ? kOrdMaxInit : ord_encode((double)mx[k]));
        if (lane == 0) { red[warp][2 * k] = a; red[warp][2 * k + 1] = b; }
    }
    int any_s = __syncthreads_or(nan_s), any_f = __syncthreads_or(nan_f), any_l = __syncthreads_or(nan_l);
    if (threadIdx.x < 12) {
        int k = threadIdx.x;
        unsigned long long r = red[0][k];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = (k & 1) ? max(r, red[w][k]) : min(r, red[w][k]);
        int quantity = k >> 1;  // 0 src x, 1 src y, 2 fld x, 3 fld y, 4 lum x, 5 lum y
        unsigned long long *dst;
        if (quantity < 2) dst = C.bnd + (long long)(side == 0 ? t1 : t2) * 8 + quantity * 2 + (k & 1);
        else if (quantity < 4) dst = C.bnd + (long long)(side == 0 ? t2 : t1) * 8 + 4 + (quantity - 2) * 2 + (k & 1);
        else dst = C.lumb + (long long)A.pair * 4 + (quantity - 4) * 2 + (k & 1);
        if (k & 1) atomicMax(dst, r); else atomicMin(dst, r);
    }
    if (threadIdx.x == 0) {
        if (any_s) atomicOr(&C.nanflag[side == 0 ? t1 : t2], 1);
        if (any_f) atomicOr(&C.nanflag[side == 0 ? t2 : t1], 2);
        if (any_l) atomicOr(&C.nanflag[side == 0 ? t1 : t2], 4);
    }
}

// ------------------------------------------------------------------ :source_slice union boxes
// Block-wide min/max of nq quantities into dst[2q] (min) and dst[2q + 1] (max), as ordered words.
template <class R>
__device__ __forceinline__ void reduce_ordered(const R *mn, const R *mx, int nq, unsigned long long *dst) {
    __shared__ unsigned long long red[8][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = 0; q < nq; ++q) {
        unsigned long long a = shfl_min_u64(mn[q] == R(INFINITY) ? kOrdMinInit : ord_encode((double)mn[q]));
        unsigned long long b = shfl_max_u64(mx[q] == R(-INFINITY) ? kOrdMaxInit : ord_encode((double)mx[q]));
        if (lane == 0) { red[warp][2 * q] = a; red[warp][2 * q + 1] = b; }
    }
    __syncthreads();
    if (threadIdx.x < 2 * nq) {
        const int k = threadIdx.x;
        unsigned long long r = red[0][k];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = (k & 1) ? max(r, red[w][k]) : min(r, red[w][k]);
        if (k & 1) atomicMax(dst + k, r); else atomicMin(dst + k, r);
    }
}

// _pic_union_bounds, states form (pic_cpu.jl:665-692), for the tasks of a front that are their source slice's
// first use: every sliced particle of the partner (field) beam, as the pair finds it, drifted to its collision
// point with the source slice, x + 0.5*(z - c_src)*px.  Flags: kUnionTrig when a drifted position is not finite
// or z is NaN (the reference's trigger), kUnionBad when an input coordinate is not finite (its search for the
// offending slice); both set is its error.  grid: (blocks per slice, kMaxSlices, tasks of the front).
template <class R>
__global__ void __launch_bounds__(256) k_union_partner(Collide C, int task0) {
    pdl_wait();
    pdl_release();
    const Task &T = C.tasks[task0 + blockIdx.z];
    if (!T.ub_first) return;
    const int fb = T.fld_beam, sl = blockIdx.y;
    const long long *r = C.slr + ((long long)fb * kMaxSlices + sl) * 2;
    const long long st = r[0], n = r[1];
    if ((long long)blockIdx.x * blockDim.x >= n) return;  // block-uniform
    const SoA S = C.beam[fb];
    const R *X = col<R>(S, 0) + st, *PX = col<R>(S, 1) + st, *Y = col<R>(S, 2) + st, *PY = col<R>(S, 3) + st,
            *Z = col<R>(S, 4) + st;
    const R c = (R)T.c_src;
    R mn[3] = {R(INFINITY), R(INFINITY), R(INFINITY)}, mx[3] = {R(-INFINITY), R(-INFINITY), R(-INFINITY)};
    bool trig = false, bad = false;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const R x = X[k], px = PX[k], y = Y[k], py = PY[k], z = Z[k];
        const R s = R(0.5) * (z - c);
        const R xv = x + s * px, yv = y + s * py;
        trig |= (z != z) | !isfinite(xv) | !isfinite(yv);
        bad |= !isfinite(x) | !isfinite(px) | !isfinite(y) | !isfinite(py) | !isfinite(z);
        mn[0] = fmin(mn[0], z); mx[0] = fmax(mx[0], z);
        mn[1] = fmin(mn[1], xv); mx[1] = fmax(mx[1], xv);
        mn[2] = fmin(mn[2], yv); mx[2] = fmax(mx[2], yv);
    }
    const int any_t = __syncthreads_or(trig), any_b = __syncthreads_or(bad);
    reduce_ordered<R>(mn, mx, 3, C.ubox + (long long)T.ub * kUnionRow);
    if (threadIdx.x == 0 && (any_t || any_b)) atomicOr(&C.uflag[T.ub], (any_t ? kUnionTrig : 0) | (any_b ? kUnionBad : 0));
}

// _pic_union_bounds_tail (pic_cpu.jl:697-712): the source slice at the two extreme drifts of the partner's z
// range, sA = 0.5*(c - zmax) and sB = 0.5*(c - zmin) (the drift is affine in s, so they bound every other).
// No box -- per-pair sizing -- when the partner's zmin is not finite.  grid: (blocks, tasks of the front).
template <class R>
__global__ void __launch_bounds__(256) k_union_source(Collide C, int task0) {
    pdl_wait();
    pdl_release();
    const Task &T = C.tasks[task0 + blockIdx.y];
    if (!T.ub_first) return;
    unsigned long long *row = C.ubox + (long long)T.ub * kUnionRow;
    const double zmin = ord_decode(row[0]), zmax = ord_decode(row[1]);
    if (!isfinite(zmin) || (C.uflag[T.ub] & (kUnionTrig | kUnionBad)) == (kUnionTrig | kUnionBad)) return;
    const SoA S = C.beam[T.src_beam];
    const long long st = T.src_start, n = T.src_n;
    const R *X = col<R>(S, 0) + st, *PX = col<R>(S, 1) + st, *Y = col<R>(S, 2) + st, *PY = col<R>(S, 3) + st;
    const R c = (R)T.c_src;
    const R sA = R(0.5) * (c - (R)zmax), sB = R(0.5) * (c - (R)zmin);
    R mn[2] = {R(INFINITY), R(INFINITY)}, mx[2] = {R(-INFINITY), R(-INFINITY)};
    bool nan = false;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const R x = X[k], px = PX[k], y = Y[k], py = PY[k];
        const R xa = x + px * sA, xb = x + px * sB, ya = y + py * sA, yb = y + py * sB;
        nan |= !isfinite(xa) | !isfinite(xb) | !isfinite(ya) | !isfinite(yb);
        mn[0] = fmin(mn[0], fmin(xa, xb)); mx[0] = fmax(mx[0], fmax(xa, xb));
        mn[1] = fmin(mn[1], fmin(ya, yb)); mx[1] = fmax(mx[1], fmax(ya, yb));
    }
    const int any = __syncthreads_or(nan);
    reduce_ordered<R>(mn, mx, 2, row + 6);
    if (threadIdx.x == 0 && any) atomicOr(&C.uflag[T.ub], kUnionSrcBad);
}

// Block-wide reduction of a thread's virtual-position extrema into a pair's luminosity box (ordered
// atomics) and the non-finite flag of its direction-1 task.
template <class R>
__device__ __forceinline__ void reduce_lum_box(Collide &C, R mnx, R mxx, R mny, R mxy, bool nan, int pair, int task) {
    __shared__ unsigned long long red[8][4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long a = shfl_min_u64(mnx == R(INFINITY) ? kOrdMinInit : ord_encode((double)mnx));
    unsigned long long b = shfl_max_u64(mxx == R(-INFINITY) ? kOrdMaxInit : ord_encode((double)mxx));
    unsigned long long c = shfl_min_u64(mny == R(INFINITY) ? kOrdMinInit : ord_encode((double)mny));
    unsigned long long d = shfl_max_u64(mxy == R(-INFINITY) ? kOrdMaxInit : ord_encode((double)mxy));
    if (lane == 0) { red[warp][0] = a; red[warp][1] = b; red[warp][2] = c; red[warp][3] = d; }
    const int any_nan = __syncthreads_or(nan);
    if (threadIdx.x < 4) {
        unsigned long long r = red[0][threadIdx.x];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = (threadIdx.x & 1) ? max(r, red[w][threadIdx.x]) : min(r, red[w][threadIdx.x]);
        unsigned long long *dst = C.lumb + (long long)pair * 4 + threadIdx.x;
        if (threadIdx.x & 1) atomicMax(dst, r); else atomicMin(dst, r);
    }
    if (threadIdx.x == 0 && any_nan) atomicOr(&C.nanflag[task], 4);
}

// :node with luminosity, turn start: every slice's virtual positions at the drift of its first pair
// (pic_cpu.jl:1279-1287, 2706-2712); later pairs get theirs from the kick of the slice's previous pair.
// grid: (blocks per slice, slices of both beams).
template <class R>
__global__ void __launch_bounds__(256) k_first_lum_bounds(Collide C, const FirstLum *first) {
    pdl_wait();
    pdl_release();
    const FirstLum F = first[blockIdx.y];
    const SoA S = C.beam[F.beam];
    const R *X = col<R>(S, 0) + F.start, *PX = col<R>(S, 1) + F.start, *Y = col<R>(S, 2) + F.start,
            *PY = col<R>(S, 3) + F.start;
    const R s = (R)F.sM;
    R mnx = R(INFINITY), mxx = R(-INFINITY), mny = R(INFINITY), mxy = R(-INFINITY);
    bool nan = false;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < F.count; k += (long long)gridDim.x * blockDim.x) {
        const R vx = X[k] + PX[k] * s, vy = Y[k] + PY[k] * s;
        nan |= (vx != vx) | (vy != vy);
        mnx = fmin(mnx, vx); mxx = fmax(mxx, vx);
        mny = fmin(mny, vy); mxy = fmax(mxy, vy);
    }
    reduce_lum_box(C, mnx, mxx, mny, mxy, nan, F.pair, F.task);
}

// Hybrid: transverse moment sums of each task's source slice relative to its first particle
// (gaussian_pic.jl:432-486), as per-block partials folded in block order by k_plan.  grid: (blocks per
// side, 2 * pairs in front), the mapping of k_pair_bounds.
// The sums are FP64 in both forms (the precision form's FP32 coordinates are widened exactly).
template <class R>
__global__ void __launch_bounds__(256) k_hyb_moments(Collide C, int task0) {
    pdl_wait();
    pdl_release();
    const int q = blockIdx.y >> 1, side = blockIdx.y & 1;
    const int t = task0 + 2 * q + side;  // side 0: direction-1 task (source beam 1), side 1: direction 2
    const Task &T = C.tasks[t];
    const SoA S = C.beam[T.src_beam];
    const long long st = T.src_start, n = T.src_n;
    const R *X = col<R>(S, 0) + st, *PX = col<R>(S, 1) + st, *Y = col<R>(S, 2) + st, *PY = col<R>(S, 3) + st;
    double a[kMomentSums];
#pragma unroll
    for (int k = 0; k < kMomentSums; ++k) a[k] = 0.0;
    const bool gate = isfinite(C.o.coupling_tol);  // the cross-plane sums only when the coupled path can read them
    if (n > 0) {
        const double x0 = X[0], px0 = PX[0], y0 = Y[0], py0 = PY[0];
        for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
            const double dx = (double)X[k] - x0, dpx = (double)PX[k] - px0, dy = (double)Y[k] - y0, dpy = (double)PY[k] - py0;
            a[0] += dx; a[1] += dpx; a[2] += dy; a[3] += dpy;
            a[4] += dx * dx; a[5] += dpx * dpx; a[6] += dy * dy; a[7] += dpy * dpy;
            a[8] += dx * dpx; a[9] += dy * dpy;
            if (gate) { a[10] += dx * dy; a[11] += dx * dpy; a[12] += dy * dpx; a[13] += dpx * dpy; }
        }
    }
    __shared__ double red[8][kMomentSums];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < kMomentSums; ++k) {
        double v = a[k];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < kMomentSums) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
        C.hmom[((long long)t * kMaxBoundBlocks + blockIdx.x) * kMomentSums + threadIdx.x] = v;
    }
}

// Fold the per-block moment partials of each task, in block order, into slot 0 (one warp per task: lane k
// sums quantity k over the blocks).
__global__ void k_hyb_fold(Collide C, int task0, int ntasks, int nblk) {
    pdl_wait();
    pdl_release();
    const int tl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (tl >= ntasks || lane >= kMomentSums) return;
    double *m = C.hmom + (long long)(task0 + tl) * kMaxBoundBlocks * kMomentSums;
    double v = 0.0;
    for (int b = 0; b < nblk; ++b) v += m[b * kMomentSums + lane];
    m[lane] = v;
}

// Drifted reference Gaussian of the source at drift s (gaussian_pic.jl:496-540, uncoupled).
__device__ __forceinline__ void hyb_boundary(const double m[10], double s, HybridTask &H, int side) {
    // m: mx, mpx, varx, cxpx, varpx, my, mpy, vary, cypy, varpy
    H.mux[side] = m[0] + m[1] * s;
    H.muy[side] = m[5] + m[6] * s;
    const double varx = m[2] + 2.0 * s * m[3] + s * s * m[4];
    const double vary = m[7] + 2.0 * s * m[8] + s * s * m[9];
    H.sigx[side] = sqrt(jmax(varx, 0.0));
    H.sigy[side] = sqrt(jmax(vary, 0.0));
    H.rx[side] = 2.0 * (m[3] + s * m[4]);
    H.ry[side] = 2.0 * (m[8] + s * m[9]);
}

// Coupled boundary (gaussian_pic.jl:449-523): the covariance transported to drift s (S = -s in the field-
// particle convention), its correlation, whether it is resolved (full rank to sqrt(eps)), the conditional slope
// and sigma.  cv: a0, b0, d0, bxx, bxpy, bypx, bypy, qxx, qxy, qyy.
__device__ __forceinline__ void hyb_coupled_boundary(const double cv[10], double s, HybridTask &H, int side, double &rxy,
                                                     bool &resolved) {
    const double S = -s;
    const double a = cv[0] - 2 * S * cv[3] + S * S * cv[7];
    const double b = cv[1] - S * (cv[4] + cv[5]) + S * S * cv[8];
    const double d = cv[2] - 2 * S * cv[6] + S * S * cv[9];
    rxy = (a <= 0 || d <= 0) ? 0.0 : (b / sqrt(a)) / sqrt(d);
    bool ok = isfinite(a) && isfinite(b) && isfinite(d) && a > 0 && d > 0;
    if (ok) {
        const double rho = (b / sqrt(a)) / sqrt(d);
        ok = isfinite(rho) && fma(-rho, rho, 1.0) > 1.4901161193847656e-08;  // sqrt(eps(Float64))
    }
    resolved = ok;
    H.sa[side] = sqrt(a);
    H.lam[side] = ok ? b / a : 0.0;
    const double rcv = ok ? jmax(fma(-rxy, rxy, 1.0), 0.0) : 0.0;
    H.sigc[side] = ok ? sqrt(d * rcv) : 0.0;
}

__device__ inline void record_error(DevStatus *st, int task, int code, int role) {
    unsigned long long key = ((unsigned long long)task << 16) | ((unsigned long long)code << 8) | (unsigned)role;
    atomicMin(&st->first_bad, key);
}

// Grid geometry and Green-cache decision per task (pic_cpu.jl:954-1064, 1729-1821).  Hybrid: the source
// moments (folded by k_hyb_fold), the reference Gaussians at both boundaries, the plain-PIC fallback test
// and the margin box around the Gaussians joined to the source extent (gaussian_pic.jl:604-660).
// R: the element type of the beams (the hybrid reads the source slice's first particle, the origin of its
// moment sums).
// grid_extent = :sigma turns a (lo, hi) extent into mean +- k sd from the sums of offsets from `origin`
// (pic_cpu.jl:1551-1593): degenerate spreads and n < 2 keep the extrema.
__device__ __forceinline__ void axis_extent_sigma(double &lo, double &hi, double origin, double ds, double ds2,
                                                  long long n, double k) {
    if (n < 2) return;
    const double invn = 1.0 / (double)n;
    const double mean_offset = ds * invn;
    const double m = origin + mean_offset;
    const double var = jmax(fma(-mean_offset, mean_offset, ds2 * invn), 0.0);  // muladd of slicing.jl:667-668
    const double half = k * sqrt(var);
    if (!(half > 0)) return;
    lo = m - half;
    hi = m + half;
}

template <class R>
__global__ void k_plan(Collide C, int task0, int ntasks, int slot_scratch0, int ext_blocks) {
    pdl_wait();
    pdl_release();
    int tl = blockIdx.x * blockDim.x + threadIdx.x;
    if (tl >= ntasks) return;
    int t = task0 + tl;
    const Task &T = C.tasks[t];
    TaskGeom &G = C.geom[t];
    G.rebuild = 0;
    G.green = -1;
    const unsigned long long *b = C.bnd + (long long)t * 8;
    double sxmin = ord_decode(b[0]), sxmax = ord_decode(b[1]), symin = ord_decode(b[2]), symax = ord_decode(b[3]);
    double fxmin = ord_decode(b[4]), fxmax = ord_decode(b[5]), fymin = ord_decode(b[6]), fymax = ord_decode(b[7]);
    if (C.o.shared_grid) {
        // :source_slice: a non-finite coordinate met by the union box comes first in the pair (pic_cpu.jl:368-371,
        // before either interaction): recorded on the pair's direction-1 task with role 0
        const int uf = C.uflag[T.ub];
        if ((uf & (kUnionTrig | kUnionBad)) == (kUnionTrig | kUnionBad) || (uf & kUnionSrcBad)) {
            record_error(C.status, T.dir == 1 ? t : t - 1, 1, 0);
            return;
        }
    }
    int nf = C.nanflag[t];
    if ((nf & 1) || !(isfinite(sxmin) && isfinite(sxmax) && isfinite(symin) && isfinite(symax))) {
        record_error(C.status, t, 1, 1);
        return;
    }
    if ((nf & 2) || !(isfinite(fxmin) && isfinite(fxmax) && isfinite(fymin) && isfinite(fymax))) {
        record_error(C.status, t, 1, 2);
        return;
    }
    if (C.o.grid_extent) {
        double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const double *es = C.esum + (long long)t * kMaxBoundBlocks * 8;
        for (int b = 0; b < ext_blocks; ++b)
            for (int q = 0; q < 8; ++q) e[q] += es[b * 8 + q];
        const SoA Ss = C.beam[T.src_beam], Sf = C.beam[T.fld_beam];
        const long long ss = T.src_start, fs = T.fld_start;
        const R sL = (R)T.sL;
        const double sx0 = (double)(col<R>(Ss, 0)[ss] + col<R>(Ss, 1)[ss] * sL);
        const double sy0 = (double)(col<R>(Ss, 2)[ss] + col<R>(Ss, 3)[ss] * sL);
        const R s0 = R(0.5) * (col<R>(Sf, 4)[fs] - (R)T.c_src);
        const double fx0 = (double)(col<R>(Sf, 0)[fs] + s0 * col<R>(Sf, 1)[fs]);
        const double fy0 = (double)(col<R>(Sf, 2)[fs] + s0 * col<R>(Sf, 3)[fs]);
        const double k = C.o.extent_k;
        axis_extent_sigma(sxmin, sxmax, sx0, e[0], e[1], 2 * T.src_n, k);
        axis_extent_sigma(symin, symax, sy0, e[2], e[3], 2 * T.src_n, k);
        axis_extent_sigma(fxmin, fxmax, fx0, e[4], e[5], T.fld_n, k);
        axis_extent_sigma(fymin, fymax, fy0, e[6], e[7], T.fld_n, k);
        if (!(isfinite(sxmin) && isfinite(sxmax) && isfinite(symin) && isfinite(symax))) {
            record_error(C.status, t, 1, 1);
            return;
        }
        if (!(isfinite(fxmin) && isfinite(fxmax) && isfinite(fymin) && isfinite(fymax))) {
            record_error(C.status, t, 1, 2);
            return;
        }
    }
    if (C.o.gaussian) {
        HybridTask &H = C.hyb[t];
        H.mode = 0;
        double sum[kMomentSums];  // folded by k_hyb_fold
        for (int k = 0; k < kMomentSums; ++k) sum[k] = C.hmom[(long long)t * kMaxBoundBlocks * kMomentSums + k];
        const SoA S = C.beam[T.src_beam];
        const long long st = T.src_start, n = T.src_n;
        const double x0 = (double)col<R>(S, 0)[st], px0 = (double)col<R>(S, 1)[st], y0 = (double)col<R>(S, 2)[st],
                     py0 = (double)col<R>(S, 3)[st];
        const double invn = 1.0 / (double)n;
        const double dmx = sum[0] * invn, dmpx = sum[1] * invn, dmy = sum[2] * invn, dmpy = sum[3] * invn;
        double m[10];
        m[0] = x0 + dmx; m[1] = px0 + dmpx; m[5] = y0 + dmy; m[6] = py0 + dmpy;
        // muladd(-a, b, c) of slicing.jl:664-668, fused on FMA hosts
        m[2] = jmax(fma(-dmx, dmx, sum[4] * invn), 0.0);
        m[7] = jmax(fma(-dmy, dmy, sum[6] * invn), 0.0);
        m[3] = fma(-dmx, dmpx, sum[8] * invn);
        m[4] = jmax(fma(-dmpx, dmpx, sum[5] * invn), 0.0);
        m[8] = fma(-dmy, dmpy, sum[9] * invn);
        m[9] = jmax(fma(-dmpy, dmpy, sum[7] * invn), 0.0);
        hyb_boundary(m, T.sL, H, 0);
        hyb_boundary(m, T.sR, H, 1);
        H.half_ns = 0.5 * (double)n;
        H.mpx = m[1];
        H.mpy = m[6];
        bool ok = n >= 2;
        for (int sd = 0; sd < 2; ++sd)
            ok = ok && isfinite(H.sigx[sd]) && isfinite(H.sigy[sd]) && H.sigx[sd] > 0 && H.sigy[sd] > 0;
        // the full covariance (gaussian_pic.jl:374-447; cross terms only under a finite coupling_tol) and the
        // control-variate mode (gaussian_pic.jl:525-536): 0 plain PIC, 1 uncoupled, 2 coupled
        const bool gate = isfinite(C.o.coupling_tol);
        double *cv = H.cov;
        cv[0] = m[2]; cv[2] = m[7]; cv[3] = m[3]; cv[6] = m[8]; cv[7] = m[4]; cv[9] = m[9];
        cv[1] = gate ? fma(-dmx, dmy, sum[10] * invn) : 0.0;
        cv[4] = gate ? fma(-dmx, dmpy, sum[11] * invn) : 0.0;
        cv[5] = gate ? fma(-dmy, dmpx, sum[12] * invn) : 0.0;
        cv[8] = gate ? fma(-dmpx, dmpy, sum[13] * invn) : 0.0;
        bool resolved[2] = {false, false};
        double rxy[2] = {0.0, 0.0};
        for (int sd = 0; sd < 2; ++sd) {
            const double sb = sd ? T.sR : T.sL;
            H.s[sd] = sb;
            H.sa[sd] = H.lam[sd] = H.sigc[sd] = 0.0;
            if (!gate) continue;
            hyb_coupled_boundary(cv, sb, H, sd, rxy[sd], resolved[sd]);
        }
        int mode = ok ? 1 : 0;
        if (ok && gate && jmax(fabs(rxy[0]), fabs(rxy[1])) > C.o.coupling_tol) mode = resolved[0] && resolved[1] ? 2 : 0;
        H.mode = mode;
        ok = mode != 0;
        if (ok && C.o.margin > 0) {
            const double mg = C.o.margin;
            sxmin = jmin(sxmin, jmin(H.mux[0] - mg * H.sigx[0], H.mux[1] - mg * H.sigx[1]));
            sxmax = jmax(sxmax, jmax(H.mux[0] + mg * H.sigx[0], H.mux[1] + mg * H.sigx[1]));
            symin = jmin(symin, jmin(H.muy[0] - mg * H.sigy[0], H.muy[1] - mg * H.sigy[1]));
            symax = jmax(symax, jmax(H.muy[0] + mg * H.sigy[0], H.muy[1] + mg * H.sigy[1]));
            if (!(isfinite(sxmin) && isfinite(sxmax) && isfinite(symin) && isfinite(symax))) {
                record_error(C.status, t, 1, 1);
                return;
            }
        }
    }
    Grid sg, fg;
    // :source_slice: the mesh is sized from the source slice's union box (pic_cpu.jl:1036-1048), while the cache's
    // coverage test below keeps this pair's own bounds.
    double gs[4] = {sxmin, sxmax, symin, symax}, gf[4] = {fxmin, fxmax, fymin, fymax};
    if (C.o.shared_grid) {
        const unsigned long long *row = C.ubox + (long long)T.ub * kUnionRow;
        if (isfinite(ord_decode(row[0])))
            for (int q = 0; q < 4; ++q) { gf[q] = ord_decode(row[2 + q]); gs[q] = ord_decode(row[6 + q]); }
    }
    if (!interaction_grids(C.o, gs[0], gs[1], gs[2], gs[3], gf[0], gf[1], gf[2], gf[3], sg, fg)) {
        record_error(C.status, t, 3, 0);
        return;
    }
    if (C.o.green_cache) {
        CacheEntry &e = C.cache[T.key];
        bool usable = e.valid && grid_size_usable(e.sg, sg, C.o.min_ratio) && grid_size_usable(e.fg, fg, C.o.min_ratio) &&
                      grid_covers(C.o, e.sg, sxmin, sxmax, symin, symax) &&
                      grid_covers(C.o, e.fg, fxmin, fxmax, fymin, fymax);
        if (usable) {
            atomicAdd((unsigned long long *)&C.status->hits, 1ull);
            e.uses += 1;
            G.sg = e.sg;
            G.fg = e.fg;
            G.green = T.key;
            return;
        }
        Grid es = expand_grid(sg, 1.0 + C.o.growth);
        Grid ef = expand_grid(fg, 1.0 + C.o.growth);
        if (C.o.green_type != 0) {  // pic_cpu.jl:1853-1862 (:integrated is left untouched)
            double hx = es.w / (double)(C.o.nx - 1), hy = es.h / (double)(C.o.ny - 1);
            align_origins(C.o.green_type, es.x0, ef.x0, hx, es.x0, ef.x0);
            align_origins(C.o.green_type, es.y0, ef.y0, hy, es.y0, ef.y0);
        }
        if (!e.valid) {
            atomicAdd((unsigned long long *)&C.status->misses, 1ull);
            e.rebuilds = 0;
        } else {
            atomicAdd((unsigned long long *)&C.status->rebuilds, 1ull);
            e.rebuilds += 1;
        }
        e.valid = 1;
        e.uses = 1;
        e.sg = es;
        e.fg = ef;
        G.sg = es;
        G.fg = ef;
        G.green = T.key;
        G.rebuild = 1;
        return;
    }
    G.sg = sg;
    G.fg = fg;
    G.green = slot_scratch0 + tl;
    G.rebuild = 1;
}

// Luminosity mesh of a pair from its virtual-position box (pic_cpu.jl:2706-2723); false with err = 1
// (non-finite position) or 3 (degenerate extent).  t1: the pair's direction-1 task.
__device__ __forceinline__ bool lum_geometry(const Collide &C, const LumJob &J, int t1, LumGeom &L, int &err) {
    L.ok = 0;
    err = 0;
    const unsigned long long *b = C.lumb + (long long)J.pair * 4;
    double xmin = ord_decode(b[0]), xmax = ord_decode(b[1]), ymin = ord_decode(b[2]), ymax = ord_decode(b[3]);
    if ((C.nanflag[t1] & 4) || (C.nanflag[t1 + 1] & 4)) { err = 1; return false; }
    double width, height;
    if (!resolve_extent(C.o, xmax - xmin, ymax - ymin, width, height)) { err = 3; return false; }
    const int nx = C.o.lnx, ny = C.o.lny;
    const double tx = width / ((double)nx - 1.1);
    const double ty = height / ((double)ny - 1.1);
    width += 0.1 * tx;
    height += 0.1 * ty;
    xmin -= 0.05 * tx;
    ymin -= 0.05 * ty;
    L.x0 = xmin;
    L.y0 = ymin;
    L.hx = width / (double)(nx - 1);
    L.hy = height / (double)(ny - 1);
    L.ok = 1;
    return true;
}

// ------------------------------------------------------------------ Green function
// pic_cpu.jl:2254-2272
__device__ __forceinline__ double atan_ratio(double num, double den) {
    if (den == 0.0) {
        if (num == 0.0) return 0.0;
        return copysign(1.5707963267948966, num);
    }
    return atan(num / den);
}
__device__ __forceinline__ double kernel_integral(double x, double y) {
    double r2 = x * x + y * y;
    if (r2 == 0.0) return 0.0;
    return (log(r2) - 3) * x * y + atan_ratio(y, x) * x * x + atan_ratio(x, y) * y * y;
}
// The same F with one arctangent: atan(x/y) = sign(xy) pi/2 - atan(y/x) off the axes; on an axis every term
// vanishes (x = 0 or y = 0 gives F = 0 exactly, as atan_ratio does).  The second arctangent's rounding
// changes F by an ulp of its magnitude, the level the Green table's second differences already carry.
__device__ __forceinline__ double kernel_integral_1atan(double x, double y) {
    if (x == 0.0 || y == 0.0) return 0.0;
    const double r2 = x * x + y * y;
    const double a = atan(y / x);
    const double b = ((x > 0.0) == (y > 0.0) ? 1.5707963267948966 : -1.5707963267948966) - a;
    return (log(r2) - 3) * x * y + a * x * x + b * y * y;
}
// One cell of the wrapped (2nx x 2ny) Green table (pic_cpu.jl:2478-2509).
__device__ __forceinline__ double green_value(int green_type, int i, int j, int nx, int ny, double dx0, double dy0,
                                              double hx, double hy) {
    int ii = i < nx ? i : i - 2 * nx;
    int jj = j < ny ? j : j - 2 * ny;
    double x = dx0 + (double)ii * hx;
    double y = dy0 + (double)jj * hy;
    double half_hx = hx / 2, half_hy = hy / 2;
    if (green_type != 0) {
        double r2 = x * x + y * y;
        if (r2 != 0.0) return -0.5 * log(r2);
    }
    double hxihyi = -0.5 / (hx * hy);
    double val = kernel_integral(x + half_hx, y + half_hy);
    val += kernel_integral(x - half_hx, y - half_hy);
    val -= kernel_integral(x + half_hx, y - half_hy);
    val -= kernel_integral(x - half_hx, y + half_hy);
    return hxihyi * val;
}

// Green table rows transformed along x: two table rows per warp as one complex line, written as
// the nx+1 non-redundant x-frequencies of each row into the slot.  A block covers kGreenRows
// consecutive table rows.  For :integrated the four corner integrals of a cell are shared with its
// neighbours: the block evaluates F once on the (2nx+1) x (kGreenRows+1) corner lattice in shared
// memory (corner a is (dx0 + (a-1)hx) + hx/2, bit-equal to the reference's "+" corner of cell a-1),
// 3.5x fewer log/atan evaluations than four per cell.
// mode 0: blockIdx.y = task of the front (only tasks that rebuild); mode 1: blockIdx.y = node mesh.
constexpr int kGreenRows = 8;
__global__ void __launch_bounds__(128) k_green_rows(Collide C, int mode, int base, int node_slot0) {
    pdl_wait();
    pdl_release();
    double2 *sm = (double2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx, NY = 2 * ny;
    const FftLen fx = fft_len(NX);
    double2 *tw = sm;
    double2 *lines = sm + NX / 2;
    double *corner = (double *)(lines + 4 * NX);  // (kGreenRows + 1) x (NX + 1)
    Grid sg, fg;
    int slot;
    if (mode == 0) {
        const TaskGeom &G = C.geom[base + blockIdx.y];
        if (!G.rebuild) return;
        sg = G.sg; fg = G.fg; slot = G.green;
    } else {
        const NodeMesh &M = C.nodes[base + blockIdx.y];
        if (!M.valid) return;
        sg = M.sg; fg = M.fg; slot = node_slot0 + base + blockIdx.y;
    }
    load_twiddles(tw, C.tw_x, NX);
    const double hx = sg.w / (double)(nx - 1), hy = sg.h / (double)(ny - 1);
    const double dx0 = fg.x0 - sg.x0, dy0 = fg.y0 - sg.y0;
    const double half_hx = hx / 2, half_hy = hy / 2;
    const int j0 = blockIdx.x * kGreenRows;             // table rows j0 .. j0+7 (never straddle ny)
    const int jj0 = j0 < ny ? j0 : j0 - NY;             // wrapped row index of j0
    const bool integrated = C.o.green_type == 0;
    if (integrated) {
        for (int e = threadIdx.x; e < (kGreenRows + 1) * (NX + 1); e += blockDim.x) {
            const int rb = e / (NX + 1), ca = e % (NX + 1);
            const int b = jj0 + rb, a = ca - nx;           // corner indices: cell b-1 "+" corner
            const double X = a > -nx ? (dx0 + (double)(a - 1) * hx) + half_hx : (dx0 + (double)a * hx) - half_hx;
            const double Y = b > -ny ? (dy0 + (double)(b - 1) * hy) + half_hy : (dy0 + (double)b * hy) - half_hy;
            corner[e] = kernel_integral_1atan(X, Y);
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double hxihyi = -0.5 / (hx * hy);
    double2 *line = lines + warp * NX;
    double2 *out = C.ghat + (long long)slot * C.gstride;
    for (int pr = warp; 2 * pr < kGreenRows; pr += 4) {
        const int r0 = 2 * pr;  // local rows r0, r0+1
        for (int i = lane; i < NX; i += 32) {
            const int ii = i < nx ? i : i - NX;
            double g[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int r = r0 + q;
                if (integrated) {
                    const double *lo = corner + r * (NX + 1), *hi = corner + (r + 1) * (NX + 1);
                    const int a = ii + nx;  // corner column of the cell's "-" x corner
                    double val = hi[a + 1];  // F(x+, y+)
                    val += lo[a];            // F(x-, y-)
                    val -= lo[a + 1];        // F(x+, y-)
                    val -= hi[a];            // F(x-, y+)
                    g[q] = hxihyi * val;
                } else {
                    g[q] = green_value(C.o.green_type, i, j0 + r, nx, ny, dx0, dy0, hx, hy);
                }
            }
            line[fft_pos(fx, i)] = make_double2(g[0], g[1]);
        }
        warp_fft(line, fx, tw, false);
        const int ja = j0 + r0, jb = ja + 1;
        for (int k = lane; k <= nx; k += 32) {
            double2 zk = line[fft_out(fx, k)], zm = conjg(line[fft_out(fx, (NX - k) % NX)]);
            double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y + zm.y));
            double2 D = csub(zk, zm);
            out[(long long)k * NY + ja] = A;
            out[(long long)k * NY + jb] = make_double2(0.5 * D.y, -0.5 * D.x);
        }
        __syncwarp();
    }
}

// Column transforms of the Green slots (length 2ny, in place, natural-order output).
__global__ void __launch_bounds__(128) k_green_cols(Collide C, int mode, int base, int node_slot0) {
    pdl_wait();
    pdl_release();
    double2 *sm = (double2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NY = 2 * ny;
    const FftLen fy = fft_len(NY);
    double2 *tw = sm;
    double2 *line = sm + NY / 2 + (threadIdx.x >> 5) * NY;
    int slot;
    if (mode == 0) {
        const TaskGeom &G = C.geom[base + blockIdx.y];
        if (!G.rebuild) return;
        slot = G.green;
    } else {
        if (!C.nodes[base + blockIdx.y].valid) return;
        slot = node_slot0 + base + blockIdx.y;
    }
    load_twiddles(tw, C.tw_y, NY);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (k > nx) return;
    double2 *col = C.ghat + (long long)slot * C.gstride + (long long)k * NY;
    for (int j = lane; j < NY; j += 32) line[fft_pos(fy, j)] = col[j];
    warp_fft(line, fy, tw, false);
    for (int j = lane; j < NY; j += 32) col[j] = line[fft_out(fy, j)];
}

// Two consecutive complex values, 2-element aligned, in one vector store (the row pairs of the forward
// x-transforms; measured: FFT phase 1.10 -> 1.07 ms per production turn).
__device__ __forceinline__ void store_pair(double2 *p, double2 a, double2 b) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y) : "memory");
}
__device__ __forceinline__ void store_pair(float2 *p, float2 a, float2 b) {
    *reinterpret_cast<float4 *>(p) = make_float4(a.x, a.y, b.x, b.y);
}

// Register-FFT forms of the two Green kernels (rfft.cuh) for NX = 8 Gx and NY = 8 Gy.  Rows: the block
// covers 8 * (32 / G) table rows, two per line, and the spectrum leaves in the same natural layout as
// k_green_rows'.  Columns: each line is one x-frequency column, stored back in register order
// (entry r * G + l holds frequency rf_spec(l, r)), the order k_conv_cols_r multiplies in.
template <int G>
__global__ void __launch_bounds__(128) k_green_rows_r(Collide C, int mode, int base, int node_slot0) {
    using RG = RfGeom<G>;
    constexpr int LPW = 32 / G, ROWS = 8 * LPW;
    double2 *sm = (double2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx, NY = 2 * ny;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, line = lane / G, l = lane & (G - 1);
    double2 *T = sm, *S = sm + RG::kTables + warp * RG::kWarpScratch;
    double *corner = (double *)(sm + RG::kTables + 4 * RG::kWarpScratch);  // (ROWS + 1) x (NX + 1)
    rf_tables<G>(T, C.tw_x);  // twiddles written once at context creation: built before the wait
    pdl_wait();
    pdl_release();
    Grid sg, fg;
    int slot;
    if (mode == 0) {
        const TaskGeom &Gm = C.geom[base + blockIdx.y];
        if (!Gm.rebuild) return;
        sg = Gm.sg; fg = Gm.fg; slot = Gm.green;
    } else {
        const NodeMesh &M = C.nodes[base + blockIdx.y];
        if (!M.valid) return;
        sg = M.sg; fg = M.fg; slot = node_slot0 + base + blockIdx.y;
    }
    const double hx = sg.w / (double)(nx - 1), hy = sg.h / (double)(ny - 1);
    const double dx0 = fg.x0 - sg.x0, dy0 = fg.y0 - sg.y0;
    const double half_hx = hx / 2, half_hy = hy / 2;
    const int j0 = blockIdx.x * ROWS;      // rows j0 .. j0 + ROWS - 1 (ROWS divides ny)
    const int jj0 = j0 < ny ? j0 : j0 - NY;
    const bool integrated = C.o.green_type == 0;
    if (integrated) {
        for (int e = threadIdx.x; e < (ROWS + 1) * (NX + 1); e += blockDim.x) {
            const int rb = e / (NX + 1), ca = e % (NX + 1);
            const int b = jj0 + rb, a = ca - nx;
            const double X = a > -nx ? (dx0 + (double)(a - 1) * hx) + half_hx : (dx0 + (double)a * hx) - half_hx;
            const double Y = b > -ny ? (dy0 + (double)(b - 1) * hy) + half_hy : (dy0 + (double)b * hy) - half_hy;
            corner[e] = kernel_integral_1atan(X, Y);
        }
    }
    __syncthreads();
    const double hxihyi = -0.5 / (hx * hy);
    const int r0 = 2 * (warp * LPW + line);
    double2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int i = l + G * m, ii = i < nx ? i : i - NX;
        double g[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int r = r0 + q;
            if (integrated) {
                const double *lo = corner + r * (NX + 1), *hi = corner + (r + 1) * (NX + 1);
                const int a = ii + nx;
                double val = hi[a + 1];
                val += lo[a];
                val -= lo[a + 1];
                val -= hi[a];
                g[q] = hxihyi * val;
            } else {
                g[q] = green_value(C.o.green_type, i, j0 + r, nx, ny, dx0, dy0, hx, hy);
            }
        }
        v[m] = make_double2(g[0], g[1]);
    }
    rf_fwd<G>(v, S, T);
    double2 *Sl = S + line * 8 * G;
#pragma unroll
    for (int r = 0; r < 8; ++r) Sl[rf_nat(rf_spec<G>(l, r))] = v[r];
    __syncwarp();
    const int ja = j0 + r0, jb = ja + 1;
    double2 *out = C.ghat + (long long)slot * C.gstride;
    for (int k = l; k <= nx; k += G) {
        const double2 zk = Sl[rf_nat(k)], zm = conjg(Sl[rf_nat((NX - k) % NX)]);
        const double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y + zm.y));
        const double2 D = csub(zk, zm);
        store_pair(out + (long long)k * NY + ja, A, make_double2(0.5 * D.y, -0.5 * D.x));  // ja even
    }
}

template <int G>
__global__ void __launch_bounds__(128) k_green_cols_r(Collide C, int mode, int base, int node_slot0) {
    using RG = RfGeom<G>;
    constexpr int LPW = 32 / G;
    double2 *sm = (double2 *)g_smem;
    const int nx = C.o.nx, NY = 2 * C.o.ny;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, line = lane / G, l = lane & (G - 1);
    double2 *T = sm, *S = sm + RG::kTables + warp * RG::kWarpScratch;
    rf_tables<G>(T, C.tw_y);  // before the wait (constant twiddles)
    pdl_wait();
    pdl_release();
    int slot;
    if (mode == 0) {
        const TaskGeom &Gm = C.geom[base + blockIdx.y];
        if (!Gm.rebuild) return;
        slot = Gm.green;
    } else {
        if (!C.nodes[base + blockIdx.y].valid) return;
        slot = node_slot0 + base + blockIdx.y;
    }
    const int k = (blockIdx.x * 4 + warp) * LPW + line;
    const bool ok = k <= nx;
    double2 *col = C.ghat + (long long)slot * C.gstride + (long long)k * NY;
    double2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = ok ? col[l + G * m] : make_double2(0.0, 0.0);
    __syncthreads();  // tables ready (the column's loads are already in flight)
    rf_fwd<G>(v, S, T);
    if (ok) {
#pragma unroll
        for (int r = 0; r < 8; ++r) col[r * G + l] = v[r];
    }
}

// ------------------------------------------------------------------ deposition
// Fixed-point CIC/TSC taps of one particle (pic_cpu.jl:2129-2146): q = round(w * 2^bits) added to an int64
// grid (a block-private shared-memory copy, merged into the plane's grid at the end of the block).
// The shared grid is addressed through an opaque generic pointer (generic_ptr): measured on B200, a
// 64-bit atomic add to shared memory issued on a generic address runs at 10.3 per clock per SM (4.1 under
// 4-way conflicts) against 5.2 (1.6) when the compiler sees the shared address space (the precision form's
// 32-bit atomics the other way round: faster on the shared-typed address, 1.45 -> 1.35 ms per turn).  Measured
// alternatives, all slower on the production turn: 32-bit split accumulators (two atomics per tap),
// warp-aggregated runs of equal cells, batched loads, and spatially sorted particles.
template <class T>
__device__ __forceinline__ T *generic_ptr(T *p) {
    asm("" : "+l"(p));  // hide the address space from the compiler
    return p;
}
// TOTAL: also return the sum of the quanta (the hybrid's neutralisation needs the plane's exact charge).
// rot (CIC): the lane's four atomics start at tap rot & 3 -- particles of a spatially ordered slice share
// cells with their warp neighbours, and rotating the tap order spreads a warp's simultaneous atomics over
// four addresses per cell.  Integer sums: the order changes nothing.
// Q: the accumulator's element type -- int64 for the plain form and for plane grids in global memory; int32 for
// the precision form's block-private shared grids, whose fixed-point scale (fixed_bits_for32) keeps a whole
// slice's charge in one cell below 2^30, so a tap is one 32-bit atomic.
__device__ __forceinline__ void atom_add(long long *p, long long v) {
    atomicAdd((unsigned long long *)p, (unsigned long long)v);
}
__device__ __forceinline__ void atom_add(int *p, int v) { atomicAdd(p, v); }
template <class Q, class R>
__device__ __forceinline__ Q quantize(R x) {
    if constexpr (sizeof(Q) == 8) return round_ll(x);
    else if constexpr (sizeof(R) == 4) return __float2int_rn(x);
    else return __double2int_rn(x);
}
template <class R, int METHOD, bool TOTAL = false, bool ROT = false, class Q = long long>
__device__ __forceinline__ long long deposit_taps(R u, R v, int nw, int nh, R scale, Q *grid, int ld, int rot = 0) {
    constexpr int NT = METHOD == 0 ? 2 : 3;
    int ix, iy;
    long long total = 0;
    R wx[NT], wy[NT];
    if (METHOD == 0) { cic_weights(u, nw, ix, wx); cic_weights(v, nh, iy, wy); }
    else { tsc_weights(u, nw, ix, wx); tsc_weights(v, nh, iy, wy); }
    const int c0 = (iy - 1) * ld + (ix - 1);
    if constexpr (METHOD == 0) {
        Q q0 = quantize<Q>(wx[0] * wy[0] * scale), q1 = quantize<Q>(wx[0] * wy[1] * scale);
        Q q2 = quantize<Q>(wx[1] * wy[0] * scale), q3 = quantize<Q>(wx[1] * wy[1] * scale);
        if (TOTAL) total = (long long)q0 + q1 + q2 + q3;
        int o0 = c0, o1 = c0 + ld, o2 = c0 + 1, o3 = c0 + ld + 1;
        if constexpr (ROT) {  // a separate instantiation: the permutation costs the unrotated deposit nothing
            if (rot & 1) {
                const int to = o0; o0 = o1; o1 = o2; o2 = o3; o3 = to;
                const Q tq = q0; q0 = q1; q1 = q2; q2 = q3; q3 = tq;
            }
            if (rot & 2) {
                int to = o0; o0 = o2; o2 = to; to = o1; o1 = o3; o3 = to;
                Q tq = q0; q0 = q2; q2 = tq; tq = q1; q1 = q3; q3 = tq;
            }
        }
        atom_add(&grid[o0], q0);
        atom_add(&grid[o1], q1);
        atom_add(&grid[o2], q2);
        atom_add(&grid[o3], q3);
    } else {
#pragma unroll
        for (int m = 0; m < NT; ++m)
#pragma unroll
            for (int k = 0; k < NT; ++k) {
                const Q qv = quantize<Q>(wx[m] * wy[k] * scale);
                if (TOTAL) total += qv;
                // a zero quantum (out-of-range particle: base 1, every weight 0) adds nothing; the unconditional
                // atomic measured faster than the test
                atom_add(&grid[c0 + k * ld + m], qv);
            }
    }
    return total;
}

// Merge a block's shared-memory grid into the plane's int64 grid.
template <class Q>
__device__ __forceinline__ void merge_grid(const Q *sq, long long *g, int cells) {
    for (int c = threadIdx.x; c < cells; c += blockDim.x) {
        const long long v = sq[c];
        if (v) atomicAdd((unsigned long long *)&g[c], (unsigned long long)v);
    }
}
// The block-private shared grid's element type: int32 in the precision form, int64 in the plain form.
template <class R>
using ShQ = typename std::conditional<sizeof(R) == 4, int, long long>::type;

// A global load that does not allocate in L1.
__device__ __forceinline__ double ld_no_l1(const double *p) {
    double v;
    asm("ld.global.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float ld_no_l1(const float *p) {
    float v;
    asm("ld.global.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

// Blocks of a k_deposit_node3 row: ceil(n / per_block), at most the grid (per_block <= 0: the whole grid).  A row
// of a large slice gets more blocks than one of a small slice, so a front's blocks fill whole waves of the SMs.
__device__ __forceinline__ int row_blocks(long long n, long long per_block) {
    if (per_block <= 0) return (int)gridDim.x;
    const long long b = (n + per_block - 1) / per_block;
    return (int)max(1ll, min((long long)gridDim.x, b));
}

// A deposit's source coordinate, read once per plane pass: the FP64 form skips L1 allocation (measured faster
// on the full turn), the FP32 form loads as usual (the hint measured slightly slower on its 64x64 grid).
__device__ __forceinline__ double ld_src(const double *p) { return ld_no_l1(p); }
__device__ __forceinline__ float ld_src(const float *p) { return *p; }

// Field-solve planes of a front.  grid: (blocks per plane, planes in front); each block deposits a
// grid-stride share of its plane's source slice into a private int64 copy of the nx*ny grid in shared
// memory, then merges it with global atomics (the consumer, k_conv_rows, clears the grid it reads).
template <class R, int METHOD>
__global__ void __launch_bounds__(1024, 1) k_deposit(Collide C, int plane0) {
    using Q = ShQ<R>;
    Q *sq = (Q *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, cells = nx * ny;
    // grids larger than shared memory (C.o.dep_global) accumulate straight into the plane's grid; the
    // block's shared grid is cleared before the wait (shared memory only)
    const bool local = !C.o.dep_global;
    if (local)
        for (int c = threadIdx.x; c < cells; c += blockDim.x) sq[c] = 0;
    pdl_wait();
    pdl_release();
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    Grid sg;
    if (P.geom >= 0) {
        if (!C.nodes[P.geom].valid) return;
        sg = C.nodes[P.geom].sg;
    } else {
        const TaskGeom &G = C.geom[P.task];
        if (G.green < 0) return;
        sg = G.sg;
    }
    __syncthreads();
    const double hx = sg.w / (double)(nx - 1), hy = sg.h / (double)(ny - 1);
    const R hxi = (R)(1.0 / hx), hyi = (R)(1.0 / hy);
    const R scale = (R)ldexp(1.0, P.fixed_bits);
    const SoA S = C.beam[P.src_beam];
    const R *X = col<R>(S, 0), *PX = col<R>(S, 1), *Y = col<R>(S, 2), *PY = col<R>(S, 3);
    const R s = (R)P.s;
    // the plane's fields in registers: the loop's atomics go through a generic pointer, which the compiler
    // cannot separate from the plane table in global memory, so it would reload them for every particle
    const int count_dropped = P.count_dropped;
    const long long src_n = P.src_n, src_start = P.src_start;
    const R s2 = count_dropped == 2 ? (R)C.tasks[P.task].sR : s;
    const R x0 = (R)sg.x0, y0 = (R)sg.y0;
    const R xlo = x0, xhi = (R)(sg.x0 + sg.w), ylo = y0, yhi = (R)(sg.y0 + sg.h);
    int outside = 0;
    long long total = 0;
    const int rot = C.o.dep_rotate ? (int)(threadIdx.x & 3) : 0;
    // the next particle's coordinates are loaded before the current one's taps, two loads in flight
    const long long stride = (long long)gridDim.x * blockDim.x;
    auto sweep = [&](auto with_total, auto rotated, auto *acc) {
        constexpr bool TOT = decltype(with_total)::value, ROT = decltype(rotated)::value;
        using QA = typename std::remove_pointer<decltype(acc)>::type;
        long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        R cx = 0, cpx = 0, cy = 0, cpy = 0;
        if (k < src_n) {
            const long long p = src_start + k;
            cx = ld_src(X + p); cpx = ld_src(PX + p); cy = ld_src(Y + p); cpy = ld_src(PY + p);
        }
        for (; k < src_n; k += stride) {
            R nx_ = 0, npx = 0, ny_ = 0, npy = 0;
            if (k + stride < src_n) {
                const long long q = src_start + k + stride;
                nx_ = ld_src(X + q); npx = ld_src(PX + q); ny_ = ld_src(Y + q); npy = ld_src(PY + q);
            }
            const R xd = cx + cpx * s;
            const R yd = cy + cpy * s;
            if (count_dropped && !(isfinite(xd) && xlo <= xd && xd <= xhi && isfinite(yd) && ylo <= yd && yd <= yhi))
                ++outside;
            else if (count_dropped == 2) {  // :sigma and :source_slice: the particle at the other boundary too
                const R x2 = cx + cpx * s2, y2 = cy + cpy * s2;
                if (!(isfinite(x2) && xlo <= x2 && x2 <= xhi && isfinite(y2) && ylo <= y2 && y2 <= yhi)) ++outside;
            }
            total += deposit_taps<R, METHOD, TOT, ROT, QA>((xd - x0) * hxi, (yd - y0) * hyi, nx, ny, scale, acc, nx, rot);
            cx = nx_; cpx = npx; cy = ny_; cpy = npy;
        }
    };
    // (the hybrid's exact plane totals and the rotation for spatially ordered slices never combine)
    auto run = [&](auto *acc) {
        if (C.o.gaussian) sweep(std::true_type(), std::false_type(), acc);
        else if (C.o.dep_rotate) sweep(std::false_type(), std::true_type(), acc);
        else sweep(std::false_type(), std::false_type(), acc);
    };
    if constexpr (sizeof(Q) == 8) {  // one pointer, one instance of the loop
        run(local ? generic_ptr(sq) : C.qgrid + (long long)pl * cells);
    } else {  // 32-bit shared atomics measured faster on the shared-typed address than on a generic one
        if (local) run(sq);
        else run(C.qgrid + (long long)pl * cells);
    }
    if (C.o.gaussian) {  // the plane's exact total charge, for the neutralised subtraction
        for (int o = 16; o; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
        if ((threadIdx.x & 31) == 0 && total) atomicAdd(&C.qtot[pl], (unsigned long long)total);
    }
    if (count_dropped) {
        for (int o = 16; o; o >>= 1) outside += __shfl_xor_sync(0xffffffffu, outside, o);
        if ((threadIdx.x & 31) == 0 && outside) atomicAdd((unsigned long long *)&C.status->dropped, (unsigned long long)outside);
    }
    if (local) {
        __syncthreads();
        merge_grid(sq, C.qgrid + (long long)pl * cells, cells);
    }
}

// The precision form's :node deposit with the three planes of a task in one pass (int32 block grids, all three
// in shared memory up to 128 x 128): L (the sL drift on the L mesh), R (sR on the R mesh) and Z (sR on the L
// mesh; only with the longitudinal kick) read the source particle and compute its two drifts once.  grid:
// (blocks per task, tasks in front); ppt = 2 or 3 planes per task, consecutive.  Every quantum is the
// expression of k_deposit, so the grids are bit-identical to k_deposit's planes.
template <class R, int METHOD>
__global__ void __launch_bounds__(1024, 1) k_deposit_node3(Collide C, int plane0, int ppt, long long per_block) {
    int *sq = (int *)g_smem;  // L | R | Z
    const int nx = C.o.nx, ny = C.o.ny, cells = nx * ny;
    for (int c = threadIdx.x; c < ppt * cells; c += blockDim.x) sq[c] = 0;
    pdl_wait();
    pdl_release();
    const int pl = ppt * blockIdx.y;
    const bool z = ppt == 3;
    const Plane &PL = C.planes[plane0 + pl], &PR = C.planes[plane0 + pl + 1];
    const int nblk = row_blocks(PL.src_n, per_block);
    if ((int)blockIdx.x >= nblk) return;  // block-uniform: this row needs fewer blocks than the grid has
    const bool okL = C.nodes[PL.geom].valid != 0, okR = C.nodes[PR.geom].valid != 0;
    if (!okL && !okR) return;  // block-uniform
    const Grid gL = C.nodes[PL.geom].sg, gR = C.nodes[PR.geom].sg;
    __syncthreads();
    const R hxiL = (R)(1.0 / (gL.w / (double)(nx - 1))), hyiL = (R)(1.0 / (gL.h / (double)(ny - 1)));
    const R hxiR = (R)(1.0 / (gR.w / (double)(nx - 1))), hyiR = (R)(1.0 / (gR.h / (double)(ny - 1)));
    const R scale = (R)ldexp(1.0, PL.fixed_bits);
    const SoA S = C.beam[PL.src_beam];
    const R *X = col<R>(S, 0), *PX = col<R>(S, 1), *Y = col<R>(S, 2), *PY = col<R>(S, 3);
    const R sL = (R)PL.s, sR = (R)PR.s;
    const long long src_n = PL.src_n, src_start = PL.src_start;
    const R xL0 = (R)gL.x0, yL0 = (R)gL.y0, xR0 = (R)gR.x0, yR0 = (R)gR.y0;
    const R xLhi = (R)(gL.x0 + gL.w), yLhi = (R)(gL.y0 + gL.h), xRhi = (R)(gR.x0 + gR.w), yRhi = (R)(gR.y0 + gR.h);
    int outside = 0;
    const long long stride = (long long)nblk * blockDim.x;
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    R cx = 0, cpx = 0, cy = 0, cpy = 0;
    if (k < src_n) {
        const long long p = src_start + k;
        cx = ld_src(X + p); cpx = ld_src(PX + p); cy = ld_src(Y + p); cpy = ld_src(PY + p);
    }
    for (; k < src_n; k += stride) {
        R nx_ = 0, npx = 0, ny_ = 0, npy = 0;
        if (k + stride < src_n) {
            const long long q = src_start + k + stride;
            nx_ = ld_src(X + q); npx = ld_src(PX + q); ny_ = ld_src(Y + q); npy = ld_src(PY + q);
        }
        const R xl = cx + cpx * sL, yl = cy + cpy * sL;
        const R xr = cx + cpx * sR, yr = cy + cpy * sR;
        if (okL) {
            if (!(isfinite(xl) && xL0 <= xl && xl <= xLhi && isfinite(yl) && yL0 <= yl && yl <= yLhi)) ++outside;
            deposit_taps<R, METHOD, false, false, int>((xl - xL0) * hxiL, (yl - yL0) * hyiL, nx, ny, scale, sq, nx);
            if (z)
                deposit_taps<R, METHOD, false, false, int>((xr - xL0) * hxiL, (yr - yL0) * hyiL, nx, ny, scale, sq + 2 * cells,
                                                           nx);
        }
        if (okR) {
            if (!(isfinite(xr) && xR0 <= xr && xr <= xRhi && isfinite(yr) && yR0 <= yr && yr <= yRhi)) ++outside;
            deposit_taps<R, METHOD, false, false, int>((xr - xR0) * hxiR, (yr - yR0) * hyiR, nx, ny, scale, sq + cells, nx);
        }
        cx = nx_; cpx = npx; cy = ny_; cpy = npy;
    }
    for (int o = 16; o; o >>= 1) outside += __shfl_xor_sync(0xffffffffu, outside, o);
    if ((threadIdx.x & 31) == 0 && outside) atomicAdd((unsigned long long *)&C.status->dropped, (unsigned long long)outside);
    __syncthreads();
    for (int g = 0; g < ppt; ++g)
        if (g == 1 ? okR : okL) merge_grid(sq + g * cells, C.qgrid + (long long)(pl + g) * cells, cells);
}

// Luminosity planes: 2 per pair (side 0 = beam-1 slice i at sM1, side 1 = beam-2 slice j at sM2)
// on the (lnx+1) x (lny+1) overlap mesh (pic_cpu.jl:2724-2735).
// Every block derives its pair's mesh (lum_geometry); block (0, side 0) publishes it and reports errors.
template <class R, int METHOD>
__global__ void __launch_bounds__(1024, 1) k_lum_deposit(Collide C, int lj0, int task0) {
    pdl_wait();
    pdl_release();
    using Q = ShQ<R>;
    Q *sq = (Q *)g_smem;
    const int ql = blockIdx.y >> 1, side = blockIdx.y & 1;
    const LumJob &J = C.lumjobs[lj0 + ql];
    LumGeom L;
    int err;
    const bool ok = lum_geometry(C, J, task0 + 2 * ql, L, err);
    if (blockIdx.x == 0 && side == 0 && threadIdx.x == 0) {
        C.lumgeom[J.pair] = L;
        if (!ok) record_error(C.status, task0 + 2 * ql, err, err == 1 ? 1 : 0);
    }
    if (!ok) return;
    const int nw = C.o.lnx + 1, nh = C.o.lny + 1, cells = nw * nh;
    const bool local = !C.o.lum_global;
    if (local)
        for (int c = threadIdx.x; c < cells; c += blockDim.x) sq[c] = 0;
    __syncthreads();
    const SoA S = C.beam[side];
    const R *X = col<R>(S, 0), *PX = col<R>(S, 1), *Y = col<R>(S, 2), *PY = col<R>(S, 3);
    const long long st = side ? J.s2_start : J.s1_start, n = side ? J.s2_n : J.s1_n;
    const R s = (R)(side ? J.sM2 : J.sM1);
    const R scale = (R)ldexp(1.0, side ? J.bits2 : J.bits1);
    const R hxi = (R)(1.0 / L.hx), hyi = (R)(1.0 / L.hy);
    const R x0 = (R)L.x0, y0 = (R)L.y0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int rot = C.o.dep_rotate ? (int)(threadIdx.x & 3) : 0;
    auto sweep = [&](auto rotated, auto *acc) {
        constexpr bool ROT = decltype(rotated)::value;
        using QA = typename std::remove_pointer<decltype(acc)>::type;
        long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        R cx = 0, cpx = 0, cy = 0, cpy = 0;
        if (k < n) {
            const long long p = st + k;
            cx = ld_src(X + p); cpx = ld_src(PX + p); cy = ld_src(Y + p); cpy = ld_src(PY + p);
        }
        for (; k < n; k += stride) {  // next particle prefetched, as in k_deposit
            R nx_ = 0, npx = 0, ny_ = 0, npy = 0;
            if (k + stride < n) {
                const long long q = st + k + stride;
                nx_ = ld_src(X + q); npx = ld_src(PX + q); ny_ = ld_src(Y + q); npy = ld_src(PY + q);
            }
            const R vx = cx + cpx * s;
            const R vy = cy + cpy * s;
            deposit_taps<R, METHOD, false, ROT, QA>((vx - x0) * hxi, (vy - y0) * hyi, nw, nh, scale, acc, nw, rot);
            cx = nx_; cpx = npx; cy = ny_; cpy = npy;
        }
    };
    auto run = [&](auto *acc) {
        if (C.o.dep_rotate) sweep(std::true_type(), acc);
        else sweep(std::false_type(), acc);
    };
    if constexpr (sizeof(Q) == 8) {
        run(local ? generic_ptr(sq) : C.lq + (long long)blockIdx.y * cells);
    } else {
        if (local) run(sq);
        else run(C.lq + (long long)blockIdx.y * cells);
    }
    if (local) {
        __syncthreads();
        merge_grid(sq, C.lq + (long long)blockIdx.y * cells, cells);
    }
}

// Overlap integral per pair: sum q1*q2 over the full (nx+1)(ny+1) extent (pic_cpu.jl:2725-2736),
// split over kLumSplit blocks per pair into fixed partial sums (deterministic), clearing both grids for
// the next front.
constexpr int kLumSplit = 16;
__global__ void __launch_bounds__(256) k_lum_overlap(Collide C, int lj0) {
    pdl_wait();
    pdl_release();
    const int ql = blockIdx.y, part = blockIdx.x;
    const LumJob &J = C.lumjobs[lj0 + ql];
    const int cells = (C.o.lnx + 1) * (C.o.lny + 1);
    const int per = (cells + kLumSplit - 1) / kLumSplit;
    const int c0 = part * per, c1 = min(cells, c0 + per);
    long long *q1 = C.lq + (long long)(2 * ql) * cells;
    long long *q2 = q1 + cells;
    const double i1 = ldexp(1.0, -J.bits1), i2 = ldexp(1.0, -J.bits2);
    double acc = 0.0;
    for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        const long long a = q1[c], b = q2[c];
        if (a && b) acc += ((double)a * i1) * ((double)b * i2);
        if (a) q1[c] = 0;
        if (b) q2[c] = 0;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x >> 1; o; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // the pair's last block to finish adds the kLumSplit partials in order and applies klum/(hx hy)
        C.lum_partial[(long long)ql * kLumSplit + part] = red[0];
        __threadfence();
        const unsigned ticket = atomicAdd(&C.lum_tick[ql], 1u);
        if (ticket == kLumSplit - 1) {
            __threadfence();
            const LumGeom &L = C.lumgeom[J.pair];
            if (L.ok) {
                double sum = 0.0;
                for (int k = 0; k < kLumSplit; ++k) sum += __ldcg(&C.lum_partial[(long long)ql * kLumSplit + k]);
                const double hxi = 1.0 / L.hx, hyi = 1.0 / L.hy;
                C.lum_parts[J.pair] = sum * C.klum * hxi * hyi;
            }
            C.lum_tick[ql] = 0u;  // ready for the next front
        }
    }
}

// Hybrid: erf-integrated CIC/TSC node profiles of the reference Gaussian of each field-solve plane
// (gaussian_pic.jl:206-237) on its source grid, and their sums (the neutralisation denominator).
// One block per plane of the front.
__device__ __forceinline__ double gauss_node_weight(int method, double xi, double h, double mu, double s) {
    const double invroot = 1.0 / (s * 1.4142135623730951);
    const double norm = 1.0 / (s * 2.5066282746310002);  // s * sqrt(2 pi)
    auto pdf = [&](double x) { return norm * exp(-((x - mu) * (x - mu)) / (2.0 * s * s)); };
    auto m0 = [&](double A, double B) { return 0.5 * (erf((B - mu) * invroot) - erf((A - mu) * invroot)); };
    auto m1 = [&](double A, double B) { return (mu - xi) * m0(A, B) - s * s * (pdf(B) - pdf(A)); };
    auto m2 = [&](double A, double B) {
        return (s * s + (mu - xi) * (mu - xi)) * m0(A, B) - s * s * ((B - mu) * pdf(B) - (A - mu) * pdf(A)) -
               2.0 * (mu - xi) * s * s * (pdf(B) - pdf(A));
    };
    if (method == 0) return m0(xi - h, xi + h) + (m1(xi - h, xi) - m1(xi, xi + h)) / h;
    const double half = h / 2.0;
    const double cL = xi - half, cR = xi + half, lL = xi - 3.0 * half, lR = xi - half, rL = xi + half,
                 rR = xi + 3.0 * half;
    return 0.75 * m0(cL, cR) - m2(cL, cR) / (h * h) + 1.125 * (m0(lL, lR) + m0(rL, rR)) +
           1.5 * (m1(lL, lR) - m1(rL, rR)) / h + 0.5 * (m2(lL, lR) + m2(rL, rR)) / (h * h);
}

// Coupled subtraction (gaussian_pic.jl:240-372): central moments c_0..c_4 of the unit Gaussian over [A, B] by
// the integration-by-parts recursion, shifted to node-centred moments about xi (d = mu - xi).
__device__ __forceinline__ void gauss_cell_moments(double A, double B, double mu, double s, double xi, double m[5]) {
    const double invroot = 1.0 / (s * 1.4142135623730951);
    const double norm = 1.0 / (s * 2.5066282746310002);  // s * sqrt(2 pi)
    const double a = A - mu, b = B - mu;
    const double GA = norm * exp(-(a * a) / (2.0 * s * s));
    const double GB = norm * exp(-(b * b) / (2.0 * s * s));
    const double s2 = s * s;
    double c[5];
    c[0] = 0.5 * (erf(b * invroot) - erf(a * invroot));
    c[1] = -s2 * (GB - GA);
    c[2] = -s2 * (b * GB - a * GA) + s2 * c[0];
    c[3] = -s2 * (b * b * GB - a * a * GA) + 2.0 * s2 * c[1];
    c[4] = -s2 * (b * b * b * GB - a * a * a * GA) + 3.0 * s2 * c[2];
    const double d = mu - xi, d2 = d * d, d3 = d2 * d, d4 = d3 * d;
    m[0] = c[0];
    m[1] = c[1] + d * c[0];
    m[2] = c[2] + 2.0 * d * c[1] + d2 * c[0];
    m[3] = c[3] + 3.0 * d * c[2] + 3.0 * d2 * c[1] + d3 * c[0];
    m[4] = c[4] + 4.0 * d * c[3] + 6.0 * d2 * c[2] + 4.0 * d3 * c[1] + d4 * c[0];
}
// Assignment-weighted moments W_k = int (x - xi)^k G W(x - xi), k = 0, 1, 2 (gaussian_pic.jl:304-324).
__device__ __forceinline__ void gauss_weighted_moments(int method, double xi, double h, double mu, double s, double W[3]) {
    if (method == 0) {
        double L[5], Rm[5];
        gauss_cell_moments(xi - h, xi, mu, s, xi, L);
        gauss_cell_moments(xi, xi + h, mu, s, xi, Rm);
        for (int k = 0; k < 3; ++k) W[k] = (L[k] + L[k + 1] / h) + (Rm[k] - Rm[k + 1] / h);
        return;
    }
    const double half = h / 2.0;
    double Cm[5], Lw[5], Rw[5];
    gauss_cell_moments(xi - half, xi + half, mu, s, xi, Cm);
    gauss_cell_moments(xi - 3.0 * half, xi - half, mu, s, xi, Lw);
    gauss_cell_moments(xi + half, xi + 3.0 * half, mu, s, xi, Rw);
    for (int k = 0; k < 3; ++k) {
        const double core = 0.75 * Cm[k] - Cm[k + 2] / (h * h);
        const double wl = 1.125 * Lw[k] + 1.0 * 1.5 * Lw[k + 1] / h + 0.5 * Lw[k + 2] / (h * h);
        const double wr = 1.125 * Rw[k] + -1.0 * 1.5 * Rw[k + 1] / h + 0.5 * Rw[k + 2] / (h * h);
        W[k] = core + wl + wr;
    }
}
// Mean-derivatives g', g'' of the 1D node profile (gaussian_pic.jl:330-348).
__device__ __forceinline__ void gauss_profile_derivs(int method, double yj, double h, double mu, double s, double &dg,
                                                     double &ddg) {
    const double invroot = 1.0 / (s * 1.4142135623730951);
    const double norm = 1.0 / (s * 2.5066282746310002);
    auto pdf = [&](double y) { return norm * exp(-((y - mu) * (y - mu)) / (2.0 * s * s)); };
    auto m0 = [&](double A, double B) { return 0.5 * (erf((B - mu) * invroot) - erf((A - mu) * invroot)); };
    if (method == 0) {
        dg = (m0(yj - h, yj) - m0(yj, yj + h)) / h;
        ddg = (pdf(yj - h) - 2.0 * pdf(yj) + pdf(yj + h)) / h;
        return;
    }
    const double half = h / 2.0;
    double Cm[5], Lw[5], Rw[5];
    gauss_cell_moments(yj - half, yj + half, mu, s, yj, Cm);
    gauss_cell_moments(yj - 3.0 * half, yj - half, mu, s, yj, Lw);
    gauss_cell_moments(yj + half, yj + 3.0 * half, mu, s, yj, Rw);
    dg = -2.0 * Cm[1] / (h * h) + (1.5 * Lw[0] + Lw[1] / h) / h + (-1.5 * Rw[0] + Rw[1] / h) / h;
    ddg = (-2.0 * m0(yj - half, yj + half) + m0(yj - 3.0 * half, yj - half) + m0(yj + half, yj + 3.0 * half)) / (h * h);
}

// Hybrid: the subtracted reference Gaussian of rows j0, j1 of a plane, amp * gx[i] * gy[j]
// (gaussian_pic.jl:580-589), or for the coupled subtraction amp * (gx[i] gy[j] + lambda m1x[i] g'y[j] +
// lambda^2 / 2 m2x[i] g''y[j]) (gaussian_pic.jl:612-630); amp neutralises it to the plane's deposited charge,
// else it carries the slice's particle count.  A precision-form difference plane, sgn (q_self - q_other),
// subtracts the same difference of the two planes' Gaussians: sgn (G_self - G_other).
struct HybRows {
    struct Side {
        const double *gx = nullptr, *m1x = nullptr, *m2x = nullptr;
        double g[2] = {0.0, 0.0}, d[2] = {0.0, 0.0}, e[2] = {0.0, 0.0};  // amp gy, amp lam g'y, amp lam^2/2 g''y
        __device__ double at(int i, int r, bool cpl) const {
            return cpl ? gx[i] * g[r] + m1x[i] * d[r] + m2x[i] * e[r] : gx[i] * g[r];
        }
    };
    Side self, other;
    bool diff = false, cpl = false;
    __device__ static void load(const Collide &C, const Plane &P, int pl, double inv, bool cpl, int j0, int j1, Side &S) {
        const int nx = C.o.nx, ny = C.o.ny, L = nx + ny;
        S.gx = C.hprof + (long long)pl * 3 * L;
        S.m1x = S.gx + L;
        S.m2x = S.gx + 2 * L;
        const double *gy = S.gx + nx, *dgy = S.m1x + nx, *ddgy = S.m2x + nx;
        double am = (double)P.src_n, lam = 0.0, half_lam2 = 0.0;
        if (cpl) {
            const HybridTask &H = C.hyb[P.task];
            lam = H.lam[P.kind == 0 ? 0 : 1];
            half_lam2 = 0.5 * lam * lam;
            const double sg = C.hsum[2 * pl];
            if (C.o.neutralize && sg != 0.0) am = ((double)(long long)C.qtot[pl] * inv) / sg;
        } else {
            const double sgx = C.hsum[2 * pl], sgy = C.hsum[2 * pl + 1];
            if (C.o.neutralize && sgx * sgy > 0.0) am = ((double)(long long)C.qtot[pl] * inv) / (sgx * sgy);
        }
        const int js[2] = {j0, j1};
        for (int r = 0; r < 2; ++r) {
            if (js[r] >= ny) continue;
            S.g[r] = am * gy[js[r]];
            if (cpl) {
                S.d[r] = am * lam * dgy[js[r]];
                S.e[r] = am * half_lam2 * ddgy[js[r]];
            }
        }
    }
    __device__ HybRows(const Collide &C, const Plane &P, int plane0, int pl, bool on, bool diff_plane, double inv, int j0,
                       int j1) {
        if (!on) return;
        cpl = C.hyb[P.task].mode == 2;
        load(C, P, pl, inv, cpl, j0, j1, self);
        diff = diff_plane;
        if (diff) {
            const int po = pl + P.other_delta;
            load(C, C.planes[plane0 + po], po, inv, cpl, j0, j1, other);
        }
    }
    __device__ double g0(int i, long long sgn) const {
        return diff ? (double)sgn * (self.at(i, 0, cpl) - other.at(i, 0, cpl)) : self.at(i, 0, cpl);
    }
    __device__ double g1(int i, long long sgn) const {
        return diff ? (double)sgn * (self.at(i, 1, cpl) - other.at(i, 1, cpl)) : self.at(i, 1, cpl);
    }
};


__global__ void __launch_bounds__(256) k_hyb_profiles(Collide C, int plane0) {
    pdl_wait();
    pdl_release();
    const int pl = blockIdx.x;
    const Plane &P = C.planes[plane0 + pl];
    const TaskGeom &G = C.geom[P.task];
    const HybridTask &H = C.hyb[P.task];
    if (G.green < 0 || !H.mode) return;
    const int nx = C.o.nx, ny = C.o.ny, side = P.kind == 0 ? 0 : 1, L = nx + ny;
    const Grid sg = G.sg;
    const double hx = sg.w / (double)(nx - 1), hy = sg.h / (double)(ny - 1);
    double *g = C.hprof + (long long)pl * 3 * L;
    if (H.mode == 2) {
        // the tilted Gaussian to second order in lambda (gaussian_pic.jl:350-370, 597-630): x moments about mux
        // (sigma sqrt(a)), the conditional y profile (sigma sigc) and its mean-derivatives
        const double mux = H.mux[side], muy = H.muy[side], sa = H.sa[side], sc = H.sigc[side];
        for (int i = threadIdx.x; i < L; i += blockDim.x) {
            if (i < nx) {
                const double xi = sg.x0 + (double)i * hx;
                double W[3];
                gauss_weighted_moments(C.o.method, xi, hx, mux, sa, W);
                const double d = mux - xi;
                g[i] = W[0];
                g[L + i] = W[1] - d * W[0];
                g[2 * L + i] = W[2] - 2.0 * d * W[1] + d * d * W[0];
            } else {
                const double yj = sg.y0 + (double)(i - nx) * hy;
                g[i] = gauss_node_weight(C.o.method, yj, hy, muy, sc);
                gauss_profile_derivs(C.o.method, yj, hy, muy, sc, g[L + i], g[2 * L + i]);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {  // sequential sums, node order; the subtracted grid's total mass
            double s[6] = {0, 0, 0, 0, 0, 0};
            for (int k = 0; k < 3; ++k) {
                for (int i = 0; i < nx; ++i) s[2 * k] += g[k * L + i];
                for (int j = 0; j < ny; ++j) s[2 * k + 1] += g[k * L + nx + j];
            }
            const double lam = H.lam[side], half_lam2 = 0.5 * lam * lam;
            C.hsum[2 * pl] = s[0] * s[1] + lam * s[2] * s[3] + half_lam2 * s[4] * s[5];
            C.hsum[2 * pl + 1] = 0.0;
        }
        return;
    }
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        if (i < nx) g[i] = gauss_node_weight(C.o.method, sg.x0 + (double)i * hx, hx, H.mux[side], H.sigx[side]);
        else g[i] = gauss_node_weight(C.o.method, sg.y0 + (double)(i - nx) * hy, hy, H.muy[side], H.sigy[side]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // sequential sums, node order
        double sx = 0.0, sy = 0.0;
        for (int i = 0; i < nx; ++i) sx += g[i];
        for (int j = 0; j < ny; ++j) sy += g[nx + j];
        C.hsum[2 * pl] = sx;
        C.hsum[2 * pl + 1] = sy;
    }
}

// ------------------------------------------------------------------ FFT convolution
__device__ __forceinline__ int plane_green(const Collide &C, const Plane &P) {
    if (P.green >= 0) return P.green;
    return C.geom[P.task].green;
}

// Forward x-transform of the charge rows: two rows per warp packed as one complex line
// (zero-padded to 2nx).  Plain form: the int64 grid is converted to FP64 and cleared as it is read.
// Precision form: the plane's int64 value is the exact difference with its partner plane when it has
// one (Plane::other_delta), and the host clears the front's grids after the launch.
template <class R>
__global__ void __launch_bounds__(128) k_conv_rows(Collide C, int plane0) {
    pdl_wait();
    pdl_release();
    using C2 = typename RealT<R>::C2;
    C2 *sm = (C2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx;
    const FftLen fx = fft_len(NX);
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    if (plane_green(C, P) < 0) return;
    C2 *tw = sm;
    C2 *line = sm + NX / 2 + (threadIdx.x >> 5) * NX;
    load_twiddles(tw, (const C2 *)C.twr_x, NX);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int j0 = 2 * r, j1 = j0 + 1;
    if (j0 >= ny) return;
    const double inv = ldexp(1.0, -P.fixed_bits);
    long long *q = C.qgrid + (long long)pl * nx * ny;
    constexpr bool kPrecision = sizeof(R) == 4;
    const long long *qo = q + (long long)P.other_delta * nx * ny;
    const bool diff = kPrecision && P.other_delta != 0;
    const long long sgn = P.self_first ? 1 : -1;
    // Hybrid: subtract amp * gx[i] * gy[j] (gaussian_pic.jl:580-589); amp neutralises the subtracted
    // Gaussian to the deposited charge, else it carries the slice's particle count.
    const bool hyb = C.o.gaussian && C.hyb[P.task].mode;
    const HybRows hr(C, P, plane0, pl, hyb, diff, inv, j0, j1);
    for (int i = lane; i < NX; i += 32) {
        C2 v;
        v.x = R(0);
        v.y = R(0);
        if (i < nx) {
            long long qa = q[(long long)j0 * nx + i];
            if (diff) qa = sgn * (qa - qo[(long long)j0 * nx + i]);
            v.x = hyb ? (R)((double)qa * inv - hr.g0(i, sgn)) : (R)((double)qa * inv);
            if (!kPrecision && qa) q[(long long)j0 * nx + i] = 0;
            if (j1 < ny) {
                long long qb = q[(long long)j1 * nx + i];
                if (diff) qb = sgn * (qb - qo[(long long)j1 * nx + i]);
                v.y = hyb ? (R)((double)qb * inv - hr.g1(i, sgn)) : (R)((double)qb * inv);
                if (!kPrecision && qb) q[(long long)j1 * nx + i] = 0;
            }
        }
        line[fft_pos(fx, i)] = v;
    }
    warp_fft(line, fx, tw, false);
    C2 *H = (C2 *)C.spec + (long long)pl * (nx + 1) * ny;
    for (int k = lane; k <= nx; k += 32) {
        C2 zk = line[fft_out(fx, k)], zm = conjg(line[fft_out(fx, (NX - k) % NX)]);
        C2 A, B;
        A.x = R(0.5) * (zk.x + zm.x);
        A.y = R(0.5) * (zk.y + zm.y);
        C2 D = csub(zk, zm);
        B.x = R(0.5) * D.y;
        B.y = R(-0.5) * D.x;
        store_pair(H + (long long)k * ny + j0, A, B);  // rows j0, j0 + 1 (j0 even, ny even)
    }
}

// y-transform, multiply by the (FP64) Green spectrum, inverse y-transform; one frequency column per
// warp.  Only rows j < ny of the result are kept (the field quadrant).  The inverse input is permuted in
// place for NY = 2^a (bit reversal is an involution) and through a second line for NY = 3 * 2^a.
template <class R>
__global__ void __launch_bounds__(128) k_conv_cols(Collide C, int plane0) {
    pdl_wait();
    pdl_release();
    using C2 = typename RealT<R>::C2;
    C2 *sm = (C2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NY = 2 * ny;
    const FftLen fy = fft_len(NY);
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    const int slot = plane_green(C, P);
    if (slot < 0) return;
    C2 *tw = sm;
    C2 *line = sm + NY / 2 + (threadIdx.x >> 5) * NY;
    C2 *line2 = sm + NY / 2 + (4 + (threadIdx.x >> 5)) * NY;  // NY = 3 * 2^a only
    load_twiddles(tw, (const C2 *)C.twr_y, NY);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (k > nx) return;
    C2 *col = (C2 *)C.spec + ((long long)pl * (nx + 1) + k) * ny;
    C2 zero;
    zero.x = R(0);
    zero.y = R(0);
    for (int j = lane; j < NY; j += 32) line[fft_pos(fy, j)] = j < ny ? col[j] : zero;
    warp_fft(line, fy, tw, false);
    const double2 *g = C.ghat + (long long)slot * C.gstride + (long long)k * NY;
    C2 *dst = fy.three ? line2 : line;
    for (int j = lane; j < NY; j += 32) {
        const double2 gv = g[j];
        C2 gg;
        gg.x = (R)gv.x;
        gg.y = (R)gv.y;
        const C2 v = cmul(line[fft_out(fy, j)], gg);
        if (fy.three) dst[fft_pos(fy, j)] = v;
        else line[fft_out(fy, j)] = v;
    }
    __syncwarp();
    if (!fy.three) {
        for (int j = lane; j < NY; j += 32) {  // bit-reverse permutation in place
            int r = bitrev(j, fy.lgM);
            if (j < r) { const int pj = sw(j), pr = sw(r); C2 t = line[pj]; line[pj] = line[pr]; line[pr] = t; }
        }
    }
    warp_fft(dst, fy, tw, true);
    for (int j = lane; j < ny; j += 32) col[j] = dst[fft_out(fy, j)];
}

// Field planes: a cell is (Ex, Ey, phi, w) as two double2 (plain form) or one float4 (precision form), so
// one tap of one plane is one 32-byte or 16-byte access, and a tap that needs only the field (the R mesh
// in :node mode) one 16-byte or 8-byte access.  The fourth word w of an L plane in :node mode carries phi of
// the task's Z plane (written by the Z plane's own k_conv_field block), so the L-mesh taps of the kick read
// Ex_L, Ey_L, phi_L and phi_Z in that one access.
__device__ __forceinline__ void store_cell(double2 *F, long long o, double phi, double ex, double ey) {
    F[2 * o] = make_double2(ex, ey);
    reinterpret_cast<double *>(F)[4 * o + 2] = phi;
}
__device__ __forceinline__ void store_cell(float4 *F, long long o, float phi, float ex, float ey) {
    reinterpret_cast<float2 *>(F)[2 * o] = make_float2(ex, ey);
    reinterpret_cast<float *>(F)[4 * o + 2] = phi;
}
__device__ __forceinline__ void store_w(double2 *F, long long o, double w) { reinterpret_cast<double *>(F)[4 * o + 3] = w; }
__device__ __forceinline__ void store_w(float4 *F, long long o, float w) { reinterpret_cast<float *>(F)[4 * o + 3] = w; }
// A plain-form cell is one 32-byte-aligned 256-bit load (sm_100 vector width); the planes are read-only
// while a kick runs, so the loads take the non-coherent path.  Measured: kick 2.49 -> 2.24 ms per
// production turn against two 128-bit loads per cell.  The address is computed from particle coordinates
// loaded after the kernel's programmatic-launch wait, which orders the load after it.
__device__ __forceinline__ void load_cell4(const double2 *F, long long c, double &phi, double &ex, double &ey, double &w) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(ex), "=d"(ey), "=d"(phi), "=d"(w) : "l"(F + 2 * c));
}
__device__ __forceinline__ void load_cell4(const float4 *F, long long c, float &phi, float &ex, float &ey, float &w) {
    const float4 v = F[c];
    ex = v.x; ey = v.y; phi = v.z; w = v.w;
}
__device__ __forceinline__ void load_field(const double2 *F, long long c, double &ex, double &ey) {
    const double2 a = F[2 * c];
    ex = a.x; ey = a.y;
}
__device__ __forceinline__ void load_field(const float4 *F, long long c, float &ex, float &ey) {
    const float2 a = reinterpret_cast<const float2 *>(F)[2 * c];
    ex = a.x; ey = a.y;
}
__device__ __forceinline__ void load_cell(const double2 *F, long long c, double &phi, double &ex, double &ey) {
    double w;
    load_cell4(F, c, phi, ex, ey, w);
}
__device__ __forceinline__ void load_cell(const float4 *F, long long c, float &phi, float &ex, float &ey) {
    const float4 v = F[c];
    ex = v.x; ey = v.y; phi = v.z;
}

// :node R planes with CIC taps are "pair cells": the kick reads only the field of an R plane, so the second
// half of cell (i, j) holds the field of cell (i + 1, j) instead of phi and w, and the two x-taps of a row
// are one 32-byte (16-byte) load.  The CIC base is clamped to i <= nx - 2, so the last cell's second half
// is never read.
__device__ __forceinline__ void store_field_pair(double2 *F, long long o, int i, double ex, double ey) {
    F[2 * o] = make_double2(ex, ey);
    if (i > 0) F[2 * o - 1] = make_double2(ex, ey);
}
__device__ __forceinline__ void store_field_pair(float4 *F, long long o, int i, float ex, float ey) {
    float2 *f = reinterpret_cast<float2 *>(F);
    f[2 * o] = make_float2(ex, ey);
    if (i > 0) f[2 * o - 1] = make_float2(ex, ey);
}
__device__ __forceinline__ void load_field_pair(const double2 *F, long long c, double &ex0, double &ey0, double &ex1,
                                                double &ey1) {
    asm("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(ex0), "=d"(ey0), "=d"(ex1), "=d"(ey1) : "l"(F + 2 * c));
}
__device__ __forceinline__ void load_field_pair(const float4 *F, long long c, float &ex0, float &ey0, float &ex1,
                                                float &ey1) {
    const float4 v = F[c];
    ex0 = v.x; ey0 = v.y; ex1 = v.z; ey1 = v.w;
}

// E = -grad(phi) on rows [jt0, jt1) of a plane (pic_cpu.jl:2531-2591) from the phi rows [ja0, ja1) held in
// shared memory, stored as field cells; the :node Z plane stores only its phi, into its L plane's w word.
template <class R>
__device__ __forceinline__ void field_cells(const Collide &C, const Plane &P, int pl, const Grid &sg, const R *phi,
                                            int ja0, int jt0, int jt1) {
    using FC = typename RealT<R>::FC;
    const int nx = C.o.nx, ny = C.o.ny;
    const double hx = sg.w / (double)(nx - 1), hy = sg.h / (double)(ny - 1);
    const R hxi = (R)(1.0 / hx), hyi = (R)(1.0 / hy);
    const R c4 = (R)(1.0 / 12.0);
    const bool fourth = C.o.fourth != 0;
    const bool zplane = P.kind == 3;  // :node Z plane: only its phi is used, stored in its L plane's w word
    const bool rpair = C.o.node && P.kind == 1 && C.o.method == 0;  // :node R plane, CIC: pair cells
    FC *F = (FC *)C.fields + (long long)(zplane ? pl - 2 : pl) * RealT<R>::kCellVec * nx * ny;
    auto Pv = [&](int i, int j) { return phi[(j - ja0) * nx + i]; };  // 0-based i, j
    for (int idx = threadIdx.x; idx < (jt1 - jt0) * nx; idx += blockDim.x) {
        const int j = jt0 + idx / nx, i = idx % nx;
        if (zplane) {
            store_w(F, (long long)j * nx + i, Pv(i, j));
            continue;
        }
        R ey, ex;
        // Ey (pic_cpu.jl:2553-2572), 1-based j' = j+1
        if (j == 0) ey = hyi * (R(1.5) * Pv(i, 0) - R(2) * Pv(i, 1) + R(0.5) * Pv(i, 2));
        else if (j == ny - 1) ey = hyi * (R(-1.5) * Pv(i, ny - 1) + R(2) * Pv(i, ny - 2) - R(0.5) * Pv(i, ny - 3));
        else if (fourth && (j == 1 || j == ny - 2)) ey = R(0.5) * hyi * (Pv(i, j - 1) - Pv(i, j + 1));
        else if (fourth) ey = c4 * hyi * ((Pv(i, j + 2) - Pv(i, j - 2)) + R(8) * (Pv(i, j - 1) - Pv(i, j + 1)));
        else ey = R(0.5) * hyi * (Pv(i, j - 1) - Pv(i, j + 1));
        // Ex (pic_cpu.jl:2573-2590)
        if (i == 0) ex = hxi * (R(1.5) * Pv(0, j) - R(2) * Pv(1, j) + R(0.5) * Pv(2, j));
        else if (i == nx - 1) ex = hxi * (R(-1.5) * Pv(nx - 1, j) + R(2) * Pv(nx - 2, j) - R(0.5) * Pv(nx - 3, j));
        else if (fourth && (i == 1 || i == nx - 2)) ex = R(0.5) * hxi * (Pv(i - 1, j) - Pv(i + 1, j));
        else if (fourth) ex = c4 * hxi * ((Pv(i + 2, j) - Pv(i - 2, j)) + R(8) * (Pv(i - 1, j) - Pv(i + 1, j)));
        else ex = R(0.5) * hxi * (Pv(i - 1, j) - Pv(i + 1, j));
        if (rpair) store_field_pair(F, (long long)j * nx + i, i, ex, ey);
        else store_cell(F, (long long)j * nx + i, Pv(i, j), ex, ey);
    }
}

// Two consecutive complex values, 2-element aligned, in one vector load (256-bit in FP64).  Measured: field
// phase 0.75 -> 0.68 ms per production turn against two loads.
// (volatile with a memory clobber: the address depends on no load, so nothing else keeps the compiler
// from moving it above the programmatic-launch wait or a barrier)
__device__ __forceinline__ void load_pair(const double2 *p, double2 &a, double2 &b) {
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p)
                 : "memory");
}
__device__ __forceinline__ void load_pair(const float2 *p, float2 &a, float2 &b) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    a.x = v.x; a.y = v.y; b.x = v.z; b.y = v.w;
}

// Inverse x-transform (two Hermitian rows per complex line) producing phi for a tile of rows plus a
// two-row halo, then E = -grad(phi) on the tile (pic_cpu.jl:2531-2591).
constexpr int kFieldTile = 8;
template <class R>
__global__ void __launch_bounds__(128) k_conv_field(Collide C, int plane0) {
    pdl_wait();
    pdl_release();
    using C2 = typename RealT<R>::C2;
    C2 *sm = (C2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx, NY = 2 * ny;
    const FftLen fx = fft_len(NX);
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    if (plane_green(C, P) < 0) return;
    Grid sg;
    if (P.geom >= 0) sg = C.nodes[P.geom].sg;
    else sg = C.geom[P.task].sg;
    C2 *tw = sm;
    C2 *lines = sm + NX / 2;
    R *phi = (R *)(lines + 4 * NX);  // (kFieldTile + 4) rows x nx
    load_twiddles(tw, (const C2 *)C.twr_x, NX);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int jt0 = blockIdx.x * kFieldTile;
    const int jt1 = min(jt0 + kFieldTile, ny);
    const int ja0 = max(jt0 - 2, 0), ja1 = min(jt1 + 2, ny);
    const int nrows = ja1 - ja0;
    const C2 *H = (const C2 *)C.spec + (long long)pl * (nx + 1) * ny;
    const R scale = (R)(1.0 / ((double)NX * (double)NY));
    C2 *line = lines + warp * NX;
    C2 zero;
    zero.x = R(0);
    zero.y = R(0);
    for (int rp = warp; 2 * rp < nrows; rp += 4) {
        const int ra = ja0 + 2 * rp, rb = ra + 1;
        const bool hb = rb < ja1;
        for (int k = lane; k < NX; k += 32) {
            C2 ca, cb;
            if (k <= nx) {
                ca = H[(long long)k * ny + ra];
                cb = hb ? H[(long long)k * ny + rb] : zero;
            } else {
                ca = conjg(H[(long long)(NX - k) * ny + ra]);
                cb = hb ? conjg(H[(long long)(NX - k) * ny + rb]) : zero;
            }
            C2 v;
            v.x = ca.x - cb.y;
            v.y = ca.y + cb.x;
            line[fft_pos(fx, k)] = v;
        }
        warp_fft(line, fx, tw, true);
        for (int i = lane; i < nx; i += 32) {
            const C2 v = line[fft_out(fx, i)];
            phi[(ra - ja0) * nx + i] = v.x * scale;
            if (hb) phi[(rb - ja0) * nx + i] = v.y * scale;
        }
        __syncwarp();
    }
    __syncthreads();
    field_cells<R>(C, P, pl, sg, phi, ja0, jt0, jt1);
}

// Register-FFT forms of the three convolution kernels (rfft.cuh) for NX = 8 Gx (rows, field) and
// NY = 8 Gy (columns); the arithmetic around the transforms is that of k_conv_rows, k_conv_cols and
// k_conv_field.  Lines that fall outside the plane (ok == false) still take part in the warp's
// transforms, on zeros, and store nothing.
template <class R, int G>
__global__ void __launch_bounds__(128) k_conv_rows_r(Collide C, int plane0) {
    using C2 = typename RealT<R>::C2;
    using RG = RfGeom<G>;
    constexpr int LPW = 32 / G;
    C2 *sm = (C2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, line = lane / G, l = lane & (G - 1);
    C2 *T = sm, *S = sm + RG::kTables + warp * RG::kWarpScratch;
    rf_tables<G>(T, (const C2 *)C.twr_x);  // before the wait (constant twiddles)
    pdl_wait();
    pdl_release();
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    if (plane_green(C, P) < 0) return;
    const int j0 = 2 * ((blockIdx.x * 4 + warp) * LPW + line), j1 = j0 + 1;
    const bool ok = j0 < ny;
    const double inv = ldexp(1.0, -P.fixed_bits);
    long long *q = C.qgrid + (long long)pl * nx * ny;
    constexpr bool kPrecision = sizeof(R) == 4;
    const long long *qo = q + (long long)P.other_delta * nx * ny;
    const bool diff = kPrecision && P.other_delta != 0;
    const long long sgn = P.self_first ? 1 : -1;
    const bool hyb = C.o.gaussian && C.hyb[P.task].mode;
    const HybRows hr(C, P, plane0, pl, hyb && ok, diff, inv, j0, j1);
    C2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        v[m].x = R(0);
        v[m].y = R(0);
        const int i = l + G * m;
        if (m < 4 && ok) {  // i < nx = 4 G
            long long qa = q[(long long)j0 * nx + i];
            if (diff) qa = sgn * (qa - qo[(long long)j0 * nx + i]);
            v[m].x = hyb ? (R)((double)qa * inv - hr.g0(i, sgn)) : (R)((double)qa * inv);
            if (!kPrecision && qa) q[(long long)j0 * nx + i] = 0;
            if (j1 < ny) {
                long long qb = q[(long long)j1 * nx + i];
                if (diff) qb = sgn * (qb - qo[(long long)j1 * nx + i]);
                v[m].y = hyb ? (R)((double)qb * inv - hr.g1(i, sgn)) : (R)((double)qb * inv);
                if (!kPrecision && qb) q[(long long)j1 * nx + i] = 0;
            }
        }
    }
    __syncthreads();  // tables ready (the rows' loads are already in flight)
    rf_fwd<G>(v, S, T);
    C2 *Sl = S + line * 8 * G;
#pragma unroll
    for (int r = 0; r < 8; ++r) Sl[rf_nat(rf_spec<G>(l, r))] = v[r];
    __syncwarp();
    if (!ok) return;
    C2 *H = (C2 *)C.spec + (long long)pl * (nx + 1) * ny;
    for (int k = l; k <= nx; k += G) {
        const C2 zk = Sl[rf_nat(k)], zm = conjg(Sl[rf_nat((NX - k) % NX)]);
        C2 A, B;
        A.x = R(0.5) * (zk.x + zm.x);
        A.y = R(0.5) * (zk.y + zm.y);
        const C2 D = csub(zk, zm);
        B.x = R(0.5) * D.y;
        B.y = R(-0.5) * D.x;
        store_pair(H + (long long)k * ny + j0, A, B);  // rows j0, j0 + 1 (j0 even, ny even)
    }
}

template <class R, int G>
__global__ void __launch_bounds__(128) k_conv_cols_r(Collide C, int plane0) {
    using C2 = typename RealT<R>::C2;
    using RG = RfGeom<G>;
    constexpr int LPW = 32 / G;
    C2 *sm = (C2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NY = 2 * ny;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, line = lane / G, l = lane & (G - 1);
    C2 *T = sm, *S = sm + RG::kTables + warp * RG::kWarpScratch;
    rf_tables<G>(T, (const C2 *)C.twr_y);  // before the wait (constant twiddles)
    pdl_wait();
    pdl_release();
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    const int slot = plane_green(C, P);
    if (slot < 0) return;
    const int k = (blockIdx.x * 4 + warp) * LPW + line;
    const bool ok = k <= nx;
    C2 *col = (C2 *)C.spec + ((long long)pl * (nx + 1) + k) * ny;
    C2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        v[m].x = R(0);
        v[m].y = R(0);
        if (m < 4 && ok) v[m] = col[l + G * m];  // rows j < ny = 4 G; the zero padding above
    }
    const double2 *g = C.ghat + (long long)slot * C.gstride + (long long)k * NY;
    double2 gpre[8];  // the Green spectrum's loads are in flight during the forward transform
#pragma unroll
    for (int r = 0; r < 8; ++r) gpre[r] = ok ? g[r * G + l] : make_double2(0.0, 0.0);
    __syncthreads();  // tables ready (the column's and the Green spectrum's loads are in flight)
    rf_fwd<G>(v, S, T);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const double2 gv = gpre[r];
        C2 gg;
        gg.x = (R)gv.x;
        gg.y = (R)gv.y;
        v[r] = cmul(v[r], gg);
    }
    rf_inv<G>(v, S, T);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 4; ++m) col[l + G * m] = v[m];
    }
}

// Tile of 12 rows: with the two-row halo, 16 rows = 8 lines, one per warp of 8 (G = 32).
constexpr int kFieldTileR = 12, kFieldWarpsR = 8;
template <class R, int G>
__global__ void __launch_bounds__(32 * kFieldWarpsR) k_conv_field_r(Collide C, int plane0) {
    using C2 = typename RealT<R>::C2;
    using RG = RfGeom<G>;
    constexpr int LPW = 32 / G;
    C2 *sm = (C2 *)g_smem;
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx, NY = 2 * ny;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, line = lane / G, l = lane & (G - 1);
    C2 *T = sm, *S = sm + RG::kTables + warp * RG::kWarpScratch;
    R *phi = (R *)(sm + RG::kTables + kFieldWarpsR * RG::kWarpScratch);  // (kFieldTileR + 4) rows x nx
    rf_tables<G>(T, (const C2 *)C.twr_x);  // before the wait (constant twiddles)
    pdl_wait();
    pdl_release();
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    if (plane_green(C, P) < 0) return;
    Grid sg;
    if (P.geom >= 0) sg = C.nodes[P.geom].sg;
    else sg = C.geom[P.task].sg;
    __syncthreads();
    const int jt0 = blockIdx.x * kFieldTileR;
    const int jt1 = min(jt0 + kFieldTileR, ny);
    const int ja0 = max(jt0 - 2, 0), ja1 = min(jt1 + 2, ny);
    const int nrows = ja1 - ja0;
    const C2 *H = (const C2 *)C.spec + (long long)pl * (nx + 1) * ny;
    const R scale = (R)(1.0 / ((double)NX * (double)NY));
    for (int rp0 = warp * LPW; 2 * rp0 < nrows; rp0 += kFieldWarpsR * LPW) {  // warp-uniform trip count
        const int ra = ja0 + 2 * (rp0 + line), rb = ra + 1;
        const bool ha = ra < ja1, hb = rb < ja1;
        C2 v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {  // x-frequency k; above nx from the conjugate of NX - k
            const int k = rf_spec<G>(l, r);
            const bool mir = k > nx;
            const C2 *h = H + (long long)(mir ? NX - k : k) * ny;
            C2 ca, cb;
            ca.x = ca.y = cb.x = cb.y = R(0);
            if (ha) load_pair(h + ra, ca, cb);  // rows ra, ra + 1 (ra even: 2-element aligned, ra + 1 < ny)
            if (!hb) cb.x = cb.y = R(0);
            if (mir) {
                ca.y = -ca.y;
                cb.y = -cb.y;
            }
            v[r].x = ca.x - cb.y;
            v[r].y = ca.y + cb.x;
        }
        rf_inv<G>(v, S, T);
        if (ha) {
#pragma unroll
            for (int m = 0; m < 4; ++m) {  // i = l + G m < nx
                phi[(ra - ja0) * nx + l + G * m] = v[m].x * scale;
                if (hb) phi[(rb - ja0) * nx + l + G * m] = v[m].y * scale;
            }
        }
    }
    __syncthreads();
    field_cells<R>(C, P, pl, sg, phi, ja0, jt0, jt1);
}

// ------------------------------------------------------------------ kick
// Weights and taps follow _pic_interpolate_kick (pic_cpu.jl:2596-2619), x-outer.
template <class R>
struct GridR {
    R x0, y0, w, h;
};
template <class R>
__device__ __forceinline__ GridR<R> grid_r(const Grid &g) {
    return GridR<R>{(R)g.x0, (R)g.y0, (R)g.w, (R)g.h};
}

template <class R, int METHOD>
struct Taps {
    static constexpr int NT = METHOD == 0 ? 2 : 3;
    int c0;          // first cell (x-outer, y-inner order follows from c0 + m + k*nx)
    R w[NT * NT];
    // hxi, hyi: reciprocals of the mesh spacing g.w/(nx-1), g.h/(ny-1), computed once per block.  The
    // reference divides by the spacing (pic_cpu.jl:2601-2602); in FP64 the product differs from that
    // quotient by at most 1.5 ulp of u, a ~1e-14 relative change of the interpolation weights.
    __device__ __forceinline__ Taps(const DevOptions &o, const GridR<R> &g, R hxi, R hyi, R x, R y) {
        const R u = (x - g.x0) * hxi, v = (y - g.y0) * hyi;
        int ix, iy; R wx[NT], wy[NT];
        if (METHOD == 0) { cic_weights(u, o.nx, ix, wx); cic_weights(v, o.ny, iy, wy); }
        else { tsc_weights(u, o.nx, ix, wx); tsc_weights(v, o.ny, iy, wy); }
        c0 = (iy - 1) * o.nx + (ix - 1);
#pragma unroll
        for (int m = 0; m < NT; ++m)
#pragma unroll
            for (int k = 0; k < NT; ++k) w[m * NT + k] = wx[m] * wy[k];
    }
    __device__ __forceinline__ int cell(int t, int nx) const { return c0 + (t / NT) + (t % NT) * nx; }
};

// Synchro-beam kick of every field particle of the front's tasks: drift in, interpolated kick,
// drift out (pic_cpu.jl:1005-1017, 1218-1243, 1248-1273; :node form 1448-1538).
// Blocks map to (task, chunk of `chunk` <= kKickChunk particles) through `blockmap`; the block reads its
// task and meshes once into shared memory, then each thread kicks chunk / blockDim particles.
constexpr int kKickThreads = 256;
constexpr int kKickChunk = 2048;
template <class R>
struct KickJob {
    GridR<R> gL, gR;
    R hxL, hyL, hxR, hyR;  // reciprocal spacings
    R c_src, hzi, zbias, ks;
    long long fld_start, fld_n, plane_off;
    int fld_beam, ok;
    int hyb;               // Gaussian-subtracted hybrid active for this task
    HybridTask H;
    int next_pair, next_task;  // luminosity box of the field slice's next pair (:node), or -1
    R next_sM;
};

template <class R>
struct Coord6 {
    R x, px, y, py, z, pz;
};
template <class R>
__device__ __forceinline__ Coord6<R> load_coord(const SoA &S, long long p) {
    // read once per kick: no L1 allocation, so L1 keeps the field cells the taps gather from (L2 as usual, where
    // the next front's deposits find the kicked slices)
    return Coord6<R>{ld_no_l1(col<R>(S, 0) + p), ld_no_l1(col<R>(S, 1) + p), ld_no_l1(col<R>(S, 2) + p),
                     ld_no_l1(col<R>(S, 3) + p), ld_no_l1(col<R>(S, 4) + p), ld_no_l1(col<R>(S, 5) + p)};
}

// HYB: the Gaussian-subtracted hybrid's add-back (FP64 Bassetti-Erskine in both forms) is compiled in, a
// separate instantiation so the plain kernels keep their register budget.
template <class R, int METHOD, bool HYB>
__device__ __forceinline__ void kick_particle(const Collide &C, const KickJob<R> &J, long long p, const Coord6<R> &q,
                                              R &xo, R &pxo, R &yo, R &pyo) {
    using FC = typename RealT<R>::FC;
    constexpr int CV = RealT<R>::kCellVec;
    constexpr int NT2 = Taps<R, METHOD>::NT * Taps<R, METHOD>::NT;
    // Precision form: the planes hold exact charge differences (see k_conv_rows), so the kick uses the
    // algebraically equal difference forms below; the plain form keeps the reference's expressions.
    constexpr bool kPrecision = sizeof(R) == 4;
    const DevOptions &o = C.o;
    const long long pc = (long long)o.nx * o.ny;
    const FC *base = (const FC *)C.fields + J.plane_off * CV * pc;
    const SoA S = C.beam[J.fld_beam];
    R x = q.x, px = q.px, y = q.y, py = q.py;
    const R z = q.z;
    R pz = q.pz;
    const bool lk = o.longitudinal_kick != 0;
    const R s = R(0.5) * (z - J.c_src);
    // Precision form: the drift and kick increments of x, y and pz are summed in registers and added
    // to the stored coordinate once, so each FP32 coordinate is rounded once per kick (the pz drift
    // terms, ~1e-7, dwarf the pz kick, ~1e-9, and three roundings of pz would cost ~3 ulps of it).
    const R px0 = px, py0 = py;
    R dpz = R(0);
    x += s * px;
    y += s * py;
    if (kPrecision) {
        if (lk) dpz = -(R(0.25) * (px * px + py * py));
    } else if (lk) {
        pz -= R(0.25) * (px * px + py * py);
    }
    const R zL = jclamp(-z * J.hzi + J.zbias, R(0), R(1));
    const R zR = R(1) - zL;
    const R ks = J.ks;
    // :sigma and :source_slice field meshes need not cover every field particle (pic_cpu.jl:1060-1090)
    if (!o.node && (o.grid_extent || o.shared_grid)) {
        const GridR<R> &gF = J.gL;
        if (!(isfinite(x) && gF.x0 <= x && x <= gF.x0 + gF.w && isfinite(y) && gF.y0 <= y && y <= gF.y0 + gF.h))
            atomicAdd((unsigned long long *)&C.status->dropped, 1ull);
    }
    if (o.node) {
        // L on gL, R on gR, Z (the R drift deposited on gL) on gL; with zL = 1, zR = 0 the reference's
        // single-plane interpolations reduce exactly to w * E (pic_cpu.jl:1517-1528).
        const GridR<R> &gL = J.gL, &gR = J.gR;
        const FC *FL = base, *FR = base + CV * pc;  // the L plane's w word holds phi_Z (k_conv_field)
        if (!(isfinite(x) && gL.x0 <= x && x <= gL.x0 + gL.w && isfinite(y) && gL.y0 <= y && y <= gL.y0 + gL.h))
            atomicAdd((unsigned long long *)&C.status->dropped, 1ull);
        R KxL = 0, KyL = 0, Kz = 0, KxR = 0, KyR = 0;
        {
            const Taps<R, METHOD> tp(o, gL, J.hxL, J.hyL, x, y);
#pragma unroll
            for (int t = 0; t < NT2; ++t) {
                R phl, exl, eyl, phz;
                load_cell4(FL, tp.cell(t, o.nx), phl, exl, eyl, phz);
                KxL += tp.w[t] * exl;
                KyL += tp.w[t] * eyl;
                if (kPrecision) Kz += tp.w[t] * phz;  // the Z plane holds phi_L - phi_Z
                else Kz += tp.w[t] * (phl - phz);
            }
        }
        {
            const Taps<R, METHOD> tp(o, gR, J.hxR, J.hyR, x, y);
            if constexpr (METHOD == 0) {
                // pair cells: row iy - 1 holds taps (0, 0) and (1, 0), row iy taps (0, 1) and (1, 1); summed in
                // the x-outer tap order t = 0..3 = (0, 0), (0, 1), (1, 0), (1, 1)
                R ex00, ey00, ex10, ey10, ex01, ey01, ex11, ey11;
                load_field_pair(FR, tp.c0, ex00, ey00, ex10, ey10);
                load_field_pair(FR, tp.c0 + o.nx, ex01, ey01, ex11, ey11);
                KxR += tp.w[0] * ex00; KyR += tp.w[0] * ey00;
                KxR += tp.w[1] * ex01; KyR += tp.w[1] * ey01;
                KxR += tp.w[2] * ex10; KyR += tp.w[2] * ey10;
                KxR += tp.w[3] * ex11; KyR += tp.w[3] * ey11;
            } else {
#pragma unroll
                for (int t = 0; t < NT2; ++t) {
                    R ex, ey;
                    load_field(FR, tp.cell(t, o.nx), ex, ey);
                    KxR += tp.w[t] * ex;
                    KyR += tp.w[t] * ey;
                }
            }
        }
        px += ks * (zL * KxL + zR * KxR);
        py += ks * (zL * KyL + zR * KyR);
        if (lk) { if (kPrecision) dpz += ks * Kz * J.hzi; else pz += ks * Kz * J.hzi; }
    } else if (o.quadratic) {
        // three nodes L, R, M (pic_cpu.jl:2648-2680) at t = 1 - zL
        const FC *FL = base, *FR = base + CV * pc, *FM = base + 2 * CV * pc;
        const R t = R(1) - zL;
        const R t2 = t * t;
        const R aL = R(2) * t2 - R(3) * t + R(1), aM = R(4) * t - R(4) * t2, aR = R(2) * t2 - t;
        const R bL = R(3) - R(4) * t, bM = R(8) * t - R(4), bR = R(1) - R(4) * t;
        const Taps<R, METHOD> tp(o, J.gL, J.hxL, J.hyL, x, y);
        R Kx = 0, Ky = 0, Kz = 0;
#pragma unroll
        for (int q = 0; q < NT2; ++q) {
            R pl, el, fl, pm, em, fm, pr, er, fr;
            load_cell(FL, tp.cell(q, o.nx), pl, el, fl);
            load_cell(FM, tp.cell(q, o.nx), pm, em, fm);
            load_cell(FR, tp.cell(q, o.nx), pr, er, fr);
            if (kPrecision) {  // L, R planes hold L - M, R - M; aL + aM + aR = 1, bL + bM + bR = 0
                Kx += tp.w[q] * (em + aL * el + aR * er);
                Ky += tp.w[q] * (fm + aL * fl + aR * fr);
                Kz += tp.w[q] * (bL * pl + bR * pr);
            } else {
                Kx += tp.w[q] * (aL * el + aM * em + aR * er);
                Ky += tp.w[q] * (aL * fl + aM * fm + aR * fr);
                Kz += tp.w[q] * (bL * pl + bM * pm + bR * pr);
            }
        }
        px += ks * Kx;
        py += ks * Ky;
        if (lk) { if (kPrecision) dpz += ks * Kz * J.hzi; else pz += ks * Kz * J.hzi; }
    } else {
        const FC *FL = base, *FR = base + CV * pc;
        const Taps<R, METHOD> tp(o, J.gL, J.hxL, J.hyL, x, y);
        R Kx = 0, Ky = 0, Kz = 0;
        // (hybrid: K is the field of the residual charge; the analytic Gaussian kick is added below)
#pragma unroll
        for (int q = 0; q < NT2; ++q) {
            R pl, el, fl, pr, er, fr;
            load_cell(FL, tp.cell(q, o.nx), pl, el, fl);
            load_cell(FR, tp.cell(q, o.nx), pr, er, fr);
            if (kPrecision) {  // the R plane holds L - R
                Kx += tp.w[q] * (el - zR * er);
                Ky += tp.w[q] * (fl - zR * fr);
                Kz += tp.w[q] * pr;
            } else {
                Kx += tp.w[q] * (zL * el + zR * er);
                Ky += tp.w[q] * (zL * fl + zR * fr);
                Kz += tp.w[q] * (pl - pr);
            }
        }
        if (HYB && J.hyb == 2) {
            // Rotated add-back of the tilted Gaussian through _cp_covariance_kick at both boundaries, blended in z
            // (gaussian_pic.jl:837-854)
            const HybridTask &H = J.H;
            const double kbb_eff = (double)ks * H.half_ns;
            GMoments M{};
            M.a0 = H.cov[0]; M.b0 = H.cov[1]; M.d0 = H.cov[2]; M.bxx = H.cov[3]; M.bxpy = H.cov[4];
            M.bypx = H.cov[5]; M.bypy = H.cov[6]; M.qxx = H.cov[7]; M.qxy = H.cov[8]; M.qyy = H.cov[9];
            double pxL = 0, pyL = 0, pzL = 0, pxR = 0, pyR = 0, pzR = 0, dens;
            coupled_kick(M, kbb_eff, -H.s[0], (double)x - H.mux[0], (double)y - H.muy[0], pxL, pyL, pzL, dens);
            coupled_kick(M, kbb_eff, -H.s[1], (double)x - H.mux[1], (double)y - H.muy[1], pxR, pyR, pzR, dens);
            const double dpxa = (double)zL * pxL + (double)zR * pxR;
            const double dpya = (double)zL * pyL + (double)zR * pyR;
            px += (R)((double)ks * (double)Kx + dpxa);
            py += (R)((double)ks * (double)Ky + dpya);
            if (lk) {
                if (kPrecision) {
                    dpz += (R)((double)ks * (double)Kz * (double)J.hzi + ((double)zL * pzL + (double)zR * pzR) +
                               0.5 * (dpxa * H.mpx + dpya * H.mpy));
                } else {
                    pz += ks * Kz * J.hzi;
                    pz += (R)((double)zL * pzL + (double)zR * pzR);
                    pz += (R)(0.5 * (dpxa * H.mpx + dpya * H.mpy));
                }
            }
        } else if (HYB && J.hyb) {
            // Analytic add-back of the subtracted Gaussian (gaussian_pic.jl:851-884): half the slice population
            // times the Bassetti-Erskine kick at both boundaries, blended in z, and its longitudinal terms.
            const HybridTask &H = J.H;
            const double kbb_eff = (double)ks * H.half_ns;
            double bLx, bLy, HxL = 0, HyL = 0, bRx, bRy, HxR = 0, HyR = 0;
            be_response(lk ? kbb_eff : 0.0, H.sigx[0], H.sigy[0], (double)x - H.mux[0], (double)y - H.muy[0], bLx, bLy,
                        HxL, HyL);
            be_response(lk ? kbb_eff : 0.0, H.sigx[1], H.sigy[1], (double)x - H.mux[1], (double)y - H.muy[1], bRx, bRy,
                        HxR, HyR);
            const double Kxa = H.half_ns * ((double)zL * bLx + (double)zR * bRx);
            const double Kya = H.half_ns * ((double)zL * bLy + (double)zR * bRy);
            const double dpxa = (double)ks * Kxa, dpya = (double)ks * Kya;
            px += (R)((double)ks * (double)Kx + dpxa);
            py += (R)((double)ks * (double)Ky + dpya);
            if (lk) {
                const double covL = (HxL * H.rx[0] + HyL * H.ry[0]) / 4.0;
                const double covR = (HxR * H.rx[1] + HyR * H.ry[1]) / 4.0;
                if (kPrecision) {  // summed in FP64, one rounding into the pz increment
                    dpz += (R)((double)ks * (double)Kz * (double)J.hzi + ((double)zL * covL + (double)zR * covR) +
                               0.5 * (dpxa * H.mpx + dpya * H.mpy));
                } else {
                    pz += ks * Kz * J.hzi;
                    pz += (R)((double)zL * covL + (double)zR * covR);
                    pz += (R)(0.5 * (dpxa * H.mpx + dpya * H.mpy));
                }
            }
        } else {
            px += ks * Kx;
            py += ks * Ky;
            if (lk) { if (kPrecision) dpz += ks * Kz * J.hzi; else pz += ks * Kz * J.hzi; }
        }
    }
    const R s2 = R(0.5) * (J.c_src - z);
    if (kPrecision) {
        x = q.x + (s * px0 + s2 * px);
        y = q.y + (s * py0 + s2 * py);
        if (lk) pz = q.pz + (dpz + R(0.25) * (px * px + py * py));
    } else {
        x += s2 * px;
        y += s2 * py;
        if (lk) pz += R(0.25) * (px * px + py * py);
    }
    col<R>(S, 0)[p] = x; col<R>(S, 1)[p] = px; col<R>(S, 2)[p] = y; col<R>(S, 3)[p] = py; col<R>(S, 5)[p] = pz;
    xo = x; pxo = px; yo = y; pyo = py;
}

template <class R, int METHOD, bool HYB>
__global__ void __launch_bounds__(kKickThreads, sizeof(R) == 8 ? 2 : 4)
    k_kick(Collide C, int plane0_front, const int2 *blockmap, int chunk) {
    pdl_wait();
    pdl_release();
    __shared__ KickJob<R> J;
    const int2 bm0 = blockmap[blockIdx.x];
    if (bm0.x < 0) return;  // a spare entry of a collide that may be captured (block-uniform)
    if (threadIdx.x == 0) {
        const int2 bm = bm0;
        const Task &T = C.tasks[bm.x];
        J.ok = 1;
        Grid gL, gR;
        if (C.o.node) {
            J.ok = C.nodes[T.nodeL].valid && C.nodes[T.nodeR].valid;
            gL = C.nodes[T.nodeL].fg;
            gR = C.nodes[T.nodeR].fg;
        } else {
            const TaskGeom &G = C.geom[bm.x];
            J.ok = G.green >= 0;
            gL = G.fg;
            gR = G.fg;
        }
        J.hyb = 0;
        if (C.o.gaussian && J.ok) {
            J.H = C.hyb[bm.x];
            J.hyb = J.H.mode;
        }
        J.gL = grid_r<R>(gL);
        J.gR = grid_r<R>(gR);
        J.hxL = (R)(1.0 / (gL.w / (double)(C.o.nx - 1))); J.hyL = (R)(1.0 / (gL.h / (double)(C.o.ny - 1)));
        J.hxR = (R)(1.0 / (gR.w / (double)(C.o.nx - 1))); J.hyR = (R)(1.0 / (gR.h / (double)(C.o.ny - 1)));
        J.c_src = (R)T.c_src; J.hzi = (R)T.hzi; J.zbias = (R)T.zbias; J.ks = (R)T.ks;
        J.fld_start = T.fld_start + bm.y;
        const long long rest = T.fld_n - (long long)bm.y;
        J.fld_n = rest < (long long)chunk ? rest : (long long)chunk;
        J.plane_off = T.plane0 - plane0_front;
        J.fld_beam = T.fld_beam;
        J.next_pair = C.o.node ? T.next_pair : -1;
        J.next_task = T.next_task;
        J.next_sM = (R)T.next_sM;
    }
    __syncthreads();
    if (!J.ok) return;
    // The next particle's coordinates are loaded before the current one is kicked, so two
    // particles' HBM loads are in flight per thread.  In :node mode with luminosity the kicked slice's
    // virtual positions for its next pair are reduced on the way (pic_cpu.jl:1279-1287).
    const SoA S = C.beam[J.fld_beam];
    const bool lum_next = J.next_pair >= 0;
    R mnx = R(INFINITY), mxx = R(-INFINITY), mny = R(INFINITY), mxy = R(-INFINITY);
    bool nan = false;
    int k = threadIdx.x;
    if (k < J.fld_n) {
        Coord6<R> cur = load_coord<R>(S, J.fld_start + k);
        for (;;) {
            const int kn = k + kKickThreads;
            Coord6<R> nxt;
            if (kn < J.fld_n) nxt = load_coord<R>(S, J.fld_start + kn);
            R x, px, y, py;
            kick_particle<R, METHOD, HYB>(C, J, J.fld_start + k, cur, x, px, y, py);
            if (lum_next) {
                const R vx = x + px * J.next_sM, vy = y + py * J.next_sM;
                nan |= (vx != vx) | (vy != vy);
                mnx = fmin(mnx, vx); mxx = fmax(mxx, vx);
                mny = fmin(mny, vy); mxy = fmax(mxy, vy);
            }
            if (kn >= J.fld_n) break;
            cur = nxt;
            k = kn;
        }
    }
    if (lum_next) reduce_lum_box(C, mnx, mxx, mny, mxy, nan, J.next_pair, J.next_task);
}

// ------------------------------------------------------------------ node meshes
// Per-slice boxes of the turn-start state (pic_cpu.jl:1317-1358), both beams and both roles in one
// pass.  Row (beam bm, slice sl) has nref = 2*o + 1 drift references, o = the other beam's slice count:
//   k <  o + 1: source role, the slice drifted to node k, x + px*d with d = 0.5*(c_sl - boundary_k);
//   k >= o + 1: field role, the slice drifted to the collision point of the other beam's slice
//               i = k - (o + 1), x + sh*px with sh = 0.5*(z - c_i).
// ref[bm][sl*nref + k] holds d or c_i.  Source boxes go to sbox[bm] ([sl][node][4]), field boxes to
// fbox[bm] ([field slice][source slice][4]), each ordered (xmin, xmax, ymin, ymax).
// A block stages a tile of particles in shared memory once; its 16-lane rows of threads each take one
// reference (4 groups of 16 references per block), so every particle is read from HBM once per turn.
constexpr int kBoxTile = 512, kBoxLanes = 16, kBoxGroups = 4, kBoxThreads = 256;
struct NodeBoxArgs {
    const void *x[2], *px[2], *y[2], *py[2], *z[2];  // slice-sorted coordinates, element type R
    const SliceInfo *info[2];                         // the device slice tables (slice starts and counts)
    const double *ref[2];
    unsigned long long *sbox[2], *fbox[2];
    int *nanf;
    int ns[2];
    long long chunk;  // particles per block
};

template <class R>
__global__ void __launch_bounds__(kBoxThreads) k_node_boxes(NodeBoxArgs A) {
    pdl_wait();
    pdl_release();
    __shared__ R tile[5][kBoxTile];
    __shared__ unsigned long long red[kBoxThreads / 32][kBoxLanes][4];
    const int bm = (int)blockIdx.y < A.ns[0] ? 0 : 1;
    const int sl = bm ? (int)blockIdx.y - A.ns[0] : (int)blockIdx.y;
    const int o = A.ns[1 - bm], nb = o + 1, nref = nb + o;
    const int g0 = blockIdx.z * kBoxGroups;
    const long long n = A.info[bm]->count[sl], k0 = (long long)blockIdx.x * A.chunk;
    if (k0 >= n || g0 * kBoxLanes >= nref) return;  // block-uniform
    const long long k1 = min(n, k0 + A.chunk), st = A.info[bm]->start[sl];
    const int ng = min(kBoxGroups, (nref - g0 * kBoxLanes + kBoxLanes - 1) / kBoxLanes);
    const R *X = (const R *)A.x[bm], *PX = (const R *)A.px[bm], *Y = (const R *)A.y[bm],
            *PY = (const R *)A.py[bm], *Z = (const R *)A.z[bm];
    const int lane16 = threadIdx.x & (kBoxLanes - 1), prow = threadIdx.x / kBoxLanes;
    constexpr int kRows = kBoxThreads / kBoxLanes;
    R sref[kBoxGroups], mnx[kBoxGroups], mxx[kBoxGroups], mny[kBoxGroups], mxy[kBoxGroups];
    bool fld[kBoxGroups], live[kBoxGroups];
#pragma unroll
    for (int g = 0; g < kBoxGroups; ++g) {
        const int k = (g0 + g) * kBoxLanes + lane16;
        live[g] = g < ng && k < nref;
        fld[g] = k >= nb;
        sref[g] = live[g] ? (R)A.ref[bm][(long long)sl * nref + k] : R(0);
        mnx[g] = mny[g] = R(INFINITY);
        mxx[g] = mxy[g] = R(-INFINITY);
    }
    bool nan = false;
    for (long long t0 = k0; t0 < k1; t0 += kBoxTile) {
        const int tn = (int)min((long long)kBoxTile, k1 - t0);
        __syncthreads();  // the previous tile is consumed
        for (int j = threadIdx.x; j < tn; j += kBoxThreads) {
            const long long p = st + t0 + j;
            tile[0][j] = X[p]; tile[1][j] = PX[p]; tile[2][j] = Y[p]; tile[3][j] = PY[p]; tile[4][j] = Z[p];
        }
        __syncthreads();
        // the rows for a block-uniform count of live reference groups, so groups past it issue nothing
        auto rows = [&](auto groups) {
            constexpr int NG = decltype(groups)::value;
            for (int j = prow; j < tn; j += kRows) {
                const R x = tile[0][j], px = tile[1][j], y = tile[2][j], py = tile[3][j], z = tile[4][j];
#pragma unroll
                for (int g = 0; g < NG; ++g) {
                    if (live[g]) {
                        const R s = fld[g] ? R(0.5) * (z - sref[g]) : sref[g];
                        const R xv = x + s * px, yv = y + s * py;
                        nan |= (xv != xv) | (yv != yv);
                        mnx[g] = fmin(mnx[g], xv); mxx[g] = fmax(mxx[g], xv);
                        mny[g] = fmin(mny[g], yv); mxy[g] = fmax(mxy[g], yv);
                    }
                }
            }
        };
        static_assert(kBoxGroups == 4, "the dispatch below covers 1..4 groups");
        switch (ng) {
        case 1: rows(std::integral_constant<int, 1>{}); break;
        case 2: rows(std::integral_constant<int, 2>{}); break;
        case 3: rows(std::integral_constant<int, 3>{}); break;
        default: rows(std::integral_constant<int, 4>{}); break;
        }
    }
    if (__syncthreads_or(nan) && threadIdx.x == 0) atomicOr(A.nanf, 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int g = 0; g < ng; ++g) {
        // lanes l and l + 16 of a warp hold the same reference
        unsigned long long v[4] = {mnx[g] == R(INFINITY) ? kOrdMinInit : ord_encode((double)mnx[g]),
                                   mxx[g] == R(-INFINITY) ? kOrdMaxInit : ord_encode((double)mxx[g]),
                                   mny[g] == R(INFINITY) ? kOrdMinInit : ord_encode((double)mny[g]),
                                   mxy[g] == R(-INFINITY) ? kOrdMaxInit : ord_encode((double)mxy[g])};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, v[q], kBoxLanes);
            v[q] = (q & 1) ? max(v[q], w) : min(v[q], w);
        }
        if (lane < kBoxLanes) {
#pragma unroll
            for (int q = 0; q < 4; ++q) red[warp][lane][q] = v[q];
        }
        __syncthreads();
        if (threadIdx.x < kBoxLanes * 4) {
            const int r = threadIdx.x >> 2, q = threadIdx.x & 3;
            unsigned long long a = red[0][r][q];
            for (int w = 1; w < kBoxThreads / 32; ++w) a = (q & 1) ? max(a, red[w][r][q]) : min(a, red[w][r][q]);
            const int k = (g0 + g) * kBoxLanes + r;
            if (k < nref) {
                unsigned long long *dst = k < nb ? A.sbox[bm] + ((long long)sl * nb + k) * 4 + q
                                                 : A.fbox[bm] + ((long long)sl * o + (k - nb)) * 4 + q;
                if (q & 1) atomicMax(dst, a); else atomicMin(dst, a);
            }
        }
        __syncthreads();
    }
}

// Node meshes of one direction (pic_cpu.jl:1359-1381): mesh (i, b) from the source drift boxes
// of nodes b and b+1 and the field boxes of the slices adjacent to node b.  sbox: [i][b][4],
// fbox: [field slice][i][4].  Meshes are written at meshes[i*nb + b-1].
// A non-finite coordinate seen by k_node_boxes (*nanf) invalidates every mesh, so no later kernel of the
// collide touches the beams, and is reported through the status with the smallest key (task 0, code 0,
// role 4 = node-mesh build): the reference fails at the turn-start mesh build, before any pair.
__global__ void k_node_plan(DevOptions o, const unsigned long long *sbox, const unsigned long long *fbox, int ns_src,
                            int nb, const long long *src_count, const int *nanf, NodeMesh *meshes, DevStatus *st) {
    pdl_wait();
    pdl_release();
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= ns_src * nb) return;
    const int i = id / nb, b = id % nb + 1;  // b is 1-based
    NodeMesh &M = meshes[id];
    M.valid = 0;
    if (*nanf) {
        if (id == 0) atomicMin(&st->first_bad, 4ull);
        return;
    }
    if (src_count[i] == 0) return;
    const int ns = nb - 1;
    const int bn = min(b + 1, nb);
    auto SB = [&](int node, int q) { return ord_decode(sbox[((long long)i * nb + node - 1) * 4 + q]); };
    auto FB = [&](int sl, int q) { return ord_decode(fbox[((long long)(sl - 1) * ns_src + i) * 4 + q]); };
    double sxmin = jmin(SB(b, 0), SB(bn, 0)), sxmax = jmax(SB(b, 1), SB(bn, 1));
    double symin = jmin(SB(b, 2), SB(bn, 2)), symax = jmax(SB(b, 3), SB(bn, 3));
    double fxmin = INFINITY, fxmax = -INFINITY, fymin = INFINITY, fymax = -INFINITY;
    for (int adj = b - 1; adj <= b; ++adj) {
        if (!(1 <= adj && adj <= ns)) continue;
        double lo = FB(adj, 0);
        if (!isfinite(lo)) continue;  // empty field slice: its sentinel decodes to NaN
        fxmin = jmin(fxmin, lo); fxmax = jmax(fxmax, FB(adj, 1));
        fymin = jmin(fymin, FB(adj, 2)); fymax = jmax(fymax, FB(adj, 3));
    }
    if (!isfinite(fxmin)) return;
    Grid sg, fg;
    if (!interaction_grids(o, sxmin, sxmax, symin, symax, fxmin, fxmax, fymin, fymax, sg, fg)) {
        atomicMin(&st->first_bad, (3ull << 8));
        return;
    }
    M.sg = sg;
    M.fg = fg;
    M.valid = 1;
}

}  // namespace octo
