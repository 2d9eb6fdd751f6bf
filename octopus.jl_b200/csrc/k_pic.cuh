// PIC wavefront kernels.  Each launch covers every directed interaction (task), deposit plane
// or pair of one collision-time wavefront (slicing.jl:601-647), so the S1*S2 pairs of a turn run
// as 2S-1 batched launch sequences instead of one launch chain per pair.
#pragma once
#include "fft.cuh"
#include "geometry.cuh"
#include "octo_internal.cuh"

namespace octo {

struct SoA {
    double *c[6];  // x, px, y, py, z, pz (slice-sorted)
};

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
    double2 *spec;             // spectral scratch: plane-in-front * (nx+1)*ny
    double *fields;            // plane-in-front * 3 * nx*ny  (phi, Ex, Ey)
    long long *lq;             // luminosity grids: (pair-in-front*2 + side) * (lnx+1)*(lny+1)
    double *lum_parts;         // [pair position]
    const double2 *tw_x, *tw_y;  // twiddles for 2nx and 2ny
    SoA beam[2];
    double klum;
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
// grid: (blocks per side, 2 * pairs in front).
__global__ void __launch_bounds__(256) k_pair_bounds(Collide C, int task0) {
    const int q = blockIdx.y >> 1, side = blockIdx.y & 1;
    const int t1 = task0 + 2 * q, t2 = t1 + 1;
    const Task &A = C.tasks[t1];  // dir 1: source beam-1 slice i, field beam-2 slice j
    const Task &B = C.tasks[t2];  // dir 2: source beam-2 slice j, field beam-1 slice i
    const Task &src_task = side == 0 ? A : B;  // this slice is the source of src_task
    const Task &fld_task = side == 0 ? B : A;  // ... and the field of fld_task
    const SoA S = C.beam[side];
    const long long st = src_task.src_start, n = src_task.src_n;
    const double sL = src_task.sL, sR = src_task.sR, sM = src_task.sM, cf = fld_task.c_src;
    unsigned long long mn[6], mx[6];
    for (int k = 0; k < 6; ++k) { mn[k] = kOrdMinInit; mx[k] = kOrdMaxInit; }
    bool nan_s = false, nan_f = false, nan_l = false;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        double x = S.c[0][st + k], px = S.c[1][st + k], y = S.c[2][st + k], py = S.c[3][st + k], z = S.c[4][st + k];
        double v[6];
        v[0] = x + px * sL;
        v[1] = x + px * sR;
        v[2] = y + py * sL;
        v[3] = y + py * sR;
        double s = 0.5 * (z - cf);
        v[4] = x + s * px;
        v[5] = y + s * py;
        double lx = x + px * sM, ly = y + py * sM;
        nan_s |= (v[0] != v[0]) | (v[1] != v[1]) | (v[2] != v[2]) | (v[3] != v[3]);
        nan_f |= (v[4] != v[4]) | (v[5] != v[5]);
        nan_l |= (lx != lx) | (ly != ly);
        unsigned long long e;
        // source x (0), source y (1), field x (2), field y (3), lum x (4), lum y (5)
        e = ord_encode(v[0]); mn[0] = min(mn[0], e); mx[0] = max(mx[0], e);
        e = ord_encode(v[1]); mn[0] = min(mn[0], e); mx[0] = max(mx[0], e);
        e = ord_encode(v[2]); mn[1] = min(mn[1], e); mx[1] = max(mx[1], e);
        e = ord_encode(v[3]); mn[1] = min(mn[1], e); mx[1] = max(mx[1], e);
        e = ord_encode(v[4]); mn[2] = min(mn[2], e); mx[2] = max(mx[2], e);
        e = ord_encode(v[5]); mn[3] = min(mn[3], e); mx[3] = max(mx[3], e);
        e = ord_encode(lx); mn[4] = min(mn[4], e); mx[4] = max(mx[4], e);
        e = ord_encode(ly); mn[5] = min(mn[5], e); mx[5] = max(mx[5], e);
    }
    __shared__ unsigned long long red[8][12];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = 0; k < 6; ++k) {
        unsigned long long a = shfl_min_u64(mn[k]), b = shfl_max_u64(mx[k]);
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

__device__ inline void record_error(DevStatus *st, int task, int code, int role) {
    unsigned long long key = ((unsigned long long)task << 16) | ((unsigned long long)code << 8) | (unsigned)role;
    atomicMin(&st->first_bad, key);
}

// Grid geometry and Green-cache decision per task (pic_cpu.jl:954-1064, 1729-1821).
__global__ void k_plan(Collide C, int task0, int ntasks, int slot_scratch0) {
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
    int nf = C.nanflag[t];
    if ((nf & 1) || !(isfinite(sxmin) && isfinite(sxmax) && isfinite(symin) && isfinite(symax))) {
        record_error(C.status, t, 1, 1);
        return;
    }
    if ((nf & 2) || !(isfinite(fxmin) && isfinite(fxmax) && isfinite(fymin) && isfinite(fymax))) {
        record_error(C.status, t, 1, 2);
        return;
    }
    Grid sg, fg;
    if (!interaction_grids(C.o, sxmin, sxmax, symin, symax, fxmin, fxmax, fymin, fymax, sg, fg)) {
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

// Luminosity mesh per pair (pic_cpu.jl:2706-2723).
__global__ void k_lum_plan(Collide C, int lj0, int npairs, int task0) {
    int ql = blockIdx.x * blockDim.x + threadIdx.x;
    if (ql >= npairs) return;
    const LumJob &J = C.lumjobs[lj0 + ql];
    LumGeom &L = C.lumgeom[J.pair];
    L.ok = 0;
    const unsigned long long *b = C.lumb + (long long)J.pair * 4;
    double xmin = ord_decode(b[0]), xmax = ord_decode(b[1]), ymin = ord_decode(b[2]), ymax = ord_decode(b[3]);
    int t1 = task0 + 2 * ql;
    if ((C.nanflag[t1] & 4) || (C.nanflag[t1 + 1] & 4)) {
        record_error(C.status, t1, 1, 1);
        return;
    }
    double width, height;
    if (!resolve_extent(C.o, xmax - xmin, ymax - ymin, width, height)) {
        record_error(C.status, t1, 3, 0);
        return;
    }
    int nx = C.o.lnx, ny = C.o.lny;
    double tx = width / ((double)nx - 1.1);
    double ty = height / ((double)ny - 1.1);
    width += 0.1 * tx;
    height += 0.1 * ty;
    xmin -= 0.05 * tx;
    ymin -= 0.05 * ty;
    L.x0 = xmin;
    L.y0 = ymin;
    L.hx = width / (double)(nx - 1);
    L.hy = height / (double)(ny - 1);
    L.ok = 1;
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

// Green table rows evaluated in registers and transformed along x: two table rows per warp as one
// complex line, written as the nx+1 non-redundant x-frequencies of each row into the slot.
// mode 0: blockIdx.y = task of the front (only tasks that rebuild); mode 1: blockIdx.y = node mesh.
__global__ void __launch_bounds__(128) k_green_rows(Collide C, int mode, int base, int node_slot0) {
    extern __shared__ double2 sm[];
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx, NY = 2 * ny;
    int lgx = 31 - __clz(NX);
    double2 *tw = sm;
    double2 *line = sm + NX / 2 + (threadIdx.x >> 5) * NX;
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
    __syncthreads();
    const double hx = sg.w / (double)(nx - 1), hy = sg.h / (double)(ny - 1);
    const double dx0 = fg.x0 - sg.x0, dy0 = fg.y0 - sg.y0;
    const int lane = threadIdx.x & 31;
    const int pair = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (2 * pair >= NY) return;
    const int j0 = 2 * pair, j1 = j0 + 1;
    for (int i = lane; i < NX; i += 32) {
        double a = green_value(C.o.green_type, i, j0, nx, ny, dx0, dy0, hx, hy);
        double b = green_value(C.o.green_type, i, j1, nx, ny, dx0, dy0, hx, hy);
        line[bitrev(i, lgx)] = make_double2(a, b);
    }
    warp_fft_passes(line, NX, tw, false);
    double2 *out = C.ghat + (long long)slot * C.gstride;
    for (int k = lane; k <= nx; k += 32) {
        double2 zk = line[k], zm = conjg(line[(NX - k) & (NX - 1)]);
        double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y + zm.y));
        double2 D = csub(zk, zm);
        double2 Bv = make_double2(0.5 * D.y, -0.5 * D.x);
        out[(long long)k * NY + j0] = A;
        out[(long long)k * NY + j1] = Bv;
    }
}

// Column transforms of the Green slots (length 2ny, in place, natural-order output).
__global__ void __launch_bounds__(128) k_green_cols(Collide C, int mode, int base, int node_slot0) {
    extern __shared__ double2 sm[];
    const int nx = C.o.nx, ny = C.o.ny, NY = 2 * ny;
    int lgy = 31 - __clz(NY);
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
    for (int j = lane; j < NY; j += 32) line[bitrev(j, lgy)] = col[j];
    warp_fft_passes(line, NY, tw, false);
    for (int j = lane; j < NY; j += 32) col[j] = line[j];
}

// ------------------------------------------------------------------ deposition
// Fixed-point deposit of a particle range into an int64 grid (ld = nw) with CIC/TSC weights:
// (pic_cpu.jl:2129-2146).  Taps are round(w * 2^bits); zero taps are skipped.
template <int METHOD>
__device__ __forceinline__ void deposit_taps(double u, double v, int nw, int nh, double scale, long long *grid, int ld,
                                             bool shared_grid) {
    if (METHOD == 0) {
        int ix, iy; double wx[2], wy[2];
        cic_weights(u, nw, ix, wx);
        cic_weights(v, nh, iy, wy);
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                long long qv = __double2ll_rn(wx[m] * wy[k] * scale);
                if (qv) atomicAdd((unsigned long long *)&grid[(iy + k - 1) * ld + (ix + m - 1)], (unsigned long long)qv);
            }
    } else {
        int ix, iy; double wx[3], wy[3];
        tsc_weights(u, nw, ix, wx);
        tsc_weights(v, nh, iy, wy);
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                long long qv = __double2ll_rn(wx[m] * wy[k] * scale);
                if (qv) atomicAdd((unsigned long long *)&grid[(iy + k - 1) * ld + (ix + m - 1)], (unsigned long long)qv);
            }
    }
}

// Field-solve planes of a front.  grid: (blocks per plane, planes in front); dynamic shared memory
// holds a private int64 copy of the nx*ny grid when it fits (use_smem), merged with global atomics.
template <int METHOD>
__global__ void __launch_bounds__(512) k_deposit(Collide C, int plane0, int use_smem) {
    extern __shared__ long long sq[];
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    const int nx = C.o.nx, ny = C.o.ny, cells = nx * ny;
    Grid sg;
    if (P.geom >= 0) {
        sg = C.nodes[P.geom].sg;
    } else {
        const TaskGeom &G = C.geom[P.task];
        if (G.green < 0) return;
        sg = G.sg;
    }
    const double hx = sg.w / (double)(nx - 1), hy = sg.h / (double)(ny - 1);
    const double hxi = 1.0 / hx, hyi = 1.0 / hy;
    const double scale = ldexp(1.0, P.fixed_bits);
    long long *gq = C.qgrid + (long long)pl * cells;
    long long *dst = use_smem ? sq : gq;
    if (use_smem) {
        for (int c = threadIdx.x; c < cells; c += blockDim.x) sq[c] = 0;
        __syncthreads();
    }
    const SoA S = C.beam[P.src_beam];
    const double s = P.s;
    const double xlo = sg.x0, xhi = sg.x0 + sg.w, ylo = sg.y0, yhi = sg.y0 + sg.h;
    int outside = 0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < P.src_n; k += (long long)gridDim.x * blockDim.x) {
        long long p = P.src_start + k;
        double xd = S.c[0][p] + S.c[1][p] * s;
        double yd = S.c[2][p] + S.c[3][p] * s;
        if (P.count_dropped && !(isfinite(xd) && xlo <= xd && xd <= xhi && isfinite(yd) && ylo <= yd && yd <= yhi))
            ++outside;
        deposit_taps<METHOD>((xd - sg.x0) * hxi, (yd - sg.y0) * hyi, nx, ny, scale, dst, nx, use_smem);
    }
    if (P.count_dropped) {
        for (int o = 16; o; o >>= 1) outside += __shfl_xor_sync(0xffffffffu, outside, o);
        if ((threadIdx.x & 31) == 0 && outside) atomicAdd((unsigned long long *)&C.status->dropped, (unsigned long long)outside);
    }
    if (use_smem) {
        __syncthreads();
        for (int c = threadIdx.x; c < cells; c += blockDim.x) {
            long long v = sq[c];
            if (v) atomicAdd((unsigned long long *)&gq[c], (unsigned long long)v);
        }
    }
}

// Luminosity planes: 2 per pair (side 0 = beam-1 slice i at sM1, side 1 = beam-2 slice j at sM2)
// on the (lnx+1) x (lny+1) overlap mesh (pic_cpu.jl:2724-2735).
template <int METHOD>
__global__ void __launch_bounds__(512) k_lum_deposit(Collide C, int lj0, int use_smem) {
    extern __shared__ long long sq[];
    const int ql = blockIdx.y >> 1, side = blockIdx.y & 1;
    const LumJob &J = C.lumjobs[lj0 + ql];
    const LumGeom &L = C.lumgeom[J.pair];
    if (!L.ok) return;
    const int nw = C.o.lnx + 1, nh = C.o.lny + 1, cells = nw * nh;
    long long *gq = C.lq + (long long)blockIdx.y * cells;
    long long *dst = use_smem ? sq : gq;
    if (use_smem) {
        for (int c = threadIdx.x; c < cells; c += blockDim.x) sq[c] = 0;
        __syncthreads();
    }
    const SoA S = C.beam[side];
    const long long st = side ? J.s2_start : J.s1_start, n = side ? J.s2_n : J.s1_n;
    const double s = side ? J.sM2 : J.sM1;
    const double scale = ldexp(1.0, side ? J.bits2 : J.bits1);
    const double hxi = 1.0 / L.hx, hyi = 1.0 / L.hy;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        long long p = st + k;
        double vx = S.c[0][p] + S.c[1][p] * s;
        double vy = S.c[2][p] + S.c[3][p] * s;
        deposit_taps<METHOD>((vx - L.x0) * hxi, (vy - L.y0) * hyi, nw, nh, scale, dst, nw, use_smem);
    }
    if (use_smem) {
        __syncthreads();
        for (int c = threadIdx.x; c < cells; c += blockDim.x) {
            long long v = sq[c];
            if (v) atomicAdd((unsigned long long *)&gq[c], (unsigned long long)v);
        }
    }
}

// Overlap integral per pair: sum q1*q2 over the full (nx+1)(ny+1) extent times klum/(hx hy)
// (pic_cpu.jl:2725-2736).  Clears both grids for the next front.
__global__ void __launch_bounds__(256) k_lum_overlap(Collide C, int lj0) {
    const int ql = blockIdx.x;
    const LumJob &J = C.lumjobs[lj0 + ql];
    const LumGeom &L = C.lumgeom[J.pair];
    const int cells = (C.o.lnx + 1) * (C.o.lny + 1);
    long long *q1 = C.lq + (long long)(2 * ql) * cells;
    long long *q2 = q1 + cells;
    const double i1 = ldexp(1.0, -J.bits1), i2 = ldexp(1.0, -J.bits2);
    double acc = 0.0;
    for (int c = threadIdx.x; c < cells; c += blockDim.x) {
        long long a = q1[c], b = q2[c];
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
    if (threadIdx.x == 0 && L.ok) {
        double hxi = 1.0 / L.hx, hyi = 1.0 / L.hy;
        C.lum_parts[J.pair] = red[0] * C.klum * hxi * hyi;
    }
}

// ------------------------------------------------------------------ FFT convolution
__device__ __forceinline__ int plane_green(const Collide &C, const Plane &P) {
    if (P.green >= 0) return P.green;
    return C.geom[P.task].green;
}

// Forward x-transform of the charge rows: two rows per warp packed as one complex line
// (zero-padded to 2nx); the int64 grid is converted to FP64 and cleared as it is read.
__global__ void __launch_bounds__(128) k_conv_rows(Collide C, int plane0) {
    extern __shared__ double2 sm[];
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx;
    const int lgx = 31 - __clz(NX);
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    if (plane_green(C, P) < 0) return;
    double2 *tw = sm;
    double2 *line = sm + NX / 2 + (threadIdx.x >> 5) * NX;
    load_twiddles(tw, C.tw_x, NX);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int j0 = 2 * r, j1 = j0 + 1;
    if (j0 >= ny) return;
    const double inv = ldexp(1.0, -P.fixed_bits);
    long long *q = C.qgrid + (long long)pl * nx * ny;
    for (int i = lane; i < NX; i += 32) {
        double a = 0.0, b = 0.0;
        if (i < nx) {
            long long qa = q[(long long)j0 * nx + i];
            a = (double)qa * inv;
            if (qa) q[(long long)j0 * nx + i] = 0;
            if (j1 < ny) {
                long long qb = q[(long long)j1 * nx + i];
                b = (double)qb * inv;
                if (qb) q[(long long)j1 * nx + i] = 0;
            }
        }
        line[bitrev(i, lgx)] = make_double2(a, b);
    }
    warp_fft_passes(line, NX, tw, false);
    double2 *H = C.spec + (long long)pl * (nx + 1) * ny;
    for (int k = lane; k <= nx; k += 32) {
        double2 zk = line[k], zm = conjg(line[(NX - k) & (NX - 1)]);
        double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y + zm.y));
        double2 D = csub(zk, zm);
        H[(long long)k * ny + j0] = A;
        if (j1 < ny) H[(long long)k * ny + j1] = make_double2(0.5 * D.y, -0.5 * D.x);
    }
}

// y-transform, multiply by the Green spectrum, inverse y-transform; one frequency column per warp,
// in place.  Only rows j < ny of the result are kept (the field quadrant).
__global__ void __launch_bounds__(128) k_conv_cols(Collide C, int plane0) {
    extern __shared__ double2 sm[];
    const int nx = C.o.nx, ny = C.o.ny, NY = 2 * ny;
    const int lgy = 31 - __clz(NY);
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    const int slot = plane_green(C, P);
    if (slot < 0) return;
    double2 *tw = sm;
    double2 *line = sm + NY / 2 + (threadIdx.x >> 5) * NY;
    load_twiddles(tw, C.tw_y, NY);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (k > nx) return;
    double2 *col = C.spec + ((long long)pl * (nx + 1) + k) * ny;
    for (int j = lane; j < NY; j += 32) line[bitrev(j, lgy)] = j < ny ? col[j] : make_double2(0.0, 0.0);
    warp_fft_passes(line, NY, tw, false);
    const double2 *g = C.ghat + (long long)slot * C.gstride + (long long)k * NY;
    for (int j = lane; j < NY; j += 32) line[j] = cmul(line[j], g[j]);
    __syncwarp();
    for (int j = lane; j < NY; j += 32) {  // bit-reverse permutation in place
        int r = bitrev(j, lgy);
        if (j < r) { double2 t = line[j]; line[j] = line[r]; line[r] = t; }
    }
    warp_fft_passes(line, NY, tw, true);
    for (int j = lane; j < ny; j += 32) col[j] = line[j];
}

// Inverse x-transform (two Hermitian rows per complex line) producing phi for a tile of rows plus a
// two-row halo, then E = -grad(phi) on the tile (pic_cpu.jl:2531-2591).
constexpr int kFieldTile = 8;
__global__ void __launch_bounds__(128) k_conv_field(Collide C, int plane0) {
    extern __shared__ double2 sm[];
    const int nx = C.o.nx, ny = C.o.ny, NX = 2 * nx, NY = 2 * ny;
    const int lgx = 31 - __clz(NX);
    const int pl = blockIdx.y;
    const Plane &P = C.planes[plane0 + pl];
    if (plane_green(C, P) < 0) return;
    Grid sg;
    if (P.geom >= 0) sg = C.nodes[P.geom].sg;
    else sg = C.geom[P.task].sg;
    double2 *tw = sm;
    double2 *lines = sm + NX / 2;
    double *phi = (double *)(lines + 4 * NX);  // (kFieldTile + 4) rows x nx
    load_twiddles(tw, C.tw_x, NX);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int jt0 = blockIdx.x * kFieldTile;
    const int jt1 = min(jt0 + kFieldTile, ny);
    const int ja0 = max(jt0 - 2, 0), ja1 = min(jt1 + 2, ny);
    const int nrows = ja1 - ja0;
    const double2 *H = C.spec + (long long)pl * (nx + 1) * ny;
    const double scale = 1.0 / ((double)NX * (double)NY);
    double2 *line = lines + warp * NX;
    for (int rp = warp; 2 * rp < nrows; rp += 4) {
        const int ra = ja0 + 2 * rp, rb = ra + 1;
        const bool hb = rb < ja1;
        for (int k = lane; k < NX; k += 32) {
            double2 ca, cb;
            if (k <= nx) {
                ca = H[(long long)k * ny + ra];
                cb = hb ? H[(long long)k * ny + rb] : make_double2(0.0, 0.0);
            } else {
                ca = conjg(H[(long long)(NX - k) * ny + ra]);
                cb = hb ? conjg(H[(long long)(NX - k) * ny + rb]) : make_double2(0.0, 0.0);
            }
            line[bitrev(k, lgx)] = make_double2(ca.x - cb.y, ca.y + cb.x);
        }
        warp_fft_passes(line, NX, tw, true);
        for (int i = lane; i < nx; i += 32) {
            phi[(ra - ja0) * nx + i] = line[i].x * scale;
            if (hb) phi[(rb - ja0) * nx + i] = line[i].y * scale;
        }
        __syncwarp();
    }
    __syncthreads();
    const double hx = sg.w / (double)(nx - 1), hy = sg.h / (double)(ny - 1);
    const double hxi = 1.0 / hx, hyi = 1.0 / hy;
    const double c4 = 1.0 / 12.0;
    const bool fourth = C.o.fourth != 0;
    double *F = C.fields + (long long)pl * 3 * nx * ny;
    auto Pv = [&](int i, int j) { return phi[(j - ja0) * nx + i]; };  // 0-based i, j
    for (int idx = threadIdx.x; idx < (jt1 - jt0) * nx; idx += blockDim.x) {
        const int j = jt0 + idx / nx, i = idx % nx;
        double ey, ex;
        // Ey (pic_cpu.jl:2553-2572), 1-based j' = j+1
        if (j == 0) ey = hyi * (1.5 * Pv(i, 0) - 2 * Pv(i, 1) + 0.5 * Pv(i, 2));
        else if (j == ny - 1) ey = hyi * (-1.5 * Pv(i, ny - 1) + 2 * Pv(i, ny - 2) - 0.5 * Pv(i, ny - 3));
        else if (fourth && (j == 1 || j == ny - 2)) ey = 0.5 * hyi * (Pv(i, j - 1) - Pv(i, j + 1));
        else if (fourth) ey = c4 * hyi * ((Pv(i, j + 2) - Pv(i, j - 2)) + 8 * (Pv(i, j - 1) - Pv(i, j + 1)));
        else ey = 0.5 * hyi * (Pv(i, j - 1) - Pv(i, j + 1));
        // Ex (pic_cpu.jl:2573-2590)
        if (i == 0) ex = hxi * (1.5 * Pv(0, j) - 2 * Pv(1, j) + 0.5 * Pv(2, j));
        else if (i == nx - 1) ex = hxi * (-1.5 * Pv(nx - 1, j) + 2 * Pv(nx - 2, j) - 0.5 * Pv(nx - 3, j));
        else if (fourth && (i == 1 || i == nx - 2)) ex = 0.5 * hxi * (Pv(i - 1, j) - Pv(i + 1, j));
        else if (fourth) ex = c4 * hxi * ((Pv(i + 2, j) - Pv(i - 2, j)) + 8 * (Pv(i - 1, j) - Pv(i + 1, j)));
        else ex = 0.5 * hxi * (Pv(i - 1, j) - Pv(i + 1, j));
        long long o = (long long)j * nx + i;
        F[o] = Pv(i, j);
        F[(long long)nx * ny + o] = ex;
        F[2LL * nx * ny + o] = ey;
    }
}

// ------------------------------------------------------------------ kick
// Gather E and phi at one particle; two-node planes L and R (pic_cpu.jl:2596-2619).
template <int METHOD>
__device__ __forceinline__ void gather_lr(const DevOptions &o, const Grid &g, double x, double y, const double *L,
                                          const double *R, double zL, double zR, bool same, double &Kx, double &Ky,
                                          double &Kz) {
    const int nx = o.nx, ny = o.ny;
    const long long pc = (long long)nx * ny;
    double hx = g.w / (double)(nx - 1), hy = g.h / (double)(ny - 1);
    double u = (x - g.x0) / hx, v = (y - g.y0) / hy;
    Kx = 0.0; Ky = 0.0; Kz = 0.0;
    constexpr int NT = METHOD == 0 ? 2 : 3;
    int ix, iy; double wx[NT], wy[NT];
    if (METHOD == 0) { cic_weights(u, nx, ix, wx); cic_weights(v, ny, iy, wy); }
    else { tsc_weights(u, nx, ix, wx); tsc_weights(v, ny, iy, wy); }
#pragma unroll
    for (int m = 0; m < NT; ++m)
#pragma unroll
        for (int k = 0; k < NT; ++k) {
            long long c = (long long)(iy + k - 1) * nx + (ix + m - 1);
            double w = wx[m] * wy[k];
            if (same) {  // zL = 1, zR = 0: 1*E + 0*E == E for finite E
                Kx += w * (zL * L[pc + c] + zR * L[pc + c]);
                Ky += w * (zL * L[2 * pc + c] + zR * L[2 * pc + c]);
                Kz += w * (L[c] - R[c]);
            } else {
                Kx += w * (zL * L[pc + c] + zR * R[pc + c]);
                Ky += w * (zL * L[2 * pc + c] + zR * R[2 * pc + c]);
                Kz += w * (L[c] - R[c]);
            }
        }
}

// Three-node planes (pic_cpu.jl:2648-2680).
template <int METHOD>
__device__ __forceinline__ void gather_lmr(const DevOptions &o, const Grid &g, double x, double y, const double *L,
                                           const double *M, const double *R, double t, double &Kx, double &Ky,
                                           double &Kz) {
    const int nx = o.nx, ny = o.ny;
    const long long pc = (long long)nx * ny;
    double hx = g.w / (double)(nx - 1), hy = g.h / (double)(ny - 1);
    double u = (x - g.x0) / hx, v = (y - g.y0) / hy;
    double t2 = t * t;
    double aL = 2.0 * t2 - 3.0 * t + 1.0, aM = 4.0 * t - 4.0 * t2, aR = 2.0 * t2 - t;
    double bL = 3.0 - 4.0 * t, bM = 8.0 * t - 4.0, bR = 1.0 - 4.0 * t;
    Kx = 0.0; Ky = 0.0; Kz = 0.0;
    constexpr int NT = METHOD == 0 ? 2 : 3;
    int ix, iy; double wx[NT], wy[NT];
    if (METHOD == 0) { cic_weights(u, nx, ix, wx); cic_weights(v, ny, iy, wy); }
    else { tsc_weights(u, nx, ix, wx); tsc_weights(v, ny, iy, wy); }
#pragma unroll
    for (int m = 0; m < NT; ++m)
#pragma unroll
        for (int k = 0; k < NT; ++k) {
            long long c = (long long)(iy + k - 1) * nx + (ix + m - 1);
            double w = wx[m] * wy[k];
            Kx += w * (aL * L[pc + c] + aM * M[pc + c] + aR * R[pc + c]);
            Ky += w * (aL * L[2 * pc + c] + aM * M[2 * pc + c] + aR * R[2 * pc + c]);
            Kz += w * (bL * L[c] + bM * M[c] + bR * R[c]);
        }
}

// Synchro-beam kick of every field particle of the front's tasks: drift in, interpolated kick,
// drift out (pic_cpu.jl:1005-1017, 1218-1243, 1248-1273; :node form 1448-1538).
// Blocks map to (task, particle chunk) through `blockmap` (task index, first particle).
template <int METHOD>
__global__ void __launch_bounds__(256) k_kick(Collide C, int plane0_front, const int2 *blockmap) {
    const int2 bm = blockmap[blockIdx.x];
    const Task &T = C.tasks[bm.x];
    const long long k = (long long)bm.y + threadIdx.x;
    if (k >= T.fld_n) return;
    const DevOptions &o = C.o;
    const long long pc = (long long)o.nx * o.ny;
    const double *base = C.fields + (long long)(T.plane0 - plane0_front) * 3 * pc;
    Grid gL, gR;
    if (o.node) {
        gL = C.nodes[T.nodeL].fg;
        gR = C.nodes[T.nodeR].fg;
    } else {
        const TaskGeom &G = C.geom[bm.x];
        if (G.green < 0) return;
        gL = G.fg;
        gR = G.fg;
    }
    const SoA S = C.beam[T.fld_beam];
    const long long p = T.fld_start + k;
    double x = S.c[0][p], px = S.c[1][p], y = S.c[2][p], py = S.c[3][p], z = S.c[4][p], pz = S.c[5][p];
    const bool lk = o.longitudinal_kick != 0;
    double s = 0.5 * (z - T.c_src);
    x += s * px;
    y += s * py;
    if (lk) pz -= 0.25 * (px * px + py * py);
    const double zL = jclamp(-z * T.hzi + T.zbias, 0.0, 1.0);
    const double zR = 1.0 - zL;
    const double ks = T.ks;
    if (o.node) {
        const double *L = base, *R = base + 3 * pc, *Z = base + 6 * pc;
        if (!(isfinite(x) && gL.x0 <= x && x <= gL.x0 + gL.w && isfinite(y) && gL.y0 <= y && y <= gL.y0 + gL.h))
            atomicAdd((unsigned long long *)&C.status->dropped, 1ull);
        double KxL, KyL, KzL, KxR, KyR, KzR;
        gather_lr<METHOD>(o, gL, x, y, L, L, 1.0, 0.0, true, KxL, KyL, KzL);
        gather_lr<METHOD>(o, gR, x, y, R, R, 1.0, 0.0, true, KxR, KyR, KzR);
        px += ks * (zL * KxL + zR * KxR);
        py += ks * (zL * KyL + zR * KyR);
        if (lk) {
            double a, b, Kz;
            gather_lr<METHOD>(o, gL, x, y, L, Z, 1.0, 0.0, true, a, b, Kz);
            pz += ks * Kz * T.hzi;
        }
    } else if (o.quadratic) {
        const double *L = base, *R = base + 3 * pc, *M = base + 6 * pc;
        double Kx, Ky, Kz;
        gather_lmr<METHOD>(o, gL, x, y, L, M, R, 1.0 - zL, Kx, Ky, Kz);
        px += ks * Kx;
        py += ks * Ky;
        if (lk) pz += ks * Kz * T.hzi;
    } else {
        const double *L = base, *R = base + 3 * pc;
        double Kx, Ky, Kz;
        gather_lr<METHOD>(o, gL, x, y, L, R, zL, zR, false, Kx, Ky, Kz);
        px += ks * Kx;
        py += ks * Ky;
        if (lk) pz += ks * Kz * T.hzi;
    }
    double s2 = 0.5 * (T.c_src - z);
    x += s2 * px;
    y += s2 * py;
    if (lk) pz += 0.25 * (px * px + py * py);
    S.c[0][p] = x; S.c[1][p] = px; S.c[2][p] = y; S.c[3][p] = py; S.c[5][p] = pz;
}

// ------------------------------------------------------------------ node meshes
// Per-slice boxes of the turn-start state (pic_cpu.jl:1317-1358).  Source mode: the source
// slice drifted to every partner node, d = 0.5*(c_i - boundary_b) from `ref[sl*nref + b]`.
// Field mode: each field particle drifted to the collision point of every source-slice center,
// sh = 0.5*(z - c_i) with c_i = ref[i].  boxes: [sl][ref][4] ordered (xmin, xmax, ymin, ymax).
struct NodeBoxArgs {
    const double *x, *px, *y, *py, *z;
    long long start[kMaxSlices], count[kMaxSlices];
    const double *ref;
    unsigned long long *boxes;
    int *nanf;
    int nsl, nref, field_mode, pad;
};

__global__ void __launch_bounds__(256) k_node_boxes(NodeBoxArgs A) {
    const int sl = blockIdx.y;
    const long long st = A.start[sl], n = A.count[sl];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __shared__ unsigned long long red[8][4];
    for (int r0 = 0; r0 < A.nref; r0 += 8) {
        const int rn = min(8, A.nref - r0);
        unsigned long long mnx[8], mxx[8], mny[8], mxy[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) { mnx[r] = mny[r] = kOrdMinInit; mxx[r] = mxy[r] = kOrdMaxInit; }
        bool nan = false;
        for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
            const long long p = st + k;
            const double x = A.x[p], px = A.px[p], y = A.y[p], py = A.py[p];
            const double z = A.field_mode ? A.z[p] : 0.0;
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                if (r < rn) {
                    double xv, yv;
                    if (A.field_mode) {
                        double sh = 0.5 * (z - A.ref[r0 + r]);
                        xv = x + sh * px;
                        yv = y + sh * py;
                    } else {
                        double d = A.ref[(long long)sl * A.nref + r0 + r];
                        xv = x + px * d;
                        yv = y + py * d;
                    }
                    nan |= (xv != xv) | (yv != yv);
                    unsigned long long ex = ord_encode(xv), ey = ord_encode(yv);
                    mnx[r] = min(mnx[r], ex); mxx[r] = max(mxx[r], ex);
                    mny[r] = min(mny[r], ey); mxy[r] = max(mxy[r], ey);
                }
            }
        }
        int anynan = __syncthreads_or(nan);
        if (anynan && threadIdx.x == 0) atomicOr(A.nanf, 1);
        for (int r = 0; r < rn; ++r) {
            unsigned long long a = shfl_min_u64(mnx[r]), b = shfl_max_u64(mxx[r]);
            unsigned long long c = shfl_min_u64(mny[r]), d = shfl_max_u64(mxy[r]);
            if (lane == 0) { red[warp][0] = a; red[warp][1] = b; red[warp][2] = c; red[warp][3] = d; }
            __syncthreads();
            if (threadIdx.x < 4) {
                unsigned long long v = red[0][threadIdx.x];
                for (int w = 1; w < nw; ++w) v = (threadIdx.x & 1) ? max(v, red[w][threadIdx.x]) : min(v, red[w][threadIdx.x]);
                unsigned long long *dst = A.boxes + ((long long)sl * A.nref + r0 + r) * 4 + threadIdx.x;
                if (threadIdx.x & 1) atomicMax(dst, v); else atomicMin(dst, v);
            }
            __syncthreads();
        }
    }
}

// Node meshes of one direction (pic_cpu.jl:1359-1381): mesh (i, b) from the source drift boxes
// of nodes b and b+1 and the field boxes of the slices adjacent to node b.  sbox: [i][b][4],
// fbox: [field slice][i][4].  Meshes are written at meshes[i*nb + b-1].
__global__ void k_node_plan(DevOptions o, const unsigned long long *sbox, const unsigned long long *fbox, int ns_src,
                            int nb, const long long *src_count, NodeMesh *meshes, DevStatus *st) {
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= ns_src * nb) return;
    const int i = id / nb, b = id % nb + 1;  // b is 1-based
    NodeMesh &M = meshes[id];
    M.valid = 0;
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
