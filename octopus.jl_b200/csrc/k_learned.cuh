// The learned field correction inside a coarse-grid collide (no reference counterpart): the
// Gaussian-subtracted hybrid (GaussianPICPoissonSolver, gaussian_pic.jl:646-884) or the plain PIC solver on a
// :slice_pair grid.  Per wavefront, after the charge deposit:
// k_cnn_prep turns each plane's int64 charge grid into the network's input; after the field solve,
// k_cnn_apply adds the network's field correction to the plane's field cells.
//
// Units.  The network works in grid units: input channel 0 is the charge of a node over the plane's total
// charge times the node count (mean 1), channel 1 is log(hy / hx) (the cell aspect), channels 2..7 zero; its
// output channels are dEx * hx and dEy * hy of a unit total charge (a point charge's field r / |r|^2 in these
// units depends only on the node offsets and the cell aspect), scaled by `out_scale`.  The correction is
// defined on the source mesh's nodes; the field mesh of the :integrated Green function is the source mesh
// shifted by a whole number of cells, so field node (i, j) takes source node (i + sx, j + sy).  Nodes within
// `edge` nodes of the mesh border (never sampled when the network was trained) get no correction.
#pragma once
#include <cuda_bf16.h>

#include "k_pic.cuh"

namespace octo {

// grid: one block per plane of the front.  qplane[pl] receives the plane's total fixed-point charge.
__global__ void __launch_bounds__(256) k_cnn_prep(Collide C, int plane0, __nv_bfloat16 *x0, long long *qplane) {
    pdl_wait();
    pdl_release();
    __shared__ long long red[256];
    const int pl = blockIdx.x;
    const Plane &P = C.planes[plane0 + pl];
    const TaskGeom &G = C.geom[P.task];
    const int nx = C.o.nx, ny = C.o.ny, cells = nx * ny;
    __nv_bfloat16 *out = x0 + (long long)pl * cells * 8;
    const long long *q = C.qgrid + (long long)pl * cells;
    long long s = 0;
    for (int c = threadIdx.x; c < cells; c += blockDim.x) s += q[c];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const long long qt = red[0];
    if (threadIdx.x == 0) qplane[pl] = qt;
    const bool ok = G.green >= 0 && qt > 0;
    const double hx = G.sg.w / (double)(nx - 1), hy = G.sg.h / (double)(ny - 1);
    const float aspect = ok ? (float)log(hy / hx) : 0.f;
    const double norm = ok ? (double)cells / (double)qt : 0.0;
    for (int c = threadIdx.x; c < cells; c += blockDim.x) {
        const float v = ok ? (float)((double)q[c] * norm) : 0.f;
        __nv_bfloat16 *o = out + (long long)c * 8;
        o[0] = __float2bfloat16_rn(v);
        o[1] = __float2bfloat16_rn(aspect);
#pragma unroll
        for (int k = 2; k < 8; ++k) o[k] = __float2bfloat16_rn(0.f);
    }
}

// grid: one block per plane of the front.  net_out: the network's head output [plane][ny][nx][8] (fp32).
// flags[0] counts the planes whose largest correction exceeds `tol` (in grid units).  A plane that holds a
// difference of two planes' fields (the precision form's q_self - q_other) gets the same difference of
// the two planes' corrections.
template <class R>
__global__ void __launch_bounds__(256) k_cnn_apply(Collide C, int plane0, const float *net_out, const long long *qplane,
                                                   float inv_scale, int edge, float tol, int *flags) {
    pdl_wait();
    pdl_release();
    __shared__ float red[256];
    const int pl = blockIdx.x;
    const Plane &P = C.planes[plane0 + pl];
    const TaskGeom &G = C.geom[P.task];
    const int nx = C.o.nx, ny = C.o.ny, cells = nx * ny;
    if (G.green < 0) return;
    const int other = P.other_delta ? pl + P.other_delta : -1;
    const double sgn_self = (other < 0 || P.self_first) ? 1.0 : -1.0;
    const double hx = G.sg.w / (double)(nx - 1), hy = G.sg.h / (double)(ny - 1);
    const int sx = (int)rint((G.fg.x0 - G.sg.x0) / hx), sy = (int)rint((G.fg.y0 - G.sg.y0) / hy);
    const double unit = ldexp(1.0, -P.fixed_bits) * (double)inv_scale;
    const double q_self = (double)qplane[pl] * unit * sgn_self;
    const double q_other = other >= 0 ? -(double)qplane[other] * unit * sgn_self : 0.0;
    const float *o_self = net_out + (long long)pl * cells * 8;
    const float *o_other = other >= 0 ? net_out + (long long)other * cells * 8 : nullptr;
    R *f = (R *)C.fields + (long long)pl * cells * 4;  // cell c: Ex, Ey, phi, w
    float big = 0.f;
    for (int c = threadIdx.x; c < cells; c += blockDim.x) {
        const int i = c % nx, j = c / nx;
        const int si = i + sx, sj = j + sy;
        if (i < edge || i >= nx - edge || j < edge || j >= ny - edge) continue;
        if (si < edge || si >= nx - edge || sj < edge || sj >= ny - edge) continue;
        const long long k = ((long long)sj * nx + si) * 8;
        const float *v = o_self + k;
        big = fmaxf(big, fmaxf(fabsf(v[0]), fabsf(v[1])));
        double dx = q_self * (double)v[0], dy = q_self * (double)v[1];
        if (o_other) {
            dx += q_other * (double)o_other[k];
            dy += q_other * (double)o_other[k + 1];
        }
        f[4LL * c + 0] += (R)(dx / hx);
        f[4LL * c + 1] += (R)(dy / hy);
    }
    red[threadIdx.x] = big;
    __syncthreads();
    for (int s = 128; s; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0 && red[0] * inv_scale > tol) atomicAdd(flags, 1);
}

}  // namespace octo
