// Interaction-mesh geometry and slice-pair Green-cache decisions, evaluated on the device
// by one thread per directed interaction (no host round trip per wavefront, unlike the
// reference CUDA route's bounds readback at pic_cuda.jl:1846).
#pragma once
#include "octo_internal.cuh"

namespace octo {

// pic_cpu.jl:1646-1672 ; returns false on a degenerate extent.
__device__ inline bool resolve_extent(const DevOptions &o, double xspan, double yspan, double &w, double &h) {
    w = jmax(xspan, o.min_ex);
    h = jmax(yspan, o.min_ey);
    return isfinite(w) && isfinite(h) && w > 0.0 && h > 0.0;
}

// pic_cpu.jl:1877-1905
__device__ inline void align_origins(int green_type, double s0, double f0, double h, double &so, double &fo) {
    double f1 = s0 / h - floor(s0 / h);
    double f2 = f0 / h - floor(f0 / h);
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

// pic_cpu.jl:1641-1644
__device__ inline double quantize_extent(double w, double q) {
    if (!(q > 0.0 && isfinite(w) && w > 0.0)) return w;
    return exp2(ceil(log2(w) / q) * q);
}

// pic_cpu.jl:1674-1718
__device__ inline bool interaction_grids(const DevOptions &o, double sxmin, double sxmax, double symin, double symax,
                                         double fxmin, double fxmax, double fymin, double fymax, Grid &sg,
                                         Grid &fg) {
    double width, height;
    if (!resolve_extent(o, jmax(sxmax - sxmin, fxmax - fxmin), jmax(symax - symin, fymax - fymin), width, height))
        return false;
    double tx = width / (double)(o.nx - 4);
    double ty = height / (double)(o.ny - 4);
    width += 3 * tx;
    height += 3 * ty;
    if (o.quantize > 0.0) {
        width = quantize_extent(width, o.quantize);
        height = quantize_extent(height, o.quantize);
        double hx = width / (double)(o.nx - 1), hy = height / (double)(o.ny - 1);
        double sx0 = rint(((sxmin + sxmax) / 2 - width / 2) / hx) * hx;
        double sy0 = rint(((symin + symax) / 2 - height / 2) / hy) * hy;
        double fx0 = rint(((fxmin + fxmax) / 2 - width / 2) / hx) * hx;
        double fy0 = rint(((fymin + fymax) / 2 - height / 2) / hy) * hy;
        align_origins(o.green_type, sx0, fx0, hx, sx0, fx0);
        align_origins(o.green_type, sy0, fy0, hy, sy0, fy0);
        sg = Grid{sx0, sy0, width, height};
        fg = Grid{fx0, fy0, width, height};
        return true;
    }
    double sx0 = sxmin - 1.5 * tx, sy0 = symin - 1.5 * ty;
    double fx0 = fxmin - 1.5 * tx, fy0 = fymin - 1.5 * ty;
    align_origins(o.green_type, sx0, fx0, tx, sx0, fx0);
    align_origins(o.green_type, sy0, fy0, ty, sy0, fy0);
    sg = Grid{sx0, sy0, width, height};
    fg = Grid{fx0, fy0, width, height};
    return true;
}

// pic_cpu.jl:1787-1808
__device__ inline bool grid_size_usable(const Grid &c, const Grid &r, double mr) {
    return c.w >= r.w && c.h >= r.h && r.w >= mr * c.w && r.h >= mr * c.h;
}
__device__ inline bool grid_covers(const DevOptions &o, const Grid &g, double xmin, double xmax, double ymin,
                                   double ymax) {
    double hx = g.w / (double)(o.nx - 1), hy = g.h / (double)(o.ny - 1);
    double m = kTemplateMarginCells;
    return g.x0 + m * hx <= xmin && g.x0 + g.w - m * hx >= xmax && g.y0 + m * hy <= ymin &&
           g.y0 + g.h - m * hy >= ymax;
}
// pic_cpu.jl:1810-1821
__device__ inline Grid expand_grid(const Grid &g, double factor) {
    if (factor <= 1.0) return g;
    double nw = g.w * factor, nh = g.h * factor;
    return Grid{g.x0 - (nw - g.w) / 2, g.y0 - (nh - g.h) / 2, nw, nh};
}

}  // namespace octo
