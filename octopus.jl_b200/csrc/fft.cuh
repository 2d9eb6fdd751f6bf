// Shared-memory FFT building blocks for the zero-padded Hockney convolution.
//
// One warp transforms one line of length L = 2^a or 3 * 2^a (L <= 1024; padded grids of 2^a or 3 * 2^a
// cells per axis) held in shared memory, in FP64 (double2) or FP32 (float2) complex arithmetic.
// Twiddles tw[k] = exp(-2 pi i k / L), k < L/2, are staged in shared memory per block.  A line is loaded
// at fft_pos(i) (bit-reversed; for 3 * 2^a the residue classes i mod 3 as three contiguous bit-reversed
// sub-lines), and warp_fft() leaves it in natural order.
// The convolution never materialises the padded (2nx x 2ny) complex plane: rows are
// transformed two at a time as one complex line (real-input packing), only the nx+1
// non-redundant x-frequencies are carried through the column pass, and the inverse
// produces only the nx x ny quadrant the field needs.
#pragma once
#include "octo_internal.cuh"

namespace octo {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 conjg(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conjg(float2 a) { return make_float2(a.x, -a.y); }

__device__ __forceinline__ int bitrev(int k, int lg) { return (int)(__brev((unsigned)k) >> (32 - lg)); }

// Shared-memory swizzle of a (sub-)line: element i sits at i ^ ((i >> 4) & 15), a bijection inside every
// aligned block of 16 (lines are multiples of 16 long).  Simulated over the access patterns of the passes
// below it cuts shared-memory wavefronts from 2.6x to 1.5x the conflict-free count for 16-byte elements
// (L = 256) and from 4x to 1.6x for 8-byte elements.
__device__ __forceinline__ int sw(int i) { return i ^ ((i >> 4) & 15); }

// Twiddle-table swizzle: entry k sits at k ^ (((k >> 3) ^ (k >> 5)) & m), m = 15 when the table length L/2 is a
// multiple of 16 (a bijection inside each aligned block of 16), else 0.  The passes read W^(j * step) with
// power-of-two steps, which without it fall into one bank (simulated: 200 -> 64 wavefronts per 256-point
// FP64 line).
__device__ __forceinline__ int tsw(int k, int m) { return k ^ (((k >> 3) ^ (k >> 5)) & m); }
__device__ __forceinline__ int tw_mask(int L) { return ((L >> 1) & 15) ? 0 : 15; }

// Butterfly passes on a buffer already loaded in bit-reversed order.  Pairs of radix-2 DIT stages
// (half-sizes h and 2h) are merged into one radix-2^2 pass over groups of four elements
// {i, i+h, i+2h, i+3h}: half the shared-memory round trips and warp syncs of plain radix-2, with the
// same twiddles (the second-stage twiddle of the odd pair is -i times that of the even pair, applied
// exactly by a swap and a sign change).  An odd log2(L) starts with one radix-2 pass.
// tws: twiddle stride, 1 for a table of length L itself, 3 for a sub-line of length L of a 3L table;
// tm: the table's swizzle mask (tw_mask of its own length).
template <class C2>
__device__ __forceinline__ void warp_fft_passes(C2 *a, int L, const C2 *tw, bool inv, int tws, int tm) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    int half = 1, step = L >> 1;
    const int lg = 31 - __clz(L);
    if (lg & 1) {  // one radix-2 pass (half = 1, twiddle 1)
        for (int b = lane; b < (L >> 1); b += 32) {
            const int i0 = b << 1;
            const C2 u = a[sw(i0)], v = a[sw(i0 + 1)];
            a[sw(i0)] = cadd(u, v);
            a[sw(i0 + 1)] = csub(u, v);
        }
        __syncwarp();
        half = 2;
        step >>= 1;
    }
    for (; half < L; half <<= 2, step >>= 2) {
        // groups of 4h elements; within each, j in [0, h): elements j, j+h, j+2h, j+3h
        const int quads = L >> 2;
        for (int b = lane; b < quads; b += 32) {
            const int j = b & (half - 1);
            const int i0 = ((b & ~(half - 1)) << 2) | j;
            C2 w1 = tw[tsw(j * step * tws, tm)];          // W_{2h}^j
            C2 w2 = tw[tsw(j * (step >> 1) * tws, tm)];   // W_{4h}^j
            if (inv) { w1.y = -w1.y; w2.y = -w2.y; }
            const C2 x0 = a[sw(i0)], x1 = a[sw(i0 + half)], x2 = a[sw(i0 + 2 * half)], x3 = a[sw(i0 + 3 * half)];
            const C2 t1 = cmul(x1, w1), t3 = cmul(x3, w1);
            const C2 a0 = cadd(x0, t1), a1 = csub(x0, t1), a2 = cadd(x2, t3), a3 = csub(x2, t3);
            const C2 u2 = cmul(a2, w2), v3 = cmul(a3, w2);
            // w3 = W_{4h}^{j+h} = w2 * (-i) forward, w2 * (+i) inverse
            C2 u3;
            if (inv) { u3.x = -v3.y; u3.y = v3.x; } else { u3.x = v3.y; u3.y = -v3.x; }
            a[sw(i0)] = cadd(a0, u2);
            a[sw(i0 + 2 * half)] = csub(a0, u2);
            a[sw(i0 + half)] = cadd(a1, u3);
            a[sw(i0 + 3 * half)] = csub(a1, u3);
        }
        __syncwarp();
    }
}

// Line geometry: M = L (power of two) or L / 3.
struct FftLen {
    int L, M, lgM, three, tm;
};
__device__ __forceinline__ FftLen fft_len(int L) {
    FftLen f;
    f.L = L;
    f.tm = tw_mask(L);
    f.three = (L % 3) == 0;
    f.M = f.three ? L / 3 : L;
    f.lgM = 31 - __clz(f.M);
    return f;
}
// Shared-memory position of input element i (digit-reversed, swizzled) and of output element k (natural
// order, swizzled) of a line.
__device__ __forceinline__ int fft_pos(const FftLen &f, int i) {
    if (!f.three) return sw(bitrev(i, f.lgM));
    const int m = i / 3;
    return (i - 3 * m) * f.M + sw(bitrev(m, f.lgM));
}
__device__ __forceinline__ int fft_out(const FftLen &f, int k) { return (k & ~(f.M - 1)) | sw(k & (f.M - 1)); }
// W_L^k for 0 <= k < L from the half table (W_L^k = -W_L^(k - L/2)), conjugated for the inverse.
template <class C2>
__device__ __forceinline__ C2 twiddle(const C2 *tw, int L, int k, bool inv, int tm) {
    C2 w;
    if (k < (L >> 1)) w = tw[tsw(k, tm)];
    else { w = tw[tsw(k - (L >> 1), tm)]; w.x = -w.x; w.y = -w.y; }
    if (inv) w.y = -w.y;
    return w;
}

// Whole-line transform in place: radix-2^2 passes for L = 2^a; for L = 3 * 2^a three length-L/3
// transforms of the residue classes (decimation in time) and one radix-3 combine,
// X[k + qM] = Y0[k] + W3^q W^k Y1[k] + W3^2q W^2k Y2[k].
template <class C2>
__device__ __forceinline__ void warp_fft(C2 *a, const FftLen &f, const C2 *tw, bool inv) {
    if (!f.three) {
        warp_fft_passes(a, f.L, tw, inv, 1, f.tm);
        return;
    }
    const int M = f.M;
    warp_fft_passes(a, M, tw, inv, 3, f.tm);
    warp_fft_passes(a + M, M, tw, inv, 3, f.tm);
    warp_fft_passes(a + 2 * M, M, tw, inv, 3, f.tm);
    __syncwarp();
    using R = decltype(a[0].x);
    const R h = R(0.5), s3 = R(0.86602540378443864676);  // sin(2 pi / 3)
    for (int k = (threadIdx.x & 31); k < M; k += 32) {
        const int ks = sw(k);
        const C2 y0 = a[ks];
        const C2 z1 = cmul(a[M + ks], twiddle(tw, f.L, k, inv, f.tm));
        const C2 z2 = cmul(a[2 * M + ks], twiddle(tw, f.L, 2 * k, inv, f.tm));
        const C2 t = cadd(z1, z2), d = csub(z1, z2);
        C2 m, x0, x1, x2;
        m.x = y0.x - h * t.x;
        m.y = y0.y - h * t.y;
        // forward: X1 = m - i s3 d, X2 = m + i s3 d (the inverse swaps them)
        const R ux = s3 * d.y, uy = -(s3 * d.x);  // -i s3 d
        x0 = cadd(y0, t);
        x1.x = m.x + (inv ? -ux : ux); x1.y = m.y + (inv ? -uy : uy);
        x2.x = m.x - (inv ? -ux : ux); x2.y = m.y - (inv ? -uy : uy);
        a[ks] = x0;
        a[M + ks] = x1;
        a[2 * M + ks] = x2;
    }
    __syncwarp();
}

// Stage the twiddle table of length L/2 into shared memory (block-wide).
template <class C2>
__device__ __forceinline__ void load_twiddles(C2 *s_tw, const C2 *g_tw, int L) {
    const int tm = tw_mask(L);
    for (int k = threadIdx.x; k < (L >> 1); k += blockDim.x) s_tw[tsw(k, tm)] = g_tw[k];
}

}  // namespace octo
