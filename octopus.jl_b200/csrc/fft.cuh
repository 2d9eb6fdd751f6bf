// Shared-memory radix-2 FFT building blocks for the zero-padded Hockney convolution.
//
// One warp transforms one line of length L = 2^lg (L <= 1024) held in shared memory, in FP64
// (double2) or FP32 (float2) complex arithmetic.
// Twiddles tw[k] = exp(-2 pi i k / L), k < L/2, are staged in shared memory per block.
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

// Butterfly passes on a buffer already loaded in bit-reversed order.  Pairs of radix-2 DIT stages
// (half-sizes h and 2h) are merged into one radix-2^2 pass over groups of four elements
// {i, i+h, i+2h, i+3h}: half the shared-memory round trips and warp syncs of plain radix-2, with the
// same twiddles (the second-stage twiddle of the odd pair is -i times that of the even pair, applied
// exactly by a swap and a sign change).  An odd log2(L) starts with one radix-2 pass.
template <class C2>
__device__ __forceinline__ void warp_fft_passes(C2 *a, int L, const C2 *tw, bool inv) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    int half = 1, step = L >> 1;
    const int lg = 31 - __clz(L);
    if (lg & 1) {  // one radix-2 pass (half = 1, twiddle 1)
        for (int b = lane; b < (L >> 1); b += 32) {
            const int i0 = b << 1;
            const C2 u = a[i0], v = a[i0 + 1];
            a[i0] = cadd(u, v);
            a[i0 + 1] = csub(u, v);
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
            C2 w1 = tw[j * step];          // W_{2h}^j
            C2 w2 = tw[j * (step >> 1)];   // W_{4h}^j
            if (inv) { w1.y = -w1.y; w2.y = -w2.y; }
            const C2 x0 = a[i0], x1 = a[i0 + half], x2 = a[i0 + 2 * half], x3 = a[i0 + 3 * half];
            const C2 t1 = cmul(x1, w1), t3 = cmul(x3, w1);
            const C2 a0 = cadd(x0, t1), a1 = csub(x0, t1), a2 = cadd(x2, t3), a3 = csub(x2, t3);
            const C2 u2 = cmul(a2, w2), v3 = cmul(a3, w2);
            // w3 = W_{4h}^{j+h} = w2 * (-i) forward, w2 * (+i) inverse
            C2 u3;
            if (inv) { u3.x = -v3.y; u3.y = v3.x; } else { u3.x = v3.y; u3.y = -v3.x; }
            a[i0] = cadd(a0, u2);
            a[i0 + 2 * half] = csub(a0, u2);
            a[i0 + half] = cadd(a1, u3);
            a[i0 + 3 * half] = csub(a1, u3);
        }
        __syncwarp();
    }
}

// Stage the twiddle table of length L/2 into shared memory (block-wide).
template <class C2>
__device__ __forceinline__ void load_twiddles(C2 *s_tw, const C2 *g_tw, int L) {
    for (int k = threadIdx.x; k < (L >> 1); k += blockDim.x) s_tw[k] = g_tw[k];
}

}  // namespace octo
