// Shared-memory radix-2 FFT building blocks for the zero-padded Hockney convolution.
//
// One warp transforms one line of length L = 2^lg (L <= 1024) held in shared memory.
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

__device__ __forceinline__ int bitrev(int k, int lg) { return (int)(__brev((unsigned)k) >> (32 - lg)); }

// Butterfly passes on a buffer already loaded in bit-reversed order.
__device__ __forceinline__ void warp_fft_passes(double2 *a, int L, const double2 *tw, bool inv) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    for (int half = 1, step = L >> 1; half < L; half <<= 1, step >>= 1) {
        for (int b = lane; b < (L >> 1); b += 32) {
            int j = b & (half - 1);
            int i0 = ((b & ~(half - 1)) << 1) | j;
            double2 w = tw[j * step];
            if (inv) w.y = -w.y;
            double2 u = a[i0];
            double2 v = cmul(a[i0 + half], w);
            a[i0] = cadd(u, v);
            a[i0 + half] = csub(u, v);
        }
        __syncwarp();
    }
}

// Stage the twiddle table of length L/2 into shared memory (block-wide).
__device__ __forceinline__ void load_twiddles(double2 *s_tw, const double2 *g_tw, int L) {
    for (int k = threadIdx.x; k < (L >> 1); k += blockDim.x) s_tw[k] = g_tw[k];
}

}  // namespace octo
