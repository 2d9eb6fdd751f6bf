// Register-resident FFT of lines of length L = 8 G held by G lanes each (G = 8, 16 or 32: L = 64, 128, 256;
// 32 / G lines per warp), in FP64 (double2) or FP32 (float2).
//
// Four-step (Bailey) decomposition with n = l + G m, k = k1 + 8 k2:
//   X[k1 + 8 k2] = sum_l W_G^(l k2) W_L^(l k1) sum_m x[l + G m] W_8^(m k1),
// and the G-point transforms split once more with l = Q a + b, k2 = c + 8 d (Q = G / 8):
//   Z[c + 8 d] = sum_b W_Q^(b d) W_G^(b c) sum_a W_8^(a c) V[Q a + b].
// Each lane holds 8 elements.  The 8-point and Q-point DFTs run in registers; between the levels the data
// moves through two shared-memory transposes per line, whose positions (rf_pos) are XOR-swizzled so that
// every quarter-warp phase of a 16-byte access touches eight distinct bank groups; twiddles come from
// per-block tables laid out in the order the lanes read them (rf_tables).  Against the radix-2^2 passes of
// fft.cuh (four shared-memory round trips of the whole line plus its staging) this moves each element
// through shared memory twice per transform.
//
// rf_fwd takes the natural order (lane l of the line, register m: x[l + G m]) to the "register order"
// (rf_spec gives the frequency a lane/register holds); rf_inv is the adjoint sequence (conjugate
// exponent, unnormalised), register order back to natural order.  A convolution multiplies in register
// order and never reorders its spectrum; the Green spectra of the y-lines are stored in register order.
#pragma once
#include "fft.cuh"

namespace octo {

template <class C2>
__device__ __forceinline__ C2 cmk(decltype(C2::x) x, decltype(C2::x) y) {
    C2 r;
    r.x = x;
    r.y = y;
    return r;
}
// a * conj(b)
template <class C2>
__device__ __forceinline__ C2 cmul_conj(C2 a, C2 b) {
    return cmk<C2>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// 2-, 4- and 8-point DFTs, natural order in and out; INV conjugates the exponent.
template <bool INV, class C2>
__device__ __forceinline__ void rf_dft2(C2 &a0, C2 &a1) {
    const C2 t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}
template <bool INV, class C2>
__device__ __forceinline__ void rf_dft4(C2 &a0, C2 &a1, C2 &a2, C2 &a3) {
    const C2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = csub(a1, a3);
    // forward: y1 = t1 - i t3, y3 = t1 + i t3
    const C2 u = INV ? cmk<C2>(-t3.y, t3.x) : cmk<C2>(t3.y, -t3.x);
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, u);
    a3 = csub(t1, u);
}
template <bool INV, class C2>
__device__ __forceinline__ void rf_dft8(C2 (&v)[8]) {
    using R = decltype(C2::x);
    const R r2 = R(0.70710678118654752440);  // 1/sqrt(2)
    C2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    rf_dft4<INV>(e0, e1, e2, e3);
    rf_dft4<INV>(o0, o1, o2, o3);
    // o_k *= W_8^k (forward W_8 = (1 - i)/sqrt 2); the inverse uses the conjugates
    if (!INV) {
        o1 = cmk<C2>((o1.x + o1.y) * r2, (o1.y - o1.x) * r2);
        o2 = cmk<C2>(o2.y, -o2.x);
        o3 = cmk<C2>((o3.y - o3.x) * r2, -(o3.x + o3.y) * r2);
    } else {
        o1 = cmk<C2>((o1.x - o1.y) * r2, (o1.x + o1.y) * r2);
        o2 = cmk<C2>(-o2.y, o2.x);
        o3 = cmk<C2>(-(o3.x + o3.y) * r2, (o3.x - o3.y) * r2);
    }
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// Lanes per line for a line of length L (0: not a register-FFT length; fft.cuh handles it).
__host__ __device__ constexpr int rf_lanes(int L) { return L == 256 ? 32 : L == 128 ? 16 : L == 64 ? 8 : 0; }

template <int G>
struct RfGeom {
    static constexpr int L = 8 * G, Q = G / 8, P = 8 / Q;
    // table entries: T1 7 G, T2 7 Q padded to a multiple of 8 (the scratch after it starts on a bank-group row)
    static constexpr int kT1 = 7 * G, kT2 = (7 * Q + 7) & ~7;
    static constexpr int kTables = kT1 + kT2;
    static constexpr int kWarpScratch = 256;            // elements per warp (32 / G lines of 8 G)
};

// Scratch position of element x of group k1 in a line: XOR-permutes inside aligned blocks of 8 elements.
template <int G>
__device__ __forceinline__ int rf_pos(int k1, int x) {
    constexpr int Q = G / 8, P = 8 / Q;
    return k1 * G + (x ^ (Q * (k1 & (P - 1)) + ((x >> 3) & (Q - 1))));
}
// Natural-order scratch position of frequency k (for the Hermitian split of packed real lines).
__device__ __forceinline__ int rf_nat(int k) { return k ^ ((k >> 3) & 7); }

// Frequency held by lane l (of its line) in register r after rf_fwd.
template <int G>
__device__ __forceinline__ int rf_spec(int l, int r) {
    constexpr int Q = G / 8, P = 8 / Q;
    const int k1 = l / Q, b = l % Q, cc = r / Q, d = r % Q;
    return k1 + 8 * (b * P + cc) + 64 * d;
}

// Twiddle tables from the natural table tw[k] = W_L^k (k < L/2): T1[(k1-1) G + l] = W_L^(l k1),
// T2[(c-1) Q + b] = W_G^(b c) = W_L^(8 b c).  Block-wide; the caller synchronises.
template <int G, class C2>
__device__ __forceinline__ void rf_tables(C2 *T, const C2 *tw) {
    constexpr int L = 8 * G, Q = G / 8;
    for (int e = threadIdx.x; e < 7 * G + 7 * Q; e += blockDim.x) {
        int k, dst;
        if (e < 7 * G) {
            k = ((e % G) * (e / G + 1)) % L;
            dst = e;
        } else {
            const int f = e - 7 * G;
            k = (8 * (f % Q) * (f / Q + 1)) % L;
            dst = RfGeom<G>::kT1 + f;
        }
        C2 w;
        if (k < L / 2) w = tw[k];
        else {
            w = tw[k - L / 2];
            w.x = -w.x;
            w.y = -w.y;
        }
        T[dst] = w;
    }
}

// Forward transform of the warp's lines: v[m] = x[l + G m] in, v[r] = X[rf_spec(l, r)] out.
// S: the warp's scratch (RfGeom::kWarpScratch elements); T: the tables.  Every lane of the warp calls it.
template <int G, class C2>
__device__ __forceinline__ void rf_fwd(C2 (&v)[8], C2 *S, const C2 *T) {
    constexpr int Q = G / 8, P = 8 / Q;
    const C2 *T1 = T, *T2 = T + RfGeom<G>::kT1;
    const int lane = threadIdx.x & 31, l = lane & (G - 1);
    C2 *Sl = S + (lane & ~(G - 1)) * 8;
    __syncwarp();
    rf_dft8<false>(v);
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1) v[k1] = cmul(v[k1], T1[(k1 - 1) * G + l]);
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) Sl[rf_pos<G>(k1, l)] = v[k1];
    __syncwarp();
    const int k1 = l / Q, b = l % Q;
#pragma unroll
    for (int a = 0; a < 8; ++a) v[a] = Sl[rf_pos<G>(k1, Q * a + b)];
    rf_dft8<false>(v);
    if constexpr (Q > 1) {
#pragma unroll
        for (int c = 1; c < 8; ++c) v[c] = cmul(v[c], T2[(c - 1) * Q + b]);
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 8; ++c) Sl[rf_pos<G>(k1, c * Q + b)] = v[c];
        __syncwarp();
#pragma unroll
        for (int cc = 0; cc < P; ++cc)
#pragma unroll
            for (int bb = 0; bb < Q; ++bb) v[cc * Q + bb] = Sl[rf_pos<G>(k1, (b * P + cc) * Q + bb)];
#pragma unroll
        for (int cc = 0; cc < P; ++cc) {
            if constexpr (Q == 4) rf_dft4<false>(v[4 * cc], v[4 * cc + 1], v[4 * cc + 2], v[4 * cc + 3]);
            else rf_dft2<false>(v[2 * cc], v[2 * cc + 1]);
        }
    }
    __syncwarp();
}

// Inverse (adjoint) transform: v[r] = X[rf_spec(l, r)] in, v[m] = L x[l + G m] out.
template <int G, class C2>
__device__ __forceinline__ void rf_inv(C2 (&v)[8], C2 *S, const C2 *T) {
    constexpr int Q = G / 8, P = 8 / Q;
    const C2 *T1 = T, *T2 = T + RfGeom<G>::kT1;
    const int lane = threadIdx.x & 31, l = lane & (G - 1);
    C2 *Sl = S + (lane & ~(G - 1)) * 8;
    const int k1 = l / Q, b = l % Q;
    __syncwarp();
    if constexpr (Q > 1) {
#pragma unroll
        for (int cc = 0; cc < P; ++cc) {
            if constexpr (Q == 4) rf_dft4<true>(v[4 * cc], v[4 * cc + 1], v[4 * cc + 2], v[4 * cc + 3]);
            else rf_dft2<true>(v[2 * cc], v[2 * cc + 1]);
        }
#pragma unroll
        for (int cc = 0; cc < P; ++cc)
#pragma unroll
            for (int bb = 0; bb < Q; ++bb) Sl[rf_pos<G>(k1, (b * P + cc) * Q + bb)] = v[cc * Q + bb];
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = Sl[rf_pos<G>(k1, c * Q + b)];
#pragma unroll
        for (int c = 1; c < 8; ++c) v[c] = cmul_conj(v[c], T2[(c - 1) * Q + b]);
        __syncwarp();
    }
    rf_dft8<true>(v);
#pragma unroll
    for (int a = 0; a < 8; ++a) Sl[rf_pos<G>(k1, Q * a + b)] = v[a];
    __syncwarp();
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) v[kk] = Sl[rf_pos<G>(kk, l)];
#pragma unroll
    for (int kk = 1; kk < 8; ++kk) v[kk] = cmul_conj(v[kk], T1[(kk - 1) * G + l]);
    rf_dft8<true>(v);
    __syncwarp();
}

}  // namespace octo
