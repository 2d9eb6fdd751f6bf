// BF16 GEMM on the fifth-generation tensor cores (tcgen05 / UMMA), the contraction behind the learned
// field correction's convolutions (forward, input gradient, weight gradient).
//
//   C[M, N] (fp32) = sum_k A[m, k] * B[n, k]            (both operands K-major)
//
// A is either a dense row-major bf16 matrix or, for a 3x3 convolution with padding 1, the implicit im2col
// of an NHWC bf16 activation tensor (row m = pixel (b, y, x), column k = (ky * 3 + kx) * C + c); B is a
// row-major bf16 matrix (for a convolution: weights [Cout][ky][kx][Cin]).
//
// A CTA of 256 threads computes 128 x BN tiles (persistent over the M tiles of its column and K range, so
// the TMEM allocation and the barriers are set up once): the K loop moves 64-wide chunks of A and B from global
// memory into shared memory with 16-byte cp.async copies (four stages, two chunks in flight ahead; zero-filled
// outside the matrix and the padded image) in the canonical no-swizzle K-major layout -- 8-row x 16-byte core
// matrices, 128 contiguous bytes each, the two K halves of one instruction LBO = 128 bytes apart and 8-row
// groups SBO = 1024 bytes apart -- and one thread issues four tcgen05.mma (M = 128, N = BN, K = 16) per
// chunk into a TMEM accumulator, committing each chunk to the stage's mbarrier so the stage can be refilled
// once its MMAs are done.  A thread always loads the same four A rows of a tile, so the implicit im2col's
// pixel coordinates are computed once per tile.  The epilogue reads the accumulator with tcgen05.ld (warps w
// and w + 4 share TMEM lanes 32w..32w+31 = tile rows, each taking half of the 32-column blocks) and writes
// fp32 (split-K partials) or bias + ReLU as bf16.
//
// Every mbarrier wait is bounded (about one second of the global timer); on expiry the kernel records
// OCTO_ERR_TIMEOUT in *error, waits (again bounded) for its MMAs, frees its TMEM and returns.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "octo_internal.cuh"

namespace octo {
namespace nn {

constexpr int kBM = 128;       // tile rows (the MMA's M)
constexpr int kBK = 64;        // K per stage
constexpr int kGemmThreads = 256;
constexpr int kTimeoutCode = 6;  // OCTO_ERR_TIMEOUT

struct GemmArgs {
    int M, N, K;                  // K a multiple of 8
    const __nv_bfloat16 *A;       // a_mode 0: A[m * lda + k]
    long long lda;
    int a_mode;                   // 0 dense, 1 implicit 3x3 / pad-1 convolution of an NHWC tensor, 2 the same
                                  // of [nearest-upsampled A, A2] concatenated along channels (a U-Net decoder)
    int H, W, C;                  // a_mode 1, 2: input height, width, channels (C a multiple of 8); K = 9 C
    const __nv_bfloat16 *A2;      // a_mode 2: the skip tensor [b][H][W][C - Cu]; A is [b][H/2][W/2][Cu]
    int Cu;                       // a_mode 2: channels from the upsampled tensor (a multiple of 8)
    const __nv_bfloat16 *B;       // B[n * ldb + k]
    long long ldb;
    float *out;                   // fp32 result (when out_bf16 is null): out[z * split_stride + m * ldc + n]
    long long ldc, split_stride;
    int k_per_split;              // K range of blockIdx.z: [z * k_per_split, (z + 1) * k_per_split), multiple of kBK
    const float *bias;            // added per column (fp32 output: only without split-K); null = none
                                  // bf16 epilogue: out_bf16[m * ldo + n] = bf16(max?(0, acc + bias[n]))
    int relu;
    __nv_bfloat16 *out_bf16;
    long long ldo;
    int *error;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for the completion of the mbarrier phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns = 1000000000ull) {
    const uint64_t t0 = global_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}
// No-swizzle K-major shared-memory matrix descriptor (version 1, the tcgen05 format).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: bf16 A and B, fp32 accumulator, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

// Byte offset of the 16-byte chunk (row r, k-chunk kc) of a stage tile in the canonical layout.
__device__ __forceinline__ uint32_t tile_off(int r, int kc) { return (uint32_t)((r >> 3) * 1024 + kc * 128 + (r & 7) * 16); }

// 16-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros (padding, tails) without reading.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

constexpr int kStages = 4;
constexpr int kDepth = kStages - 2;  // K chunks in flight ahead of the one being multiplied (a refill waits for
                                     // the MMAs of the chunk two back, which are done by then)
constexpr int kRowsPerThread = (kBM * 8) / kGemmThreads;  // A rows (one 16-byte k-chunk each) a thread loads

// The thread -> chunk mapping of a stage: chunk c = it * kGemmThreads + tid covers row (c & 7) + 8 * (c >> 6)
// and k-chunk (c >> 3) & 7, so a thread loads the same rows and the same k-chunk column in every stage; a
// group of 8 consecutive threads writes 8 rows of one k-chunk (128 contiguous bytes of shared memory).
__device__ __forceinline__ int map_row(int it, int tid) {
    return (tid & 7) + 8 * ((kGemmThreads / 64) * it + (tid >> 6));
}
__device__ __forceinline__ int map_kc(int tid) { return (tid >> 3) & 7; }

// q = v / d for 0 <= v < 2^24, 1 <= d < 2^24: a float estimate corrected by one step either way.
__device__ __forceinline__ int div_small(int v, int d, float inv_d) {
    int q = (int)((float)v * inv_d);
    if ((q + 1) * d <= v) ++q;
    if (q * d > v) --q;
    return q;
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 2) k_umma_gemm(const GemmArgs g) {
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "BN");
    constexpr uint32_t kStageA = kBM * kBK * 2, kStageB = BN * kBK * 2;
    constexpr uint32_t kCols = BN < 32 ? 32 : BN;
    extern __shared__ __align__(1024) unsigned char g_umma_smem[];
    __shared__ __align__(8) uint64_t bar[kStages];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    pdl_wait();
    pdl_release();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * g.k_per_split;
    const int ke = min(g.K, kb + g.k_per_split);
    const int nk = ke > kb ? (ke - kb + kBK - 1) / kBK : 0;
    const int tiles_m = (g.M + kBM - 1) / kBM;
    unsigned char *const smA = g_umma_smem, *const smB = g_umma_smem + kStages * kStageA;
    const uint32_t sA0 = smem_u32(smA), sB0 = smem_u32(smB);
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[s])));
        // the barriers are signalled by tcgen05.commit: make their initialisation visible to that proxy
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        abort_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = umma_idesc_bf16(BN);
    uint32_t commits[kStages] = {0, 0, 0, 0};  // commits issued per stage (thread 0), across all tiles
    const int kc_t = map_kc(tid);
    const int Cs = g.C - g.Cu;
    const int hw = g.H * g.W;
    const float inv_hw = 1.0f / (float)(hw > 0 ? hw : 1), inv_w = 1.0f / (float)(g.W > 0 ? g.W : 1);
    const bool direct_bf16 = g.out_bf16 != nullptr;  // bf16 (bias, ReLU) straight from the accumulator
    bool failed = false;

    // persistent over the M tiles of this (n, split) column
    for (int tile = blockIdx.x; tile < tiles_m && !failed; tile += gridDim.x) {
        const int m0 = tile * kBM;
        // this thread's A rows: (b, y, x) of the pixel and its element offset (convolutions), or the row offset
        // (dense); rows past M are marked y = -1 (zero fill)
        long long rbase[kRowsPerThread];
        int ry[kRowsPerThread], rx[kRowsPerThread], rb[kRowsPerThread];
#pragma unroll
        for (int it = 0; it < kRowsPerThread; ++it) {
            const int m = m0 + map_row(it, tid);
            ry[it] = -1; rx[it] = 0; rb[it] = 0; rbase[it] = 0;
            if (m < g.M) {
                if (g.a_mode == 0) {
                    ry[it] = 0;
                    rbase[it] = (long long)m * g.lda;
                } else {
                    const int b = div_small(m, hw, inv_hw), rem = m - b * hw;
                    const int y = div_small(rem, g.W, inv_w), x = rem - y * g.W;
                    ry[it] = y; rx[it] = x; rb[it] = b;
                    rbase[it] = (long long)m * g.C;
                }
            }
        }
        // loads of K chunk i into stage s (every thread: its A rows, then its share of B)
        auto load_stage = [&](int i, int s) {
            const int k = kb + i * kBK + kc_t * 8;
            int dy = 0, dx = 0, c = k;
            if (g.a_mode != 0) {  // both convolution modes: tap (ky, kx) and channel of k
                const int tap = k / g.C;
                c = k - tap * g.C;
                dy = tap / 3 - 1;
                dx = tap - 3 * (tap / 3) - 1;
            }
            const bool kin = k < g.K;
#pragma unroll
            for (int it = 0; it < kRowsPerThread; ++it) {
                const int r = map_row(it, tid);
                const __nv_bfloat16 *src = g.A;
                int bytes = 0;
                if (kin && ry[it] >= 0) {
                    if (g.a_mode == 0) {
                        src = g.A + rbase[it] + k;
                        bytes = 16;
                    } else {
                        const int yy = ry[it] + dy, xx = rx[it] + dx;
                        if (yy >= 0 && yy < g.H && xx >= 0 && xx < g.W) {
                            if (g.a_mode == 1) {
                                src = g.A + rbase[it] + ((long long)dy * g.W + dx) * g.C + c;
                            } else if (c < g.Cu) {  // the coarse tensor's pixel (yy / 2, xx / 2)
                                src = g.A + (((long long)rb[it] * (g.H >> 1) + (yy >> 1)) * (g.W >> 1) + (xx >> 1)) * g.Cu + c;
                            } else {
                                src = g.A2 + (((long long)rb[it] * g.H + yy) * g.W + xx) * Cs + (c - g.Cu);
                            }
                            bytes = 16;
                        }
                    }
                }
                cp_async16(sA0 + s * kStageA + tile_off(r, kc_t), src, bytes);
            }
#pragma unroll
            for (int it = 0; it < (BN * 8 + kGemmThreads - 1) / kGemmThreads; ++it) {
                const int cc = it * kGemmThreads + tid;
                if (cc >= BN * 8) break;
                const int r = (cc & 7) + ((cc >> 6) << 3), kcb = (cc >> 3) & 7;
                const int n = n0 + r, kk = kb + i * kBK + kcb * 8;
                const bool ok = n < g.N && kk < ke;
                cp_async16(sB0 + s * kStageB + tile_off(r, kcb), ok ? (const void *)(g.B + (long long)n * g.ldb + kk) : g.B,
                           ok ? 16 : 0);
            }
        };
        // prologue: chunks 0 .. kStages-2 in flight.  Every stage's MMAs of the previous tile are complete
        // (the previous tile waited for all of them before its epilogue), so no stage needs a wait here.
#pragma unroll
        for (int s = 0; s < kDepth; ++s) {
            if (s < nk) load_stage(s, s);
            cp_async_commit();
        }
        for (int i = 0; i < nk; ++i) {
            const int s = i % kStages;
            cp_async_wait<kDepth - 1>();  // this thread's copies of chunk i have landed
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();  // ... and every thread's
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t a0 = sA0 + s * kStageA, b0 = sB0 + s * kStageB;
#pragma unroll
                for (int ks = 0; ks < kBK / 16; ++ks) {
                    const uint64_t da = umma_desc(a0 + ks * 256, 128, 1024);
                    const uint64_t db = umma_desc(b0 + ks * 256, 128, 1024);
                    const uint32_t acc = (i > 0 || ks > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        :
                        : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&bar[s]))
                             : "memory");
                ++commits[s];
                // the stage the next load refills held chunk i + kDepth - kStages: its MMAs must be done
                const int sp = (i + kDepth) % kStages;
                if (i + kDepth >= kStages && i + kDepth < nk && !mbar_wait(smem_u32(&bar[sp]), (commits[sp] - 1) & 1))
                    abort_flag = 1;
            }
            if (i + kDepth < nk) {
                __syncthreads();
                if (abort_flag) break;
                load_stage(i + kDepth, (i + kDepth) % kStages);
            }
            cp_async_commit();
        }
        cp_async_wait<0>();
        // every stage's last commit (the last one covers all earlier MMAs of the issuing thread)
        if (tid == 0) {
            bool ok = true;
            for (int s = 0; s < kStages && ok; ++s)
                if (commits[s] && !mbar_wait(smem_u32(&bar[s]), (commits[s] - 1) & 1)) ok = false;
            if (!ok) abort_flag = 1;
        }
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        failed = abort_flag != 0;
        if (failed) break;
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (tile rows); warps 0-3 take column blocks
        // 0, 64, ..., warps 4-7 blocks 32, 96, ...  A 32 x 32 block goes through this warp's staging area of
        // the (now idle) A stages -- row stride 33 words, so the row-wise writes and the chunk-wise reads are
        // both free of bank conflicts -- and leaves in 16-byte row chunks: one store instruction covers whole
        // 64-byte (bf16) or 128-byte (fp32) row segments instead of 32 scattered rows.
        float *stg = reinterpret_cast<float *>(smA) + warp * (32 * 33);
        const int rbase0 = m0 + (warp & 3) * 32;
        if (nk > 0) {
#pragma unroll 1
            for (int c0 = (warp >> 2) * 32; c0 < BN; c0 += 64) {
                uint32_t r[32];
                const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                    "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                      "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                      "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int nb = n0 + c0;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    float v = __uint_as_float(r[j]);
                    if (g.bias && nb + j < g.N) v += g.bias[nb + j];
                    if (direct_bf16 && g.relu) v = fmaxf(v, 0.f);
                    stg[lane * 33 + j] = v;
                }
                __syncwarp();
                if (direct_bf16) {
                    // 32 rows x 4 chunks of 8 columns
                    const bool vec = ((g.ldo & 7) == 0) && ((reinterpret_cast<uintptr_t>(g.out_bf16) & 15) == 0);
#pragma unroll
                    for (int it = 0; it < 4; ++it) {
                        const int q = it * 32 + lane, rr = q >> 2, part = q & 3;
                        const int m = rbase0 + rr, n = nb + part * 8;
                        if (m >= g.M || n >= g.N) continue;
                        const float *src = stg + rr * 33 + part * 8;
                        __nv_bfloat16 *o = g.out_bf16 + (long long)m * g.ldo + n;
                        if (vec && n + 8 <= g.N) {
                            uint4 w;
                            __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&w);
#pragma unroll
                            for (int e = 0; e < 4; ++e) h[e] = __floats2bfloat162_rn(src[2 * e], src[2 * e + 1]);
                            *reinterpret_cast<uint4 *>(o) = w;
                        } else {
                            for (int e = 0; e < 8 && n + e < g.N; ++e) o[e] = __float2bfloat16_rn(src[e]);
                        }
                    }
                } else {
                    // 32 rows x 8 chunks of 4 columns
                    float *base = g.out + (long long)blockIdx.z * g.split_stride;
                    const bool vec = ((g.ldc & 3) == 0) && ((g.split_stride & 3) == 0) &&
                                     ((reinterpret_cast<uintptr_t>(g.out) & 15) == 0);
#pragma unroll
                    for (int it = 0; it < 8; ++it) {
                        const int q = it * 32 + lane, rr = q >> 3, part = q & 7;
                        const int m = rbase0 + rr, n = nb + part * 4;
                        if (m >= g.M || n >= g.N) continue;
                        const float *src = stg + rr * 33 + part * 4;
                        float *o = base + (long long)m * g.ldc + n;
                        if (vec && n + 4 <= g.N) {
                            *reinterpret_cast<float4 *>(o) = make_float4(src[0], src[1], src[2], src[3]);
                        } else {
                            for (int e = 0; e < 4 && n + e < g.N; ++e) o[e] = src[e];
                        }
                    }
                }
                __syncwarp();
            }
        } else if (!direct_bf16 && warp < 4 && rbase0 + lane < g.M) {  // an empty K range contributes zeros
            float *o = g.out + (long long)blockIdx.z * g.split_stride + (long long)(rbase0 + lane) * g.ldc;
            for (int n = n0; n < min(g.N, n0 + BN); ++n) o[n] = 0.f;
        }
        // the next tile's first MMA overwrites the accumulator: every TMEM read of this tile precedes it
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    if (failed && tid == 0 && g.error) atomicExch(g.error, kTimeoutCode);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// Split-K partials of a convolution summed in a fixed order, plus bias and ReLU, rounded to bf16:
// out[m * ldo + n] = bf16(relu?(sum_z part[z][m][n] + bias[n])).  (A fused variant in which the last CTA of a
// tile reduces measured slower: that CTA's serial reduction lies on the layer's critical path.)
__global__ void k_umma_split_epilogue(const float *__restrict__ part, int splits, long long M, int N,
                                      const float *__restrict__ bias, int relu, __nv_bfloat16 *__restrict__ out,
                                      long long ldo) {
    pdl_wait();
    pdl_release();
    const long long n_all = M * N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_all; i += (long long)gridDim.x * blockDim.x) {
        float v = 0.f;
        for (int z = 0; z < splits; ++z) v += part[(long long)z * n_all + i];
        const int n = (int)(i % N);
        v += bias ? bias[n] : 0.f;
        if (relu) v = fmaxf(v, 0.f);
        out[(i / N) * ldo + n] = __float2bfloat16_rn(v);
    }
}

inline size_t umma_smem_bytes(int bn) { return kStages * ((size_t)(kBM * kBK * 2) + (size_t)(bn * kBK * 2)); }

}  // namespace nn
}  // namespace octo
