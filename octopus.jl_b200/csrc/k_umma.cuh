// BF16 GEMM on the fifth-generation tensor cores (tcgen05 / UMMA), the contraction behind the learned
// field correction's convolutions (forward, input gradient, weight gradient).
//
//   C[M, N] (fp32) = sum_k A[m, k] * B[n, k]            (both operands K-major)
//
// A is either a dense row-major bf16 matrix or, for a 3x3 convolution with padding 1, the implicit im2col
// of an NHWC bf16 activation tensor (row m = pixel (b, y, x), column k = (ky * 3 + kx) * C + c); B is a
// row-major bf16 matrix (for a convolution: weights [Cout][ky][kx][Cin]).
//
// One CTA of 128 threads computes a 128 x BN tile: the K loop moves 64-wide chunks of A and B from global
// memory into shared memory (two stages) in the canonical no-swizzle K-major layout -- 8-row x 16-byte core
// matrices, 128 contiguous bytes each, the two K halves of one instruction LBO = 128 bytes apart and 8-row
// groups SBO = 1024 bytes apart -- and one thread issues four tcgen05.mma (M = 128, N = BN, K = 16) per
// chunk into a TMEM accumulator, committing each chunk to the stage's mbarrier so the stage can be refilled
// while the next chunk's MMAs run.  The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31 = tile rows) and writes fp32 (split-K partials) or bias + ReLU as bf16.
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
constexpr int kGemmThreads = 128;
constexpr int kTimeoutCode = 6;  // OCTO_ERR_TIMEOUT

struct GemmArgs {
    int M, N, K;                  // K a multiple of 8
    const __nv_bfloat16 *A;       // a_mode 0: A[m * lda + k]
    long long lda;
    int a_mode;                   // 0 dense, 1 implicit 3x3 / pad-1 convolution of an NHWC tensor
    int H, W, C;                  // a_mode 1: input height, width, channels (C a multiple of 8); K = 9 C
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

// One 16-byte chunk (8 consecutive k) of row m of A, or zeros outside the matrix / the padded image.
__device__ __forceinline__ uint4 load_a_chunk(const GemmArgs &g, int m, int k) {
    uint4 v = make_uint4(0, 0, 0, 0);
    if (m >= g.M || k >= g.K) return v;
    if (g.a_mode == 0) return *reinterpret_cast<const uint4 *>(g.A + (long long)m * g.lda + k);
    const int tap = k / g.C, c = k - tap * g.C;
    const int hw = g.H * g.W;
    const int b = m / hw, rem = m - b * hw, y = rem / g.W, x = rem - y * g.W;
    const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
    if (yy < 0 || yy >= g.H || xx < 0 || xx >= g.W) return v;
    return *reinterpret_cast<const uint4 *>(g.A + (((long long)b * g.H + yy) * g.W + xx) * g.C + c);
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1) k_umma_gemm(const GemmArgs g) {
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "BN");
    constexpr uint32_t kStageA = kBM * kBK * 2, kStageB = BN * kBK * 2;
    constexpr uint32_t kCols = BN < 32 ? 32 : BN;
    extern __shared__ __align__(1024) unsigned char g_umma_smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    pdl_wait();
    pdl_release();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * g.k_per_split;
    const int ke = min(g.K, kb + g.k_per_split);
    const int nk = ke > kb ? (ke - kb + kBK - 1) / kBK : 0;
    unsigned char *const smA = g_umma_smem, *const smB = g_umma_smem + 2 * kStageA;  // stage s at + s * size
    if (tid == 0) {
        for (int s = 0; s < 2; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[s])));
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
    uint32_t commits[2] = {0, 0};  // commits issued per stage (thread 0)

    for (int i = 0; i < nk; ++i) {
        const int s = i & 1;
        if (i >= 2) {  // the MMAs that read this stage (chunk i - 2) must be done before it is refilled
            if (tid == 0 && !mbar_wait(smem_u32(&bar[s]), (commits[s] - 1) & 1)) abort_flag = 1;
            __syncthreads();
            if (abort_flag) break;
        }
        const int k0 = kb + i * kBK;
        // A: 128 rows x 8 chunks; a group of 8 consecutive threads writes 8 rows of one k-chunk (128
        // contiguous bytes of shared memory, conflict-free)
#pragma unroll
        for (int it = 0; it < (kBM * 8) / kGemmThreads; ++it) {
            const int c = it * kGemmThreads + tid;
            const int r = (c & 7) + ((c >> 6) << 3), kc = (c >> 3) & 7;
            const uint4 v = load_a_chunk(g, m0 + r, k0 + kc * 8);
            *reinterpret_cast<uint4 *>(smA + s * kStageA + tile_off(r, kc)) = v;
        }
#pragma unroll
        for (int it = 0; it < (BN * 8 + kGemmThreads - 1) / kGemmThreads; ++it) {
            const int c = it * kGemmThreads + tid;
            if (c >= BN * 8) break;
            const int r = (c & 7) + ((c >> 6) << 3), kc = (c >> 3) & 7;
            const int n = n0 + r, k = k0 + kc * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (n < g.N && k < ke) v = *reinterpret_cast<const uint4 *>(g.B + (long long)n * g.ldb + k);
            *reinterpret_cast<uint4 *>(smB + s * kStageB + tile_off(r, kc)) = v;
        }
        // A chunks past this split's K range read zeros too: load_a_chunk tests k < K; within the range
        // the split boundary is a multiple of kBK, so only the last split has a tail
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(smA + s * kStageA), b0 = smem_u32(smB + s * kStageB);
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
        }
    }
    // wait for every stage's last commit (the last one covers all earlier MMAs of the issuing thread)
    if (tid == 0) {
        bool ok = true;
        for (int s = 0; s < 2; ++s)
            if (commits[s] && !mbar_wait(smem_u32(&bar[s]), (commits[s] - 1) & 1)) ok = false;
        if (!ok) abort_flag = 1;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const bool failed = abort_flag != 0;
    if (failed) {
        if (tid == 0 && g.error) atomicExch(g.error, kTimeoutCode);
    } else if (nk > 0) {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
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
            if (row < g.M) {
                if (g.out_bf16) {
                    __nv_bfloat16 *o = g.out_bf16 + (long long)row * g.ldo + n0 + c0;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int n = n0 + c0 + j;
                        if (n < g.N) {
                            float v = __uint_as_float(r[j]) + (g.bias ? g.bias[n] : 0.f);
                            if (g.relu) v = fmaxf(v, 0.f);
                            o[j] = __float2bfloat16_rn(v);
                        }
                    }
                } else {
                    float *o = g.out + (long long)blockIdx.z * g.split_stride + (long long)row * g.ldc + n0 + c0;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int n = n0 + c0 + j;
                        if (n < g.N) o[j] = __uint_as_float(r[j]) + (g.bias ? g.bias[n] : 0.f);
                    }
                }
            }
        }
    } else if (!g.out_bf16) {  // an empty K range contributes zeros
        const int row = m0 + warp * 32 + lane;
        if (row < g.M) {
            float *o = g.out + (long long)blockIdx.z * g.split_stride + (long long)row * g.ldc;
            for (int n = n0; n < min(g.N, n0 + BN); ++n) o[n] = 0.f;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

inline size_t umma_smem_bytes(int bn) { return 2 * (size_t)(kBM * kBK * 2) + 2 * (size_t)(bn * kBK * 2); }

}  // namespace nn
}  // namespace octo
