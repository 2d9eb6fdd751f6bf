// Element-wise and reduction kernels of the learned field correction's CNN (a 4-level U-Net of 3x3
// convolutions, 32 base channels).  The convolutions themselves are tensor-core GEMMs (k_umma.cuh); these
// kernels move activations between them: 2x2 average pooling, nearest upsampling with skip concatenation,
// the adjoints of both, ReLU masks, transposes and im2col for the weight gradients, the fixed-order
// reductions of the weight and bias gradients, the loss, and Adam.  Activations are NHWC bf16 with rows
// m = (b * H + y) * W + x; gradients are accumulated in fp32 and rounded to bf16 where a GEMM reads them.
// Every reduction folds in a fixed order, so a training step is deterministic.
#pragma once
#include <cuda_bf16.h>

#include "octo_internal.cuh"

namespace octo {
namespace nn {

using bf16 = __nv_bfloat16;

// out[b][y][x][c] = mean of the 2x2 block of in (H, W even).
__global__ void k_cnn_pool(const bf16 *__restrict__ in, bf16 *__restrict__ out, int B, int H, int W, int C) {
    pdl_wait();
    pdl_release();
    const int Ho = H / 2, Wo = W / 2;
    const long long n = (long long)B * Ho * Wo * C;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long p = i / C;
        const int x = (int)(p % Wo); p /= Wo;
        const int y = (int)(p % Ho);
        const int b = (int)(p / Ho);
        const long long r0 = (((long long)b * H + 2 * y) * W + 2 * x) * C + c;
        const float s = __bfloat162float(in[r0]) + __bfloat162float(in[r0 + C]) + __bfloat162float(in[r0 + (long long)W * C]) +
                        __bfloat162float(in[r0 + (long long)W * C + C]);
        out[i] = __float2bfloat16_rn(0.25f * s);
    }
}

// out[b][y][x][0..Cu) = coarse[b][y/2][x/2][..] (nearest upsampling), out[..][Cu..Cu+Cs) = skip[b][y][x][..].
__global__ void k_cnn_upcat(const bf16 *__restrict__ coarse, const bf16 *__restrict__ skip, bf16 *__restrict__ out, int B,
                            int H, int W, int Cu, int Cs) {
    pdl_wait();
    pdl_release();
    const int C = Cu + Cs;
    const long long n = (long long)B * H * W * C;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long p = i / C;
        if (c < Cu) {
            const int x = (int)(p % W);
            const long long q = p / W;
            const int y = (int)(q % H);
            const int b = (int)(q / H);
            out[i] = coarse[(((long long)b * (H / 2) + y / 2) * (W / 2) + x / 2) * Cu + c];
        } else {
            out[i] = skip[p * Cs + (c - Cu)];
        }
    }
}

// g = bf16(dy * (y > 0)): the gradient through a ReLU whose output y was stored.
__global__ void k_cnn_relu_grad(const float *__restrict__ dy, const bf16 *__restrict__ y, bf16 *__restrict__ g, long long n) {
    pdl_wait();
    pdl_release();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        g[i] = __float2bfloat16_rn(__bfloat162float(y[i]) > 0.f ? dy[i] : 0.f);
}

// Adjoint of k_cnn_upcat: dcoarse[b][y][x][c] = sum of the 2x2 fine children's du[..][c] (c < Cu), and
// dskip (fine) = du[..][Cu + c] (accumulate != 0: added to dskip).
__global__ void k_cnn_upcat_adj(const float *__restrict__ du, float *__restrict__ dcoarse, float *__restrict__ dskip, int B,
                                int H, int W, int Cu, int Cs, int accumulate) {
    pdl_wait();
    pdl_release();
    const int C = Cu + Cs, Hc = H / 2, Wc = W / 2;
    const long long nc = (long long)B * Hc * Wc * Cu, nf = (long long)B * H * W * Cs;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nc + nf; i += (long long)gridDim.x * blockDim.x) {
        if (i < nc) {
            const int c = (int)(i % Cu);
            long long p = i / Cu;
            const int x = (int)(p % Wc); p /= Wc;
            const int y = (int)(p % Hc);
            const int b = (int)(p / Hc);
            const long long f0 = (((long long)b * H + 2 * y) * W + 2 * x) * C + c;
            dcoarse[i] = (du[f0] + du[f0 + C]) + (du[f0 + (long long)W * C] + du[f0 + (long long)W * C + C]);
        } else {
            const long long j = i - nc;
            const int c = (int)(j % Cs);
            const long long p = j / Cs;
            const float v = du[p * C + Cu + c];
            dskip[j] = accumulate ? dskip[j] + v : v;
        }
    }
}

// Adjoint of k_cnn_pool added into the fine gradient: ds[child] += dp[parent] / 4.
__global__ void k_cnn_pool_adj_add(const float *__restrict__ dp, float *__restrict__ ds, int B, int H, int W, int C) {
    pdl_wait();
    pdl_release();
    const long long n = (long long)B * H * W * C;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long p = i / C;
        const int x = (int)(p % W); p /= W;
        const int y = (int)(p % H);
        const int b = (int)(p / H);
        ds[i] += 0.25f * dp[(((long long)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
    }
}

// out[c][m] = g[m][c] for m < M, zero for M <= m < ld (ld a multiple of 8).
__global__ void k_cnn_transpose(const bf16 *__restrict__ g, bf16 *__restrict__ out, long long M, int C, long long ld) {
    pdl_wait();
    pdl_release();
    __shared__ bf16 tile[32][33];
    const long long m0 = (long long)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const long long m = m0 + r;
        const int c = c0 + threadIdx.x;
        tile[r][threadIdx.x] = (m < M && c < C) ? g[m * C + c] : __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int c = c0 + r;
        const long long m = m0 + threadIdx.x;
        if (c < C && m < ld) out[(long long)c * ld + m] = tile[threadIdx.x][r];
    }
}

// Transposed im2col of a 3x3 / pad-1 convolution's NHWC input: out[(tap * C + c)][m] = x[pixel m shifted by
// tap][c] (zero outside the image and for M <= m < ld).
__global__ void k_cnn_im2col_t(const bf16 *__restrict__ x, bf16 *__restrict__ out, int B, int H, int W, int C, long long ld) {
    pdl_wait();
    pdl_release();
    const long long M = (long long)B * H * W;
    const long long n = (long long)9 * C * ld;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long m = i % ld;
        const long long row = i / ld;
        const int c = (int)(row % C), tap = (int)(row / C);
        bf16 v = __float2bfloat16_rn(0.f);
        if (m < M) {
            const int xx0 = (int)(m % W);
            const long long q = m / W;
            const int yy0 = (int)(q % H);
            const int b = (int)(q / H);
            const int yy = yy0 + tap / 3 - 1, xx = xx0 + tap % 3 - 1;
            if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = x[(((long long)b * H + yy) * W + xx) * C + c];
        }
        out[i] = v;
    }
}

// dW[co][k] = sum over split s (in order) of part[s][k][co]: the weight-gradient GEMM's split-K partials,
// transposed to the weights' [Cout][9 Cin] layout.
__global__ void k_cnn_wgrad_reduce(const float *__restrict__ part, int splits, int K9, int Cout, float *__restrict__ dw) {
    pdl_wait();
    pdl_release();
    const long long n = (long long)K9 * Cout;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int co = (int)(i % Cout);
        const long long k = i / Cout;
        float s = 0.f;
        for (int z = 0; z < splits; ++z) s += part[(long long)z * n + i];
        dw[(long long)co * K9 + k] = s;
    }
}

// db[c] = sum_m g[m][c], one block per channel, fixed-order tree.
__global__ void __launch_bounds__(256) k_cnn_bias_grad(const bf16 *__restrict__ g, long long M, int C, float *__restrict__ db) {
    pdl_wait();
    pdl_release();
    __shared__ float red[256];
    const int c = blockIdx.x;
    float s = 0.f;
    for (long long m = threadIdx.x; m < M; m += blockDim.x) s += __bfloat162float(g[m * C + c]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[c] = red[0];
}

// Weights of one layer from the fp32 master copy: w[co][tap][ci] as bf16, and the flipped transpose the input
// gradient's convolution uses: wf[ci][tap'][co] = w[co][8 - tap'][ci].
__global__ void k_cnn_weights(const float *__restrict__ master, int Cout, int Cin, bf16 *__restrict__ w, bf16 *__restrict__ wf) {
    pdl_wait();
    pdl_release();
    const int n = Cout * 9 * Cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ci = i % Cin, tap = (i / Cin) % 9, co = i / (9 * Cin);
        const bf16 v = __float2bfloat16_rn(master[i]);
        w[i] = v;
        if (wf) wf[((long long)ci * 9 + (8 - tap)) * Cout + co] = v;
    }
}

// Masked mean-square loss over output channels 0 and 1 of an 8-channel fp32 head: out[m][c] against
// target[m][c] (2 channels), weight mask[m] (null = 1).  Writes the loss gradient 2 w (out - target) * scale
// as bf16 (channels 2..7 zero) and per-block partial sums of w (out - target)^2 and of w.
__global__ void __launch_bounds__(256) k_cnn_loss(const float *__restrict__ out, const float *__restrict__ target,
                                                   const float *__restrict__ mask, long long M, float scale,
                                                   bf16 *__restrict__ dout, double *__restrict__ partial) {
    pdl_wait();
    pdl_release();
    __shared__ double red[2][256];
    double se = 0.0, sw = 0.0;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < M; m += (long long)gridDim.x * blockDim.x) {
        const float w = mask ? mask[m] : 1.f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float gv = 0.f;
            if (c < 2) {
                const float d = out[m * 8 + c] - target[m * 2 + c];
                se += (double)w * (double)d * (double)d;
                gv = 2.f * w * d * scale;
            }
            dout[m * 8 + c] = __float2bfloat16_rn(gv);
        }
        sw += (double)w;
    }
    red[0][threadIdx.x] = se;
    red[1][threadIdx.x] = sw;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if ((int)threadIdx.x < o) {
            red[0][threadIdx.x] += red[0][threadIdx.x + o];
            red[1][threadIdx.x] += red[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = red[0][0];
        partial[2 * blockIdx.x + 1] = red[1][0];
    }
}

// Adam (Kingma & Ba 2015) on the fp32 master parameters; bias corrections from the step count t.
__global__ void k_cnn_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m1, float *__restrict__ m2,
                           long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    pdl_wait();
    pdl_release();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float a = b1 * m1[i] + (1.f - b1) * gi;
        const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
        m1[i] = a;
        m2[i] = b;
        p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    }
}

}  // namespace nn
}  // namespace octo
