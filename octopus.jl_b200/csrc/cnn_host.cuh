// Host side of the learned field correction's CNN: parameters, device buffers, and the launch sequences of
// the forward pass, the backward pass and the Adam update.  Included by octo_b200.cu after DevBuf, CK,
// launch_pdl and launch_gemm.
//
// Network (a 4-level U-Net, 32 base channels, 3x3 convolutions with padding 1, ReLU, 2x2 average pooling,
// nearest upsampling with skip concatenation; 641k parameters):
//   level 0 (H x W):       e1a 8 -> 32, e1b 32 -> 32 (skip s1)
//   level 1 (H/2 x W/2):   e2a 32 -> 64, e2b 64 -> 64 (skip s2)
//   level 2 (H/4 x W/4):   e3a 64 -> 128, e3b 128 -> 128 (skip s3)
//   level 3 (H/8 x W/8):   b 128 -> 128
//   decoder: d3 [up(b), s3] 256 -> 64 (level 2), d2 [up(d3), s2] 128 -> 32 (level 1),
//            d1 [up(d2), s1] 64 -> 32 (level 0), head 32 -> 8 without ReLU (channels 0, 1 are the output).
// Parameters (fp32 master copy): per layer the weights [Cout][ky][kx][Cin] then the bias [Cout].
#pragma once
#include <random>

#include "k_cnn.cuh"
#include "k_umma.cuh"

namespace octo {
namespace nn {

struct LayerSpec {
    int cin, cout, level, relu;
};
constexpr int kCnnLayers = 11;
constexpr int kCnnIn = 8, kCnnOut = 8;
constexpr LayerSpec kLayers[kCnnLayers] = {
    {8, 32, 0, 1},    {32, 32, 0, 1},   {32, 64, 1, 1},  {64, 64, 1, 1},  {64, 128, 2, 1}, {128, 128, 2, 1},
    {128, 128, 3, 1}, {256, 64, 2, 1},  {128, 32, 1, 1}, {64, 32, 0, 1},  {32, 8, 0, 0},
};
enum { L_E1A, L_E1B, L_E2A, L_E2B, L_E3A, L_E3B, L_B, L_D3, L_D2, L_D1, L_HEAD };

inline long long round8(long long v) { return (v + 7) / 8 * 8; }
inline unsigned ew_blocks(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); }

struct Cnn {
    int device = 0, H = 0, W = 0, maxB = 0;
    long long nparams = 0;
    long long woff[kCnnLayers] = {0}, boff[kCnnLayers] = {0};
    DevBuf<float> master, grad, adam_m, adam_v;
    DevBuf<bf16> w[kCnnLayers], wf[kCnnLayers];
    // forward activations (NHWC bf16)
    DevBuf<bf16> x0, a0, s1, p1, a2, s2, p2, a4, s3, p3, b6, u3, d7, u2, d8, u1, d9;
    DevBuf<float> out;  // head output [M0][8]
    // backward scratch
    DevBuf<bf16> g, gt, colt;
    DevBuf<float> fa, dc, ds1, ds2, ds3, part, splitbuf;
    DevBuf<double> loss_part;
    PinBuf<double> h_loss;
    long long part_floats = 0;
    int adam_t = 0;
    bool weights_dirty = true;
    int *err = nullptr;

    int hl(int l) const { return H >> l; }
    int wl(int l) const { return W >> l; }
    long long ml(int l, int B) const { return (long long)B * hl(l) * wl(l); }

    void create(int dev, int h, int wd, int maxb, uint64_t seed) {
        device = dev; H = h; W = wd; maxB = maxb;
        CK(cudaSetDevice(device));
        long long off = 0;
        for (int l = 0; l < kCnnLayers; ++l) {
            woff[l] = off;
            off += (long long)kLayers[l].cout * 9 * kLayers[l].cin;
            boff[l] = off;
            off += kLayers[l].cout;
        }
        nparams = off;
        master.ensure(nparams); grad.ensure(nparams); adam_m.ensure(nparams); adam_v.ensure(nparams);
        CK(cudaMemset(adam_m.p, 0, sizeof(float) * nparams));
        CK(cudaMemset(adam_v.p, 0, sizeof(float) * nparams));
        CK(cudaMemset(grad.p, 0, sizeof(float) * nparams));
        for (int l = 0; l < kCnnLayers; ++l) {
            const long long n = (long long)kLayers[l].cout * 9 * kLayers[l].cin;
            w[l].ensure(n);
            if (l > 0) wf[l].ensure(n);
        }
        // He-normal initialisation (std sqrt(2 / fan_in)); the head starts small and its unused channels
        // 2..7 at zero (their outputs carry no loss, so they stay zero)
        std::vector<float> hp((size_t)nparams, 0.f);
        std::mt19937_64 rng(seed);
        std::normal_distribution<double> nd(0.0, 1.0);
        for (int l = 0; l < kCnnLayers; ++l) {
            const LayerSpec &L = kLayers[l];
            const double sd = std::sqrt(2.0 / (9.0 * L.cin)) * (l == L_HEAD ? 0.1 : 1.0);
            for (int co = 0; co < L.cout; ++co)
                for (int k = 0; k < 9 * L.cin; ++k) {
                    const double v = nd(rng) * sd;
                    if (l != L_HEAD || co < 2) hp[(size_t)(woff[l] + (long long)co * 9 * L.cin + k)] = (float)v;
                }
        }
        CK(cudaMemcpy(master.p, hp.data(), sizeof(float) * nparams, cudaMemcpyHostToDevice));
        const long long M0 = ml(0, maxB), M1 = ml(1, maxB), M2 = ml(2, maxB), M3 = ml(3, maxB);
        x0.ensure(M0 * 8); a0.ensure(M0 * 32); s1.ensure(M0 * 32); p1.ensure(M1 * 32);
        a2.ensure(M1 * 64); s2.ensure(M1 * 64); p2.ensure(M2 * 64);
        a4.ensure(M2 * 128); s3.ensure(M2 * 128); p3.ensure(M3 * 128);
        b6.ensure(M3 * 128); u3.ensure(M2 * 256); d7.ensure(M2 * 64); u2.ensure(M1 * 128); d8.ensure(M1 * 32);
        u1.ensure(M0 * 64); d9.ensure(M0 * 32); out.ensure(M0 * 8);
        const long long ld0 = round8(M0);
        g.ensure(M0 * 32); gt.ensure(32 * ld0 + 64); colt.ensure(576 * ld0 + 64);
        fa.ensure(M0 * 64); dc.ensure(M0 * 8 + 64); ds1.ensure(M0 * 32); ds2.ensure(M1 * 64); ds3.ensure(M2 * 128);
        long long pmax = 0;
        for (int l = 0; l < kCnnLayers; ++l) {
            const LayerSpec &L = kLayers[l];
            const int s = wgrad_splits(l, maxB);
            pmax = std::max(pmax, (long long)s * 9 * L.cin * L.cout);
        }
        part.ensure(pmax);
        part_floats = pmax;
        loss_part.ensure(2 * 1024);
        h_loss.ensure(2 * 1024);
        CK(cudaMalloc(&err, sizeof(int)));
        CK(cudaMemset(err, 0, sizeof(int)));
    }

    void release() {
        master.release(); grad.release(); adam_m.release(); adam_v.release();
        for (auto &b : w) b.release();
        for (auto &b : wf) b.release();
        for (DevBuf<bf16> *b : {&x0, &a0, &s1, &p1, &a2, &s2, &p2, &a4, &s3, &p3, &b6, &u3, &d7, &u2, &d8, &u1, &d9, &g, &gt, &colt})
            b->release();
        for (DevBuf<float> *b : {&out, &fa, &dc, &ds1, &ds2, &ds3, &part, &splitbuf}) b->release();
        loss_part.release();
        h_loss.release();
        if (err) cudaFree(err);
        err = nullptr;
    }

    // split-K count of a layer's weight-gradient GEMM: about two waves of CTAs over the GPU
    int wgrad_splits(int l, int B) const {
        const LayerSpec &L = kLayers[l];
        const long long K = round8(ml(L.level, B));
        const int bn = L.cout <= 32 ? 32 : (L.cout <= 64 ? 64 : (L.cout <= 128 ? 128 : 256));
        const long long tiles = ((9LL * L.cin + kBM - 1) / kBM) * ((L.cout + bn - 1) / bn);
        const long long chunks = (K + kBK - 1) / kBK;
        return (int)std::max<long long>(1, std::min<long long>(chunks, (296 + tiles - 1) / tiles));
    }

    void refresh_weights(cudaStream_t st) {
        for (int l = 0; l < kCnnLayers; ++l) {
            const LayerSpec &L = kLayers[l];
            const int n = L.cout * 9 * L.cin;
            launch_pdl(k_cnn_weights, ew_blocks(n), 256, 0, st, (const float *)(master.p + woff[l]), L.cout, L.cin, w[l].p,
                       l > 0 ? wf[l].p : (bf16 *)nullptr);
        }
        weights_dirty = false;
    }

    // A 3x3 convolution layer as one tensor-core GEMM.  Layers with too few output tiles to fill the GPU (the
    // coarse levels) split K over more CTAs; their fp32 partials are summed in a fixed order by the
    // bias / ReLU / bf16 epilogue kernel.
    // skip != null: the layer's input is [nearest-upsampled in (cu channels), skip] (a decoder level), read
    // by the GEMM directly instead of a materialised concatenation.
    void gemm_conv(int l, const bf16 *in, int B, bf16 *out_bf, float *out_f, cudaStream_t st, const bf16 *skip = nullptr,
                   int cu = 0) {
        const LayerSpec &L = kLayers[l];
        GemmArgs a{};
        a.M = (int)ml(L.level, B); a.N = L.cout; a.K = 9 * L.cin;
        a.A = in; a.a_mode = skip ? 2 : 1; a.H = hl(L.level); a.W = wl(L.level); a.C = L.cin;
        a.A2 = skip; a.Cu = cu;
        a.B = w[l].p; a.ldb = 9 * L.cin;
        a.bias = master.p + boff[l];
        a.relu = L.relu;
        a.out_bf16 = out_bf; a.ldo = L.cout;
        a.out = out_f; a.ldc = L.cout; a.split_stride = 0; a.k_per_split = ((a.K + kBK - 1) / kBK) * kBK;
        a.error = err;
        const int bn = L.cout <= 32 ? 32 : (L.cout <= 64 ? 64 : (L.cout <= 128 ? 128 : 256));
        const long long tiles = ((long long)(a.M + kBM - 1) / kBM) * ((L.cout + bn - 1) / bn);
        const int chunks = (a.K + kBK - 1) / kBK;
        const int splits = (out_bf && tiles < 148 && chunks >= 4)
                               ? (int)std::min<long long>(chunks / 2, (296 + tiles - 1) / tiles) : 1;
        if (splits <= 1) {
            launch_gemm(a, 1, st);
            return;
        }
        a.k_per_split = ((chunks + splits - 1) / splits) * kBK;
        const int used = (chunks * kBK + a.k_per_split - 1) / a.k_per_split;
        splitbuf.ensure((size_t)used * a.M * L.cout);
        a.out = splitbuf.p; a.ldc = L.cout; a.split_stride = (long long)a.M * L.cout;
        a.out_bf16 = nullptr; a.bias = nullptr; a.relu = 0;
        launch_gemm(a, used, st);
        launch_pdl(k_umma_split_epilogue, ew_blocks((long long)a.M * L.cout), 256, 0, st, (const float *)splitbuf.p, used,
                   (long long)a.M, L.cout, (const float *)(master.p + boff[l]), L.relu, out_bf, (long long)L.cout);
    }

    void pool(const bf16 *in, bf16 *o, int B, int level, int C, cudaStream_t st) {
        const long long n = ml(level + 1, B) * C;
        launch_pdl(k_cnn_pool, ew_blocks(n), 256, 0, st, in, o, B, hl(level), wl(level), C);
    }
    void upcat(const bf16 *coarse, const bf16 *skip, bf16 *o, int B, int level, int Cu, int Cs, cudaStream_t st) {
        const long long n = ml(level, B) * (Cu + Cs);
        launch_pdl(k_cnn_upcat, ew_blocks(n), 256, 0, st, coarse, skip, o, B, hl(level), wl(level), Cu, Cs);
    }

    // Forward pass of B inputs already in x0; the head's fp32 output lands in `out` ([M0][8]).  Inference
    // (materialize = false) reads each decoder level's [upsampled, skip] input inside the GEMM; training keeps
    // the concatenations, whose transposed im2col the weight gradients read.
    void forward(int B, cudaStream_t st, bool materialize = true) {
        if (weights_dirty) refresh_weights(st);
        if (!materialize) {
            gemm_conv(L_E1A, x0.p, B, a0.p, nullptr, st);
            gemm_conv(L_E1B, a0.p, B, s1.p, nullptr, st);
            pool(s1.p, p1.p, B, 0, 32, st);
            gemm_conv(L_E2A, p1.p, B, a2.p, nullptr, st);
            gemm_conv(L_E2B, a2.p, B, s2.p, nullptr, st);
            pool(s2.p, p2.p, B, 1, 64, st);
            gemm_conv(L_E3A, p2.p, B, a4.p, nullptr, st);
            gemm_conv(L_E3B, a4.p, B, s3.p, nullptr, st);
            pool(s3.p, p3.p, B, 2, 128, st);
            gemm_conv(L_B, p3.p, B, b6.p, nullptr, st);
            gemm_conv(L_D3, b6.p, B, d7.p, nullptr, st, s3.p, 128);
            gemm_conv(L_D2, d7.p, B, d8.p, nullptr, st, s2.p, 64);
            gemm_conv(L_D1, d8.p, B, d9.p, nullptr, st, s1.p, 32);
            gemm_conv(L_HEAD, d9.p, B, nullptr, out.p, st);
            return;
        }
        gemm_conv(L_E1A, x0.p, B, a0.p, nullptr, st);
        gemm_conv(L_E1B, a0.p, B, s1.p, nullptr, st);
        pool(s1.p, p1.p, B, 0, 32, st);
        gemm_conv(L_E2A, p1.p, B, a2.p, nullptr, st);
        gemm_conv(L_E2B, a2.p, B, s2.p, nullptr, st);
        pool(s2.p, p2.p, B, 1, 64, st);
        gemm_conv(L_E3A, p2.p, B, a4.p, nullptr, st);
        gemm_conv(L_E3B, a4.p, B, s3.p, nullptr, st);
        pool(s3.p, p3.p, B, 2, 128, st);
        gemm_conv(L_B, p3.p, B, b6.p, nullptr, st);
        upcat(b6.p, s3.p, u3.p, B, 2, 128, 128, st);
        gemm_conv(L_D3, u3.p, B, d7.p, nullptr, st);
        upcat(d7.p, s2.p, u2.p, B, 1, 64, 64, st);
        gemm_conv(L_D2, u2.p, B, d8.p, nullptr, st);
        upcat(d8.p, s1.p, u1.p, B, 0, 32, 32, st);
        gemm_conv(L_D1, u1.p, B, d9.p, nullptr, st);
        gemm_conv(L_HEAD, d9.p, B, nullptr, out.p, st);
    }

    // Weight and bias gradients of layer l from its input activation and the bf16 output gradient in g.
    void wgrad(int l, const bf16 *in, int B, cudaStream_t st) {
        const LayerSpec &L = kLayers[l];
        const long long M = ml(L.level, B), ld = round8(M);
        const int hh = hl(L.level), ww = wl(L.level);
        launch_pdl(k_cnn_transpose, dim3((unsigned)((ld + 31) / 32), (unsigned)((L.cout + 31) / 32)), dim3(32, 8), 0, st,
                   (const bf16 *)g.p, gt.p, M, L.cout, ld);
        launch_pdl(k_cnn_im2col_t, ew_blocks(9LL * L.cin * ld), 256, 0, st, in, colt.p, B, hh, ww, L.cin, ld);
        const int splits = wgrad_splits(l, B);
        GemmArgs a{};
        a.M = 9 * L.cin; a.N = L.cout; a.K = (int)ld;
        a.A = colt.p; a.lda = ld; a.a_mode = 0;
        a.B = gt.p; a.ldb = ld;
        a.out = part.p; a.ldc = L.cout; a.split_stride = (long long)a.M * L.cout;
        const long long chunks = (ld + kBK - 1) / kBK;
        a.k_per_split = (int)(((chunks + splits - 1) / splits) * kBK);
        a.error = err;
        const int used = (int)((chunks * kBK + a.k_per_split - 1) / a.k_per_split);
        launch_gemm(a, used, st);
        const long long n = (long long)a.M * L.cout;
        launch_pdl(k_cnn_wgrad_reduce, ew_blocks(n), 256, 0, st, (const float *)part.p, used, a.M, L.cout, grad.p + woff[l]);
        launch_pdl(k_cnn_bias_grad, L.cout, 256, 0, st, (const bf16 *)g.p, M, L.cout, grad.p + boff[l]);
    }

    // Input gradient of layer l (fp32, into fa) from the bf16 output gradient in g.
    void dgrad(int l, int B, cudaStream_t st) {
        const LayerSpec &L = kLayers[l];
        GemmArgs a{};
        a.M = (int)ml(L.level, B); a.N = L.cin; a.K = 9 * L.cout;
        a.A = g.p; a.a_mode = 1; a.H = hl(L.level); a.W = wl(L.level); a.C = L.cout;
        a.B = wf[l].p; a.ldb = 9 * L.cout;
        a.out = fa.p; a.ldc = L.cin; a.split_stride = 0; a.k_per_split = ((a.K + kBK - 1) / kBK) * kBK;
        a.error = err;
        launch_gemm(a, 1, st);
    }
    void relu_grad(const float *dy, const bf16 *y, long long n, cudaStream_t st) {
        launch_pdl(k_cnn_relu_grad, ew_blocks(n), 256, 0, st, dy, y, g.p, n);
    }

    // Loss of the last forward pass against target ([M0][2]) with per-pixel weights mask (null = 1),
    // normalised by the total weight; then the gradients of every parameter into `grad`.  Returns the
    // partial-sum count; the host folds loss_part.
    int backward(int B, const float *target, const float *mask, double weight_total, cudaStream_t st) {
        const long long M0 = ml(0, B), M1 = ml(1, B), M2 = ml(2, B), M3 = ml(3, B);
        const int nblk = (int)std::min<long long>(1024, (M0 + 255) / 256);
        const float scale = (float)(1.0 / (2.0 * std::max(weight_total, 1e-300)));  // mean over 2 channels
        launch_pdl(k_cnn_loss, nblk, 256, 0, st, (const float *)out.p, target, mask, M0, scale, g.p, loss_part.p);
        // head
        wgrad(L_HEAD, d9.p, B, st);
        dgrad(L_HEAD, B, st);
        relu_grad(fa.p, d9.p, M0 * 32, st);
        // d1: input [up(d2), s1]
        wgrad(L_D1, u1.p, B, st);
        dgrad(L_D1, B, st);
        launch_pdl(k_cnn_upcat_adj, ew_blocks(M1 * 32 + M0 * 32), 256, 0, st, (const float *)fa.p, dc.p, ds1.p, B, hl(0), wl(0), 32,
                   32, 0);
        relu_grad(dc.p, d8.p, M1 * 32, st);
        // d2: input [up(d3), s2]
        wgrad(L_D2, u2.p, B, st);
        dgrad(L_D2, B, st);
        launch_pdl(k_cnn_upcat_adj, ew_blocks(M2 * 64 + M1 * 64), 256, 0, st, (const float *)fa.p, dc.p, ds2.p, B, hl(1), wl(1), 64,
                   64, 0);
        relu_grad(dc.p, d7.p, M2 * 64, st);
        // d3: input [up(b), s3]
        wgrad(L_D3, u3.p, B, st);
        dgrad(L_D3, B, st);
        launch_pdl(k_cnn_upcat_adj, ew_blocks(M3 * 128 + M2 * 128), 256, 0, st, (const float *)fa.p, dc.p, ds3.p, B, hl(2), wl(2),
                   128, 128, 0);
        relu_grad(dc.p, b6.p, M3 * 128, st);
        // b: input pool(s3)
        wgrad(L_B, p3.p, B, st);
        dgrad(L_B, B, st);
        launch_pdl(k_cnn_pool_adj_add, ew_blocks(M2 * 128), 256, 0, st, (const float *)fa.p, ds3.p, B, hl(2), wl(2), 128);
        relu_grad(ds3.p, s3.p, M2 * 128, st);
        // e3b, e3a
        wgrad(L_E3B, a4.p, B, st);
        dgrad(L_E3B, B, st);
        relu_grad(fa.p, a4.p, M2 * 128, st);
        wgrad(L_E3A, p2.p, B, st);
        dgrad(L_E3A, B, st);
        launch_pdl(k_cnn_pool_adj_add, ew_blocks(M1 * 64), 256, 0, st, (const float *)fa.p, ds2.p, B, hl(1), wl(1), 64);
        relu_grad(ds2.p, s2.p, M1 * 64, st);
        // e2b, e2a
        wgrad(L_E2B, a2.p, B, st);
        dgrad(L_E2B, B, st);
        relu_grad(fa.p, a2.p, M1 * 64, st);
        wgrad(L_E2A, p1.p, B, st);
        dgrad(L_E2A, B, st);
        launch_pdl(k_cnn_pool_adj_add, ew_blocks(M0 * 32), 256, 0, st, (const float *)fa.p, ds1.p, B, hl(0), wl(0), 32);
        relu_grad(ds1.p, s1.p, M0 * 32, st);
        // e1b, e1a
        wgrad(L_E1B, a0.p, B, st);
        dgrad(L_E1B, B, st);
        relu_grad(fa.p, a0.p, M0 * 32, st);
        wgrad(L_E1A, x0.p, B, st);
        return nblk;
    }

    void adam(float lr, cudaStream_t st) {
        ++adam_t;
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        const float c1 = (float)(1.0 - std::pow((double)b1, adam_t)), c2 = (float)(1.0 - std::pow((double)b2, adam_t));
        launch_pdl(k_cnn_adam, ew_blocks(nparams), 256, 0, st, master.p, (const float *)grad.p, adam_m.p, adam_v.p, nparams, lr, b1,
                   b2, eps, c1, c2);
        weights_dirty = true;
    }
};

}  // namespace nn
}  // namespace octo
