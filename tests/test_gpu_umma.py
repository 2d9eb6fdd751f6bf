"""The tensor-core GEMM (tcgen05.mma, TMEM accumulator) behind the learned field correction, against a
plain PyTorch fp32 product of the same bf16-rounded operands: dense A, the implicit im2col of a 3x3
convolution (against torch's conv2d), split-K partials, and the fused bias + ReLU bf16 epilogue.  The
tolerance is fp32 accumulation-order rounding: |got - ref| <= 2e-6 * sum_k |a_mk b_nk| + 1e-30."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _gemm(desc):
    import torch
    from octo_b200 import _lib
    rc = _lib.lib().octo_gemm_bf16(0, C.byref(desc), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.OCTO_OK, rc


def _desc(**kw):
    from octo_b200 import _lib
    d = _lib.OctoGemmDesc()
    d.splits = 1
    for k, v in kw.items():
        setattr(d, k, v)
    return d


def _check(got, ref, bound):
    import torch
    err = (got - ref).abs() - (2e-6 * bound + 1e-30)
    assert float(err.max()) <= 0.0, float(((got - ref).abs() / (bound + 1e-30)).max())


@pytest.mark.parametrize("M,N,K,splits", [(128, 32, 64, 1), (300, 40, 72, 1), (1000, 96, 136, 1),
                                          (256, 256, 1024, 1), (513, 200, 640, 3), (129, 16, 4096, 8)])
def test_dense_gemm_matches_torch(M, N, K, splits):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    out = torch.full((splits, M, N), float("nan"), device="cuda")
    _gemm(_desc(M=M, N=N, K=K, splits=splits, A=A.data_ptr(), lda=K, B=B.data_ptr(), ldb=K, out=out.data_ptr(),
                ldc=N))
    torch.cuda.synchronize()
    ref = A.float() @ B.float().T
    bound = A.float().abs() @ B.float().abs().T
    _check(out.sum(0), ref, bound)


@pytest.mark.parametrize("Bn,H,W,Cin,Cout", [(2, 48, 48, 8, 32), (3, 24, 24, 32, 64), (1, 12, 12, 64, 128),
                                             (2, 6, 6, 128, 128), (1, 7, 5, 16, 24)])
def test_implicit_conv3x3_matches_torch(Bn, H, W, Cin, Cout):
    import torch
    import torch.nn.functional as F
    g = torch.Generator(device="cuda").manual_seed(H * Cin + Cout)
    X = torch.randn(Bn, H, W, Cin, device="cuda", generator=g).to(torch.bfloat16)       # NHWC
    Wt = torch.randn(Cout, 3, 3, Cin, device="cuda", generator=g).to(torch.bfloat16)   # [Cout][ky][kx][Cin]
    M, K = Bn * H * W, 9 * Cin
    out = torch.empty(M, Cout, device="cuda")
    _gemm(_desc(M=M, N=Cout, K=K, a_mode=1, H=H, W=W, C=Cin, A=X.data_ptr(), B=Wt.data_ptr(), ldb=K,
                out=out.data_ptr(), ldc=Cout))
    torch.cuda.synchronize()
    xin = X.float().permute(0, 3, 1, 2)
    w = Wt.float().permute(0, 3, 1, 2)
    ref = F.conv2d(xin, w, padding=1).permute(0, 2, 3, 1).reshape(M, Cout)
    bound = F.conv2d(xin.abs(), w.abs(), padding=1).permute(0, 2, 3, 1).reshape(M, Cout)
    _check(out, ref, bound)


def test_bias_relu_bf16_epilogue():
    import torch
    M, N, K = 700, 64, 288
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    o = torch.zeros(M, N, device="cuda", dtype=torch.bfloat16)
    _gemm(_desc(M=M, N=N, K=K, A=A.data_ptr(), lda=K, B=B.data_ptr(), ldb=K, bias=bias.data_ptr(), relu=1,
                out_bf16=o.data_ptr(), ldo=N))
    torch.cuda.synchronize()
    ref = torch.relu(A.float() @ B.float().T + bias)
    # one bf16 rounding of the result (2^-8 relative) on top of the fp32 accumulation
    assert float(((o.float() - ref).abs() - 2 ** -8 * ref.abs() - 1e-3).max()) <= 0.0
