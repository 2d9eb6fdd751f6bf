"""The learned correction's network on the GPU against its CPU oracle (oracle/cnn_oracle.py, which mirrors the
product's bf16 rounding points and is itself pinned by finite differences in tests/test_cnn_oracle.py):
the forward output, the loss and the gradient of every parameter tensor, per tensor within 1e-2 relative
(L2 norm of the difference over the norm of the oracle's gradient; bf16 storage of activations and
gradients, fp32 versus float64 sums); and a few Adam steps lower the loss on a fixed batch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(B, H, W, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = np.zeros((B, H, W, 8), dtype=np.float32)
    x[..., 0] = rng.standard_normal((B, H, W))
    x[..., 1] = 0.5
    t = (0.2 * rng.standard_normal((B, H, W, 2))).astype(np.float32)
    mask = (rng.random((B, H, W)) > 0.1).astype(np.float32)
    xb = torch.from_numpy(x).to("cuda").to(torch.bfloat16)
    return xb, torch.from_numpy(t).cuda(), torch.from_numpy(mask).cuda()


def test_gradients_match_cpu_oracle():
    import torch
    from oracle import cnn_oracle as co
    from octo_b200.learned import FieldCorrectionNet
    B, H, W = 2, 48, 48
    net = FieldCorrectionNet(H, W, max_batch=4, seed=11)
    p = net.get_params()
    # the head's bias and some channels are zero at initialisation: give every parameter a value
    rng = np.random.default_rng(3)
    p = p + (0.01 * rng.standard_normal(p.size)).astype(np.float32)
    net.set_params(p)
    xb, t, mask = _inputs(B, H, W, 5)
    out = net.forward(xb).cpu().numpy()
    loss, g = net.train_step(xb, t, mask, update=False, want_grads=True)
    ref = co.Net(p.astype(np.float64), rounding=True)
    x64 = xb.float().cpu().numpy().astype(np.float64)
    loss_ref, g_ref = ref.loss_and_grads(x64, t.cpu().numpy().astype(np.float64), mask.cpu().numpy())
    out_ref = ref.st["out"][..., :2]
    assert np.linalg.norm(out - out_ref) / np.linalg.norm(out_ref) < 1e-2
    assert abs(loss / loss_ref - 1) < 1e-3, (loss, loss_ref)
    off = 0
    for k, (cin, cout, _, _) in enumerate(co.LAYERS):
        n = cout * 9 * cin
        for name, a, b in (("w", g[off:off + n], g_ref[off:off + n]),
                           ("b", g[off + n:off + n + cout], g_ref[off + n:off + n + cout])):
            if name == "w" and cout == 8:
                a, b = a.reshape(8, -1)[:2], b.reshape(8, -1)[:2]
            if name == "b" and cout == 8:
                a, b = a[:2], b[:2]
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert rel < 1e-2, (k, name, rel)
        off += n + cout
    net.close()


def test_adam_steps_reduce_the_loss():
    """A learnable target (a pixel-wise linear map of the input) on a fixed batch."""
    from octo_b200.learned import FieldCorrectionNet
    net = FieldCorrectionNet(48, 48, max_batch=8, seed=2)
    xb, _, mask = _inputs(8, 48, 48, 9)
    x0 = xb[..., 0].float()
    t = torch_stack(0.3 * x0, -0.2 * x0)
    first = net.train_step(xb, t, mask, lr=3e-3)
    for _ in range(60):
        last = net.train_step(xb, t, mask, lr=3e-3)
    assert last < 0.3 * first, (first, last)
    net.close()


def torch_stack(a, b):
    import torch
    return torch.stack([a, b], dim=-1).contiguous()
