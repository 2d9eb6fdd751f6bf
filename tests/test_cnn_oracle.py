"""The CNN oracle (oracle/cnn_oracle.py) pinned on the CPU: in plain float64 (no bf16 rounding) its
analytic gradients equal central finite differences of its own loss, for parameters of every layer; the
bf16 rounding helper rounds to nearest even.  The GPU network's gradients are then checked against this
oracle in tests/test_gpu_cnn.py."""
import numpy as np

from oracle import cnn_oracle as co


def test_bf16_rounding_is_round_to_nearest_even():
    assert co.bf16(1.0 + 2 ** -8)[()] == 1.0             # tie -> even (mantissa ...0)
    assert co.bf16(1.0 + 3 * 2 ** -8)[()] == 1.0 + 2 ** -6  # tie -> even (rounds up)
    assert co.bf16(1.0 + 2 ** -7)[()] == 1.0 + 2 ** -7
    assert co.bf16(-3.0)[()] == -3.0


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(7)
    n = co.num_params()
    p = np.zeros(n)
    off = 0
    for cin, cout, _, _ in co.LAYERS:
        k = cout * 9 * cin
        p[off:off + k] = rng.standard_normal(k) * np.sqrt(2.0 / (9 * cin))
        off += k
        p[off:off + cout] = 0.05 * rng.standard_normal(cout)
        off += cout
    B, H, W = 1, 16, 16
    x = np.zeros((B, H, W, 8))
    x[..., 0] = rng.standard_normal((B, H, W))
    x[..., 1] = 0.3
    t = 0.1 * rng.standard_normal((B, H, W, 2))
    mask = (rng.random((B, H, W)) > 0.2).astype(float)
    net = co.Net(p, rounding=False)
    loss, g = net.loss_and_grads(x, t, mask)
    # a few coordinates of every layer's weights and its bias
    idx, off = [], 0
    for cin, cout, _, _ in co.LAYERS:
        k = cout * 9 * cin
        if cout == 8:  # head: only output channels 0, 1 carry loss
            idx += [off + 5, off + 9 * cin + 3]
        else:
            idx += list(off + rng.integers(0, k, 2))
        idx.append(off + k)  # first bias
        off += k + cout
    h = 1e-6
    for i in idx:
        pp = p.copy(); pp[i] += h
        lp, _ = co.Net(pp, rounding=False).loss_and_grads(x, t, mask)
        pm = p.copy(); pm[i] -= h
        lm, _ = co.Net(pm, rounding=False).loss_and_grads(x, t, mask)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(fd)) + 1e-9, (i, fd, g[i])
