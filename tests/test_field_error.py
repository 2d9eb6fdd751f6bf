"""Exact Bassetti-Erskine field used to assess the solver's field error (the precision form's accuracy
criterion), checked against its round closed form and far-field limit, and the FP64 oracle's PIC field
checked against it on flat beams (128^2, CIC, second-order derivative: the production solver)."""
import math

import numpy as np
import pytest

from oracle import oracle as orc
from octo_b200.diagnostics import bassetti_erskine, quantile_lattice


def test_bassetti_erskine_round_limit_and_far_field():
    x = np.linspace(-4e-4, 4e-4, 41)
    X, Y = np.meshgrid(x, x)
    a = bassetti_erskine(X, Y, 1e-4 * (1 + 1e-6), 1e-4)
    b = bassetti_erskine(X, Y, 1e-4, 1e-4)
    assert np.max(np.hypot(a[0] - b[0], a[1] - b[1])) / np.max(np.hypot(*b)) < 1e-5
    # sx < sy is the axis-exchanged case
    c = bassetti_erskine(Y, X, 1e-4, 1e-4 * (1 + 1e-6))
    assert np.max(np.hypot(c[0] - b[1], c[1] - b[0])) / np.max(np.hypot(*b)) < 1e-5
    ex, ey = bassetti_erskine(np.array([1e-1, 0.0, -3e-2]), np.array([0.0, 2e-1, 4e-2]), 1e-4, 1e-5)
    np.testing.assert_allclose(ex, [10.0, 0.0, -12.0], rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(ey, [0.0, 5.0, 16.0], rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("aspect", [1, 25])
def test_oracle_pic_field_within_one_percent_of_bassetti_erskine(aspect):
    sy = 8.5e-6
    sx = sy * aspect
    xs, ys = quantile_lattice(200, sx, sy)
    g = np.linspace(-4, 4, 41)
    P, Q = np.meshgrid(g * sx, g * sy, indexing="ij")
    xp, yp = P.ravel(), Q.ravel()
    opt = orc.OracleOptions(grid=(128, 128))
    sg, fg = orc.interaction_grids(opt, xs.min(), xs.max(), ys.min(), ys.max(), xp.min(), xp.max(), yp.min(),
                                   yp.max())
    F = orc.solve_field(opt, xs, ys, sg, fg)
    bx, by = bassetti_erskine(xp, yp, sx, sy)
    err = np.empty(xp.size)
    for k in range(xp.size):
        ax, ay, _ = orc.interpolate(opt, fg, xp[k], yp[k], F, F, 1.0)
        err[k] = math.hypot(ax / xs.size - bx[k], ay / xs.size - by[k])
    rms = float(np.sqrt(np.mean(err ** 2)) / np.max(np.hypot(bx, by)))
    assert rms < 0.01, rms
