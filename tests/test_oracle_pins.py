"""Pins of the FP64 CPU oracle against the reference's own known answers.

Every parity claim of the CUDA path rests on the oracle, so the oracle is checked first against
the reference's golden vectors, known-answer tests and analytic identities (see oracle/oracle.h)."""
import math

import numpy as np
import pytest
from scipy import special

from helpers import E_PARAMS, P_PARAMS, beams
from oracle import oracle as orc


def test_philox_random123_known_answers():
    """counter_rng.jl:250-258 (Random123 kat_vectors for philox4x32-10)."""
    assert orc.philox4x32_block((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert orc.philox4x32_block((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF)) == \
        (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    assert orc.philox4x32_block((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == \
        (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


def test_counter_normals_are_standard():
    z = np.array([orc.lib().oo_normal(123456789, 0, 1, i, 1) for i in range(1, 20001)])
    assert abs(z.mean()) < 0.03 and abs(z.std() - 1) < 0.03


def test_beam_is_standardised_then_scaled():
    e, _ = beams(20000, 10)
    sig = (106e-6, 9.5e-6, 0.7e-2)
    for k, s in zip((0, 2, 4), sig):
        assert abs(e[k].mean()) < 1e-18 + 1e-12 * s
        assert abs(e[k].std() / s - 1) < 1e-12


def test_integrated_green_kernel_is_zero_on_the_axes():
    """runtests.jl:2576-2591"""
    for x, y in ((0.0, 1.0), (1.0, 0.0), (0.0, 2.5), (-3.0, 0.0)):
        assert orc.lib().oo_kernel_integral(x, y) == 0.0
    L = orc.lib()
    assert math.isclose(L.oo_atan_ratio(1.0, 0.0), math.pi / 2)
    assert math.isclose(L.oo_atan_ratio(-1.0, 0.0), -math.pi / 2)
    assert L.oo_atan_ratio(0.0, 0.0) == 0.0
    assert math.isclose(L.oo_atan_ratio(1.0, 1.0), math.pi / 4)


def _weights(fn, u, n, k):
    import ctypes as C
    base = C.c_int32()
    w = (C.c_double * k)()
    fn(u, n, C.byref(base), w)
    return base.value, list(w)


def test_cic_and_tsc_weights():
    L = orc.lib()
    b, w = _weights(L.oo_cic_weights, 4.0, 5, 2)       # boundary node keeps the charge (U5-7)
    assert (b, w) == (4, [0.0, 1.0])
    b, w = _weights(L.oo_cic_weights, -1e-9, 5, 2)     # outside: zero weights
    assert w == [0.0, 0.0]
    b, w = _weights(L.oo_cic_weights, float("nan"), 5, 2)
    assert w == [0.0, 0.0]
    for u in np.linspace(0.0, 9.0, 37):
        b, w = _weights(L.oo_tsc_weights, float(u), 10, 3)
        assert abs(sum(w) - 1.0) < 1e-15 and 1 <= b <= 8
        b, w = _weights(L.oo_cic_weights, float(u), 10, 2)
        assert abs(sum(w) - 1.0) < 1e-15


def test_quadratic_interpolation_identities():
    """runtests.jl:9741-9776: endpoint collapse, mid-slice reduction, partition of unity, gauge invariance."""
    opt = orc.OracleOptions(grid=(8, 8))
    rng = np.random.default_rng(7)
    planes = [tuple(rng.normal(size=(8, 8)) * s for _ in range(3)) for s in (1.0, 2.0, 3.0)]
    L, M, R = planes
    grid = (-0.5, -0.5, 1.0, 1.0)
    quad = lambda t, L=L, M=M, R=R: orc.interpolate(opt, grid, 0.13, -0.07, L, R, t, M=M)
    lin = lambda zl: orc.interpolate(opt, grid, 0.13, -0.07, L, R, zl)
    assert np.allclose(quad(0.0)[:2], lin(1.0)[:2], rtol=1e-12)
    assert np.allclose(quad(1.0)[:2], lin(0.0)[:2], rtol=1e-12)
    assert math.isclose(quad(0.5)[2], lin(0.5)[2], rel_tol=1e-12)
    flat = tuple(np.ones((8, 8)) for _ in range(3))
    for t in (0.0, 0.25, 0.5, 0.75, 1.0):
        kx, ky, _ = orc.interpolate(opt, grid, 0.13, -0.07, flat, flat, t, M=flat)
        assert math.isclose(kx, 1.0, rel_tol=1e-12) and math.isclose(ky, 1.0, rel_tol=1e-12)
        shifted = [(p[0] + 17.0, p[1], p[2]) for p in (L, M, R)]
        kz0 = quad(t)[2]
        kz1 = orc.interpolate(opt, grid, 0.13, -0.07, shifted[0], shifted[2], t, M=shifted[1])[2]
        assert abs(kz0 - kz1) < 1e-12


def _median_field_error(fd):
    """runtests.jl:9660-9693: deterministic Gaussian quantile source, 64^2, field vs exact round BE."""
    sig, n = 2.0e-3, 200
    u = (np.arange(1, n + 1) - 0.5) / n
    q = np.sqrt(2.0) * special.erfinv(2 * u - 1)
    sx = np.repeat(sig * q, n)
    sy = np.tile(sig * q, n)
    xg = np.linspace(-2 * sig, 2 * sig, 41)
    opt = orc.OracleOptions(grid=(64, 64), field_derivative=fd)
    sg, fg = orc.interaction_grids(opt, sx.min(), sx.max(), sy.min(), sy.max(), xg.min(), xg.max(), xg.min(),
                                   xg.max())
    phi, ex, ey = orc.solve_field(opt, sx, sy, sg, fg)
    P = (phi, ex, ey)
    errs, nrm = [], []
    for y in xg:
        for x in xg:
            r2 = x * x + y * y
            f = 2 * (1 - math.exp(-r2 / (2 * sig * sig))) / r2 if r2 > 0 else 0.0
            ekx, eky = f * x, f * y
            ax, ay, _ = orc.interpolate(opt, fg, x, y, P, P, 1.0)
            errs.append(math.hypot(2 * ax / sx.size - ekx, 2 * ay / sx.size - eky))
            nrm.append(math.hypot(ekx, eky))
    return float(np.median(errs)) / max(nrm)


def test_fourth_order_field_beats_second_order_against_bassetti_erskine():
    """runtests.jl:9628-9693: the 4th-order derivative's median error is < 0.75x the 2nd-order one."""
    e2, e4 = _median_field_error("second"), _median_field_error("fourth")
    assert e4 < e2 and e4 < 0.75 * e2
    assert e2 < 5e-3  # the PIC field is within a fraction of a percent of exact BE


def test_luminosity_overlap_covers_full_extent():
    """runtests.jl:10047-10075: CIC never reaches the top row/column, TSC does."""
    n = 200
    x1 = np.array([1.0e-4 * (i - 1) / (n - 1) for i in range(1, n + 1)])
    y1 = np.array([1.0e-4 * ((i * 7) % n) / n for i in range(1, n + 1)])
    x2, y2 = x1.copy(), y1[::-1].copy()
    out = {}
    for m in ("CIC", "TSC"):
        opt = orc.OracleOptions(grid=(16, 16), deposit_method=m)
        lum, q1, q2 = orc.luminosity(opt, x1, y1, x2, y2, 1.0)
        excluded = q1[16, :].sum() + q1[:, 16].sum() - q1[16, 16]
        out[m] = (lum, excluded)
    assert out["CIC"][1] == 0.0
    assert out["TSC"][1] > 0.0


def test_erfinv_matches_scipy():
    for x in np.concatenate([np.linspace(-0.999, 0.999, 201), [1e-300, -1e-10, 0.5, 0.9999999]]):
        a, b = orc.erfinv(float(x)), special.erfinv(float(x))
        assert abs(a - b) <= 2 * np.spacing(abs(b)) + 1e-300, (x, a, b)


def test_wavefront_batches():
    """collision_pair_batches: 2S-1 fronts with widths 1..S..1 for equal slice counts (slicing.jl:601-647)."""
    for S in (5, 15, 31):
        c = np.sort(np.random.default_rng(S).normal(size=S))
        batches, order = orc.pair_batches(c, c)
        assert len(batches) == 2 * S - 1
        widths = [len(b) for b in batches]
        assert max(widths) == S and widths[0] == 1 and widths[-1] == 1
        for b in batches:  # conflict-free
            assert len({i for i, _ in b}) == len(b) and len({j for _, j in b}) == len(b)


def test_slicing_quantiles_and_centroids():
    e, _ = beams(50000, 10)
    b, c, w, cnt, order = orc.slices(e[4], 15)
    z = e[4]
    mu, sd = z.mean(), z.std()
    assert b[0] == z.min() and b[-1] == z.max()
    for s in range(1, 15):
        assert abs(b[s] - (mu + sd * math.sqrt(2) * special.erfinv(2 * s / 15 - 1))) < 1e-12 * sd
    start = 0
    for s in range(15):
        idx = order[start:start + cnt[s]]
        assert np.all(np.diff(idx) > 0)
        assert abs(c[s] - z[idx].mean()) < 1e-15 * abs(z).max() * 10
        assert np.all((z[idx] >= b[s]) & (z[idx] <= b[s + 1]))
        start += cnt[s]
    assert abs(w.sum() - 1) < 1e-15


def test_linear6d_matrix_is_symplectic():
    m = orc.linear6d_matrix((0.55, 0.056, 12.7), (0.0, 0.0, 0.0), (0.08, 0.06, -0.069)).reshape(6, 6)
    J = np.kron(np.eye(3), np.array([[0, 1], [-1, 0]]))
    assert np.allclose(m.T @ J @ m, J, atol=1e-13)


def test_zero_width_slice_remains_finite():
    """runtests.jl:7528-7544: z = 0 for every particle, one slice, kbb overrides."""
    n = 16
    x = np.linspace(-1.0e-3, 1.0e-3, n)
    y = x[::-1].copy()
    b1 = np.vstack([x, np.zeros(n), y, np.zeros(n), np.zeros(n), np.zeros(n)])
    b2 = np.vstack([y, np.zeros(n), x, np.zeros(n), np.zeros(n), np.zeros(n)])
    o = orc.Oracle(orc.OracleOptions(grid=(16, 16), green_cache="none", kbb1=1e-4, kbb2=1e-4, luminosity_scale=1.0))
    p = orc.beam_params(1.0, 1.0, 1.0, 1.0)
    lum = o.collide(b1, b2, p, p)
    assert math.isfinite(lum) and np.all(np.isfinite(b1)) and np.all(np.isfinite(b2))


def test_nonfinite_input_fails_fast_with_location():
    e, p = beams(500, 500)
    e[0, 37] = np.nan
    o = orc.Oracle(orc.OracleOptions(grid=(32, 32), nslices1=3, nslices2=3))
    pe = orc.beam_params(-1.0, orc.EMASS_EV, 10e9, E_PARAMS["npart"], orc.RE)
    pp = orc.beam_params(1.0, orc.PMASS_EV, 275e9, P_PARAMS["npart"], P_PARAMS["r0"])
    with pytest.raises(orc.OracleErrorPy) as err:
        o.collide(e, p, pe, pp)
    assert err.value.code == orc.ERR_NONFINITE and "source" in str(err.value)


@pytest.mark.slow
def test_production_golden_luminosity():
    """Golden CPU luminosity of one production collide (docs/history/cpu_benchmark_history.tsv:2,6,10):
    2.56M/1.024M, seed 123456789, 15 :normal_quantile centroid slices, 128^2, CIC, slice-pair cache."""
    e = orc.beam_gaussian(2_560_000, rng_id=1, beta=(0.55, 0.056, 0.7e-2 / 5.5e-4), sigma=(106e-6, 9.5e-6, 0.7e-2))
    p = orc.beam_gaussian(1_024_000, rng_id=2, beta=(0.8, 0.072, 6e-2 / 6.6e-4), sigma=(95e-6, 8.5e-6, 6e-2))
    pe = orc.beam_params(-1.0, orc.EMASS_EV, 10e9, 1.7203e11)
    pp = orc.beam_params(1.0, orc.PMASS_EV, 275e9, 0.6881e11)
    o = orc.Oracle(orc.OracleOptions(grid=(128, 128), nslices1=15, nslices2=15, nthreads=8))
    lum = o.collide(e, p, pe, pp)
    assert abs(lum / 1.0254361754701657e+30 - 1) < 1e-12
    assert o.cache_stats() == (0, 450, 0)
