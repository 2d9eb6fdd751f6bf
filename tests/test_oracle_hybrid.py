"""The oracle's Gaussian-subtracted hybrid (GaussianPICPoissonSolver, gaussian_pic.jl) and its pieces:
the Faddeeva function (Weideman N = 32 + continued fraction) against scipy.special.wofz, the erf-integrated
CIC/TSC node profiles, the Bassetti-Erskine kick response in every regime (round, near-round series,
blend, elliptic, flat) against the exact field and its Hessians against finite differences, and the
hybrid collide itself: on a coarse grid its kicks are closer to a fine-grid plain-PIC solution than the
coarse plain-PIC kicks are (the point of the control variate)."""
import numpy as np
import pytest
from scipy.special import wofz

from helpers import beams, oracle_params, tilt
from oracle import oracle as orc
from octo_b200.diagnostics import bassetti_erskine


def test_faddeeva_matches_scipy():
    rng = np.random.default_rng(3)
    zs = np.concatenate([rng.uniform(-10, 10, 2000) + 1j * rng.uniform(-3, 12, 2000),
                         rng.uniform(-5000, 5000, 100) + 1j * rng.uniform(0, 3000, 100),
                         rng.uniform(0, 30, 200) + 1j * rng.uniform(0, 1e-9, 200)])
    err = max(abs(orc.faddeeva(complex(z)) - wofz(z)) / abs(wofz(z)) for z in zs)
    assert err < 1e-12, err


@pytest.mark.parametrize("method", ["CIC", "TSC"])
def test_gaussian_profile_conserves_charge_and_centroid(method):
    g = orc.gaussian_profile(method, -1.0, 0.02, 0.013, 0.1, 101)
    x = -1.0 + 0.02 * np.arange(101)
    assert abs(g.sum() - 1) < 1e-13 and abs((g * x).sum() - 0.013) < 1e-13


@pytest.mark.parametrize("sig", [(2.0, 1.0), (1.0, 3.0), (1.0, 1.0), (1.0 + 1e-5, 1.0), (1.0 + 3e-4, 1.0),
                                 (25.0, 1.0)])
def test_bassetti_erskine_response(sig):
    """Round, near-round series (eta < 2.2e-4), blend (2.2e-4 .. 4.4e-4), elliptic and flat regimes."""
    sx, sy = sig
    rng = np.random.default_rng(5)
    for _ in range(100):
        x, y = rng.uniform(-4 * sx, 4 * sx), rng.uniform(-4 * sy, 4 * sy)
        Kx, Ky, Hx, Hy = orc.be_response(1.0, sx, sy, x, y)
        bx, by = bassetti_erskine(np.array([x]), np.array([y]), sx, sy)
        # the reference's normalised kick is twice the unit-charge field: Kx = 2x(1 - e^-r^2/2s^2)/r^2
        assert abs(Kx - 2 * bx[0]) + abs(Ky - 2 * by[0]) <= 1e-11 * (abs(2 * bx[0]) + abs(2 * by[0])) + 1e-14
        hx, hy = 1e-5 * sx, 1e-5 * sy
        dKx = (orc.be_response(1.0, sx, sy, x + hx, y)[0] - orc.be_response(1.0, sx, sy, x - hx, y)[0]) / (2 * hx)
        dKy = (orc.be_response(1.0, sx, sy, x, y + hy)[1] - orc.be_response(1.0, sx, sy, x, y - hy)[1]) / (2 * hy)
        assert abs(Hx + dKx) <= 1e-6 * (abs(dKx) + 1e-6) and abs(Hy + dKy) <= 1e-6 * (abs(dKy) + 1e-6)


def _collide(opts, e, p):
    pe, pp = oracle_params()
    e, p = e.copy(), p.copy()
    lum = orc.Oracle(opts).collide(e, p, pe, pp)
    return e, p, lum


def test_hybrid_coarse_grid_beats_plain_pic_on_the_same_grid():
    e, p = beams(20000, 20000, (95e-6, 8.5e-6, 7e-3), (95e-6, 8.5e-6, 6e-2))
    kw = dict(nslices1=3, nslices2=3, nthreads=8)
    fine, _, _ = _collide(orc.OracleOptions(grid=(256, 256), **kw), e, p)
    plain, _, _ = _collide(orc.OracleOptions(grid=(32, 32), **kw), e, p)
    hyb, _, lum = _collide(orc.OracleOptions(grid=(32, 32), gaussian=True, **kw), e, p)
    for row in (1, 3):
        kick_ref = fine[row] - e[row]
        err_plain = np.sqrt(np.mean((plain[row] - fine[row]) ** 2))
        err_hyb = np.sqrt(np.mean((hyb[row] - fine[row]) ** 2))
        assert err_hyb < 0.7 * err_plain, (row, err_hyb, err_plain, np.sqrt(np.mean(kick_ref ** 2)))
    assert np.isfinite(lum) and np.all(np.isfinite(hyb))


def test_hybrid_falls_back_to_plain_pic_for_degenerate_slices():
    """A source slice with zero transverse spread has no resolved reference Gaussian: the hybrid runs the
    plain PIC interaction (gaussian_pic.jl:542-553), so both collides agree exactly."""
    e, p = beams(2000, 2000)
    e[0] = 1e-5
    e[1] = 0.0
    kw = dict(grid=(32, 32), nslices1=1, nslices2=1, min_transverse_extent=(1e-4, 1e-4))
    pe1, pp1, l1 = _collide(orc.OracleOptions(gaussian=True, **kw), e, p)
    pe2, pp2, l2 = _collide(orc.OracleOptions(**kw), e, p)
    np.testing.assert_array_equal(pp1, pp2)


def test_hybrid_rejects_options_it_does_not_read():
    e, p = beams(500, 500)
    for kw in (dict(slice_interpolation="quadratic"), dict(interaction_grid="node")):
        with pytest.raises(orc.OracleErrorPy):
            _collide(orc.OracleOptions(grid=(32, 32), gaussian=True, **kw), e, p)


def test_coupled_subtraction_beats_uncoupled_on_tilted_beams():
    """coupling_tol finite: the tilted reference Gaussian (conditional expansion to second order in
    lambda = sigma_xy / sigma_x^2, gaussian_pic.jl:240-372) and the rotated Bassetti-Erskine add-back
    (_cp_covariance_kick).  On a coarse grid and beams tilted by 0.3 rad its kicks are closer to a fine-grid
    plain-PIC solution than the uncoupled subtraction's.  Beams tilted by 0.05 rad (|r_xy| ~ 0.5 for the 11:1
    flat beams; lambda sigma_x / sigma_c ~ 0.5, inside the expansion's range): the uncoupled subtraction leaves
    the tilt to the coarse grid and its vertical kicks degrade; the coupled one removes most of that."""
    e, p = beams(20000, 20000, (95e-6, 8.5e-6, 7e-3), (95e-6, 8.5e-6, 6e-2))
    e, p = tilt(e, 0.05), tilt(p, 0.05)
    kw = dict(nslices1=3, nslices2=3, nthreads=8)
    fine, _, _ = _collide(orc.OracleOptions(grid=(256, 256), **kw), e, p)
    unc, _, _ = _collide(orc.OracleOptions(grid=(32, 32), gaussian=True, **kw), e, p)
    cpl, _, lum = _collide(orc.OracleOptions(grid=(32, 32), gaussian=True, coupling_tol=0.01, **kw), e, p)
    err = {row: (np.sqrt(np.mean((unc[row] - fine[row]) ** 2)), np.sqrt(np.mean((cpl[row] - fine[row]) ** 2)))
           for row in (1, 3)}
    assert err[3][1] < 0.75 * err[3][0], err  # py: the coupled subtraction removes the tilt's error
    assert err[1][1] <= 1.0 * err[1][0], err  # px: no worse
    assert np.isfinite(lum) and np.all(np.isfinite(cpl))


def test_coupled_tolerance_above_the_correlation_keeps_the_uncoupled_subtraction():
    """|r_xy| below coupling_tol at both boundaries: the uncoupled subtraction runs, bit for bit."""
    e, p = beams(4000, 4000, (95e-6, 8.5e-6, 7e-3), (95e-6, 8.5e-6, 6e-2))
    kw = dict(grid=(32, 32), nslices1=2, nslices2=2, gaussian=True)
    a = _collide(orc.OracleOptions(**kw), e, p)
    b = _collide(orc.OracleOptions(coupling_tol=0.99, **kw), e, p)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2] == b[2]


def test_coupled_rank_deficient_source_falls_back_to_plain_pic():
    """y = 0.3 x, py = 0.3 px: |r_xy| = 1, the coupled covariance is rank-deficient, so the interaction runs
    plain PIC (gaussian_pic.jl:525-536) and the kicks it gives equal the plain PIC collide's exactly."""
    e, p = beams(2000, 2000)
    e[2] = 0.3 * e[0]
    e[3] = 0.3 * e[1]
    kw = dict(grid=(32, 32), nslices1=1, nslices2=1)
    pe1, pp1, l1 = _collide(orc.OracleOptions(gaussian=True, coupling_tol=0.5, **kw), e, p)
    pe2, pp2, l2 = _collide(orc.OracleOptions(**kw), e, p)
    np.testing.assert_array_equal(pp1, pp2)
