"""The oracle's soft-Gaussian solver (gaussian.jl restated) against physics it must reproduce: one slice
each, long bunches made short (no hourglass), the luminosity of two Gaussian beams
N1 N2 / (2 pi sqrt(sx1^2 + sx2^2) sqrt(sy1^2 + sy2^2)) to sampling accuracy, whichever beam is sampled; and
the kick of a particle far outside the other beam approaches the point-charge kick 2 kbb / r."""
import numpy as np

from oracle import oracle as orc


def test_luminosity_of_two_gaussians():
    rng = np.random.default_rng(1)
    n1, n2 = 200_000, 150_000
    s1, s2 = (20e-6, 4e-6), (16e-6, 3e-6)

    def beam(n, s):
        b = np.zeros((6, n))
        b[0] = rng.normal(size=n) * s[0]
        b[2] = rng.normal(size=n) * s[1]
        b[4] = rng.normal(size=n) * 1e-9   # short bunches: no hourglass over the drift
        return b

    N1, N2 = 1e11, 7e10
    p1 = orc.beam_params(-1.0, orc.EMASS_EV, 10e9, N1)
    p2 = orc.beam_params(1.0, orc.PMASS_EV, 275e9, N2)
    opt = orc.OracleOptions(nslices1=1, nslices2=1, kbb1=0.0, kbb2=0.0)
    want = N1 * N2 / (2 * np.pi * np.hypot(s1[0], s2[0]) * np.hypot(s1[1], s2[1]))
    for g in (1, 2):
        b1, b2 = beam(n1, s1), beam(n2, s2)
        lum = orc.gaussian_collide(opt, b1, b2, p1, p2, gaussian_when_luminosity=g)
        assert abs(lum / want - 1) < 0.01, (g, lum, want)


def test_far_kick_is_point_charge():
    rng = np.random.default_rng(2)
    n2 = 100_000
    b2 = np.zeros((6, n2))
    b2[0] = rng.normal(size=n2) * 10e-6
    b2[2] = rng.normal(size=n2) * 10e-6
    b1 = np.zeros((6, 1))
    b1[0, 0] = 2e-3  # 200 sigma away
    kbb = 1e-4
    opt = orc.OracleOptions(nslices1=1, nslices2=1, kbb1=kbb, kbb2=0.0, longitudinal_kick=False)
    p = orc.beam_params(1.0, orc.PMASS_EV, 275e9, 1e11)
    orc.gaussian_collide(opt, b1, b2, p, p)
    # Kx -> 2 x / r^2 for a unit-normalised Gaussian; the slice weight is 1
    assert abs(b1[1, 0] / (kbb * 2 / 2e-3) - 1) < 1e-4
    # the y kick is the sampled centroid's offset (~1e-8 in y) seen from 2 mm
    assert abs(b1[3, 0]) < 1e-4 * abs(b1[1, 0])


def test_coupled_kick_is_rotated_bassetti_erskine():
    """include_sigma_xy: a Gaussian tilted in x-y kicks as the principal-axis Bassetti-Erskine field of its
    covariance's eigenframe, rotated back (strong_beam.jl:634-682 at S = 0)."""
    rng = np.random.default_rng(4)
    n2 = 200_000
    phi = 0.35
    u, v = rng.normal(size=n2) * 30e-6, rng.normal(size=n2) * 8e-6
    b2 = np.zeros((6, n2))
    b2[0] = np.cos(phi) * u - np.sin(phi) * v
    b2[2] = np.sin(phi) * u + np.cos(phi) * v
    pts = [(12e-6, -5e-6), (-40e-6, 30e-6), (3e-6, 2e-6)]
    b1 = np.zeros((6, len(pts)))
    for k, (x, y) in enumerate(pts):
        b1[0, k], b1[2, k] = x, y
    kbb = 1e-4
    opt = orc.OracleOptions(nslices1=1, nslices2=1, kbb1=kbb, kbb2=0.0, longitudinal_kick=False)
    p = orc.beam_params(1.0, orc.PMASS_EV, 275e9, 1e11)
    got = b1.copy()
    orc.gaussian_collide(opt, got, b2.copy(), p, p, include_sigma_xy=True)
    mx, my = b2[0].mean(), b2[2].mean()
    C = np.cov(np.stack([b2[0], b2[2]]), bias=True)
    w, V = np.linalg.eigh(C)
    s1, s2 = np.sqrt(w[1]), np.sqrt(w[0])
    e1 = V[:, 1]
    for k, (x, y) in enumerate(pts):
        dx, dy = x - mx, y - my
        xh, yh = e1[0] * dx + e1[1] * dy, -e1[1] * dx + e1[0] * dy
        kx, ky, _, _ = orc.be_response(0.0, s1, s2, xh, yh)
        fx = kbb * (e1[0] * kx - e1[1] * ky)
        fy = kbb * (e1[1] * kx + e1[0] * ky)
        assert abs(got[1, k] - fx) < 1e-9 * abs(fx) + 1e-15 and abs(got[3, k] - fy) < 1e-9 * abs(fy) + 1e-15, \
            (k, got[1, k], fx, got[3, k], fy)
    # with no tilt the coupled and uncoupled kicks agree
    b2r = np.zeros((6, n2))
    b2r[0], b2r[2] = u, v
    g1, g2 = b1.copy(), b1.copy()
    orc.gaussian_collide(opt, g1, b2r.copy(), p, p, include_sigma_xy=True)
    orc.gaussian_collide(opt, g2, b2r.copy(), p, p)
    np.testing.assert_allclose(g1[1], g2[1], rtol=2e-3)


def test_agrees_with_pic_on_gaussian_beams():
    """On Gaussian beams the soft-Gaussian solver and the PIC solver (two independent restatements) give the
    same luminosity to the PIC grid's accuracy and nearly the same kicks: the soft-Gaussian field is the
    Gaussian fit of what the PIC solve sees."""
    import sys
    import os
    sys.path.insert(0, os.path.dirname(__file__))
    from helpers import beams, oracle_params
    pe, pp = oracle_params()
    e, p = beams(200_000, 100_000)
    e1, p1, e2, p2 = e.copy(), p.copy(), e.copy(), p.copy()
    lum_pic = orc.Oracle(orc.OracleOptions(grid=(128, 128), nslices1=7, nslices2=7, nthreads=8)).collide(e1, p1, pe, pp)
    lum_soft = orc.gaussian_collide(orc.OracleOptions(nslices1=7, nslices2=7), e2, p2, pe, pp)
    assert abs(lum_soft / lum_pic - 1) < 5e-3
    for b0, b1, b2 in ((e, e1, e2), (p, p1, p2)):
        for k in (1, 3):
            d1, d2 = b1[k] - b0[k], b2[k] - b0[k]
            assert np.corrcoef(d1, d2)[0, 1] > 0.999
            assert np.sqrt(np.mean((d1 - d2) ** 2)) < 0.06 * np.sqrt(np.mean(d1 ** 2))


def test_rotation_term_series_matches_elliptic():
    """The coupled kick's rotation term L / D has two independent forms: the near-round series
    (strong_beam.jl:930-932) and (Kx y - Ky x) / D of the elliptic kick (:1107-1108).  Around the blend region
    eta in [inner, outer] (:779-797) they agree to the series' truncation error, and the principal-axis
    response takes the series below inner and the elliptic form above outer."""
    import math
    inner = math.sqrt(math.sqrt((8 / 3) * 64 * 2.220446049250313e-16)) / 2
    outer = 2 * inner
    v = 1e-8
    for eta in (0.5 * inner, inner, 1.5 * inner, outer, 1.5 * outer):
        s1, s2 = math.sqrt(v * (1 + eta)), math.sqrt(v * (1 - eta))
        for x, y in ((1.3e-4, 0.7e-4), (-2e-5, 3e-5), (0.5e-4, -1.2e-4)):
            series = orc.be_near_round_L(1.0, v, eta, x, y)[4]
            kx, ky = orc.be_elliptic(s1, s2, x, y)
            exact = (kx * y - ky * x) / (s1 * s1 - s2 * s2)
            principal = orc.be_principal_L(1.0, s1, s2, x, y)[4]
            assert abs(series - exact) < 2e-10 * abs(exact), (eta, series, exact)
            assert abs(principal - exact) < 2e-10 * abs(exact)
            if eta >= outer:  # the elliptic form itself (its denominator rounds as 2 v eta there)
                assert abs(principal - exact) <= 1e-14 * abs(exact)
