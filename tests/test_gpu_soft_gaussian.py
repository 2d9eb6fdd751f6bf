"""The soft-Gaussian solver (GaussianPoissonSolver, src/tasks/strongstrong/gaussian.jl) on the GPU against
the oracle's restatement: coordinates within the reference contract's atol = rtol = 1e-10
(Contracts.jl:1173-1232), luminosity within 1e-12 relative.  The two sides differ only in the order of the
moment and luminosity sums."""
import numpy as np
import pytest

from oracle import oracle as orc
from helpers import beams, oracle_params, within, E_PARAMS, P_PARAMS

pytestmark = pytest.mark.gpu


def run_both(solver, e, p, turns=1, dtype=None):
    import octo_b200 as ob
    import torch
    dtype = dtype or torch.float64
    pe, pp = oracle_params()
    s1, s2 = solver.resolved_slicing1, solver.resolved_slicing2
    opt = orc.OracleOptions(nslices1=s1.nslices, nslices2=s2.nslices,
                            method1="specified" if s1.method == "specified" else "normal_quantile",
                            method2="specified" if s2.method == "specified" else "normal_quantile",
                            center_position1=s1.center_position, center_position2=s2.center_position,
                            positions1=list(s1.positions), positions2=list(s2.positions),
                            kbb1=solver.kbb1, kbb2=solver.kbb2, luminosity_scale=solver.luminosity_scale,
                            longitudinal_kick=solver.longitudinal_kick)
    be = ob.Beam.from_numpy(e, ob.BeamParams(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"],
                                             E_PARAMS["r0"], E_PARAMS["npart"]), dtype=dtype)
    bp = ob.Beam.from_numpy(p, ob.BeamParams(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"],
                                             P_PARAMS["r0"], P_PARAMS["npart"]), dtype=dtype)
    rt = ob.StrongStrongRuntime()
    oe, op = e.copy(), p.copy()
    lums = []
    for t in range(turns):
        lum = ob.collide(solver, be, bp, ob.CUDABackend, ob.TrackingContext(turn=t), runtime=rt)
        lum_ref = orc.gaussian_collide(opt, oe, op, pe, pp, solver.min_sigma, solver.gaussian_when_luminosity,
                                       solver.ignore_centroid1, solver.ignore_centroid2, solver.virtual_drift,
                                       solver.include_sigma_xy)
        lums.append((lum, lum_ref))
    rt.close()
    return (be.coords.to(torch.float64).cpu().numpy(), bp.coords.to(torch.float64).cpu().numpy(), oe, op, lums)


@pytest.mark.parametrize("kw", [
    dict(),
    dict(gaussian_when_luminosity=1),
    dict(longitudinal_kick=False),
    dict(ignore_centroid1=True, min_sigma=2e-6),
    dict(kbb1=-3e-4, kbb2=2e-4, luminosity_scale=1.5e20),
    dict(virtual_drift="chromatic"),
    dict(virtual_drift="exact"),
    dict(virtual_drift="exact", longitudinal_kick=False),
    dict(include_sigma_xy=True),
    dict(include_sigma_xy=True, virtual_drift="chromatic", min_sigma=2e-6),
])
def test_matches_oracle(kw):
    import octo_b200 as ob
    e, p = beams(40_000, 24_000)
    solver = ob.GaussianPoissonSolver(slicing=ob.LongitudinalSlicing(nslices=7, method="normal_quantile"), **kw)
    ge, gp, oe, op, lums = run_both(solver, e, p, turns=2)
    assert within(ge, oe, 1e-10, 1e-10) <= 1.0 and within(gp, op, 1e-10, 1e-10) <= 1.0
    for lum, ref in lums:
        assert abs(lum / ref - 1.0) < 1e-12, (lum, ref)


def test_uneven_slicings_and_empty_slices():
    import octo_b200 as ob
    e, p = beams(30_000, 20_000)
    # far tails give slices with no particles; the reference still runs those pairs
    solver = ob.GaussianPoissonSolver(
        slicing1=ob.LongitudinalSlicing(nslices=5, method="specified", positions=(-9.0, -8.5, 0.0, 8.5)),
        slicing2=ob.LongitudinalSlicing(nslices=9, method="normal_quantile"), min_sigma=1e-6)
    ge, gp, oe, op, lums = run_both(solver, e, p)
    assert within(ge, oe, 1e-10, 1e-10) <= 1.0 and within(gp, op, 1e-10, 1e-10) <= 1.0
    assert abs(lums[0][0] / lums[0][1] - 1.0) < 1e-12


def test_production_size_matches_oracle():
    import octo_b200 as ob
    e, p = beams(400_000, 160_000)
    solver = ob.GaussianPoissonSolver(slicing=ob.LongitudinalSlicing(nslices=15, method="normal_quantile"))
    ge, gp, oe, op, lums = run_both(solver, e, p)
    assert within(ge, oe, 1e-10, 1e-10) <= 1.0 and within(gp, op, 1e-10, 1e-10) <= 1.0
    assert abs(lums[0][0] / lums[0][1] - 1.0) < 1e-12


def test_nonfinite_and_unsupported():
    import octo_b200 as ob
    e, p = beams(5000, 4000)
    e[0, 77] = np.nan
    solver = ob.GaussianPoissonSolver(slicing=ob.LongitudinalSlicing(nslices=3, method="normal_quantile"))
    be = ob.Beam.from_numpy(e, ob.BeamParams(-1.0, ob.EMASS_EV, 10e9, ob.RE, 1.7e11))
    bp = ob.Beam.from_numpy(p, ob.BeamParams(1.0, ob.PMASS_EV, 275e9, ob.RE * ob.ME0 / ob.PMASS_EV, 6.9e10))
    with pytest.raises(ob.CollisionError) as err:
        ob.collide(solver, be, bp)
    assert err.value.code == 1 and "source" in str(err.value)
    with pytest.raises(ob.ArgumentError):
        ob.GaussianPoissonSolver(virtual_drift="paraxial")


@pytest.mark.parametrize("kw", [dict(), dict(include_sigma_xy=True, virtual_drift="chromatic")])
def test_float32_beams_match_oracle(kw):
    """float32 beams: coordinates stored in float and computed in FP64 (the reference promotes a Float32 beam
    against the solver's Float64 moments and scales), against the FP64 oracle on the same float32-rounded
    inputs.  Each kick rounds the stored coordinates once, S times per collide (S the other beam's slices), so a
    coordinate may differ by (S + 1) half-ulps of float32 of itself, plus a few ulps at its row's scale where it
    is a small difference of larger drift terms; luminosity within 1e-6."""
    import octo_b200 as ob
    import torch
    e, p = beams(40_000, 24_000)
    e = e.astype(np.float32).astype(np.float64)
    p = p.astype(np.float32).astype(np.float64)
    solver = ob.GaussianPoissonSolver(slicing=ob.LongitudinalSlicing(nslices=7, method="normal_quantile"), **kw)
    ge, gp, oe, op, lums = run_both(solver, e, p, turns=1, dtype=torch.float32)
    bound = 8 * 2.0 ** -24
    for g, o in ((ge, oe), (gp, op)):
        for row in range(6):
            scale = 4 * 2.0 ** -24 * np.max(np.abs(o[row]))
            assert np.max(np.abs(g[row] - o[row]) / (bound * np.abs(o[row]) + scale)) <= 1.0, row
    assert abs(lums[0][0] / lums[0][1] - 1.0) < 1e-6, lums
