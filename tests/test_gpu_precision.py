"""The precision form (float32 beams: FP32 particle arithmetic, field planes and FFTs; FP64 Green
function, slice statistics, grid geometry and luminosity sums; int64 fixed-point charge grids)
against the FP64 oracle run on the same float32-rounded inputs, and its field accuracy against exact
Bassetti-Erskine next to the plain form's.

Tolerances, per particle and coordinate: |gpu - oracle| <= (S + 1) * 2^-24 |oracle| + RTOL * scale.  The
first term is FP32 storage rounding: a particle is kicked once per slice pair, S times per collide (S the
other beam's slice count), and each kick rounds the stored coordinate once (half an ulp); it matters for
pz, whose kick is only ~25 float32 ulps of pz for the protons.  scale is the largest kick on a momentum
coordinate (RTOL 2e-4: FP32 FFT and interpolation error) or the
coordinate's range on a position (RTOL 2e-5: FP32 kick errors carried through drifts of up to half the
slice-centre separation); luminosity to 1e-5 relative; RMS field error vs Bassetti-Erskine below 1 %
for aspect ratios 1-25 and within 1e-4 of the plain form's."""
import numpy as np
import pytest
import torch

from helpers import beams, oracle_options, oracle_params, E_PARAMS, P_PARAMS

pytestmark = pytest.mark.gpu

POS_RTOL = 2e-5
KICK_RTOL = 2e-4
LUM_RTOL = 1e-5


def _params(ob):
    pe = ob.BeamParams(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"], E_PARAMS["r0"], E_PARAMS["npart"])
    pp = ob.BeamParams(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"], P_PARAMS["r0"], P_PARAMS["npart"])
    return pe, pp


def run_precision(solver, n1, n2, turns=2, e_sigma=None, p_sigma=None, seed=123456789, transform=None):
    kicks = {"e": solver.resolved_slicing2.nslices, "p": solver.resolved_slicing1.nslices}
    import octo_b200 as ob
    from oracle import oracle as orc
    e, p = beams(n1, n2, e_sigma, p_sigma, seed=seed)
    if transform is not None:
        e, p = transform(e), transform(p)
    e = e.astype(np.float32).astype(np.float64)
    p = p.astype(np.float32).astype(np.float64)
    pe, pp = _params(ob)
    be = ob.Beam.from_numpy(e, pe, dtype=torch.float32)
    bp = ob.Beam.from_numpy(p, pp, dtype=torch.float32)
    rt = ob.StrongStrongRuntime()
    ctx = rt.context("ip", solver, 0, torch.float32)
    oracle = orc.Oracle(oracle_options(solver))
    ope, opp = oracle_params()
    out = []
    for t in range(turns):
        e_prev, p_prev = e.copy(), p.copy()
        lum_g = ctx.collide(be, bp, turn=t + 1)
        lum_o = oracle.collide(e, p, ope, opp)
        r = dict(lum_g=lum_g, lum_o=lum_o)
        for name, g, o, prev in (("e", be, e, e_prev), ("p", bp, p, p_prev)):
            gv = g.coords.to(torch.float64).cpu().numpy()
            for row in range(6):
                if row in (0, 2, 4):
                    scale = POS_RTOL * float(np.ptp(o[row]))
                else:
                    scale = KICK_RTOL * float(np.max(np.abs(o[row] - prev[row])))
                bound = (kicks[name] + 1) * 2.0 ** -24 * np.abs(o[row]) + scale
                r[f"{name}{row}"] = float(np.max(np.abs(gv[row] - o[row]) / bound))
        out.append(r)
        # continue both from the same (float32) state so each turn's error is that turn's own
        e = be.coords.to(torch.float64).cpu().numpy()
        p = bp.coords.to(torch.float64).cpu().numpy()
    rt.close()
    return out


def check(out):
    import json
    bad = []
    for r in out:
        if abs(r["lum_g"] / r["lum_o"] - 1) > LUM_RTOL:
            bad.append("luminosity")
        for name in ("e", "p"):
            bad += [f"{name}{row}" for row in range(6) if r[f"{name}{row}"] > 1.0]
    assert not bad, (bad, json.dumps(out))


def test_precision_form_node_cic():
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), interaction_grid="node",
                            slicing=ob.LongitudinalSlicing(nslices=7, method="normal_quantile"))
    check(run_precision(s, 20000, 10000, e_sigma=(95e-6, 8.5e-6, 0.7e-2), p_sigma=(95e-6, 8.5e-6, 6e-2)))


def test_precision_form_node_tsc_fourth():
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), interaction_grid="node", deposit_method="TSC", field_derivative="fourth",
                            slicing=ob.LongitudinalSlicing(nslices=7, method="normal_quantile"))
    check(run_precision(s, 20000, 10000, e_sigma=(95e-6, 8.5e-6, 0.7e-2), p_sigma=(95e-6, 8.5e-6, 6e-2)))


def test_precision_form_slice_pair_tsc_fourth_quadratic():
    """The precision configuration's options (TSC, 4th-order, quadratic) on the :slice_pair grid, the
    grid the reference allows :quadratic with (pic_cpu.jl:568-574)."""
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), deposit_method="TSC", field_derivative="fourth",
                            slice_interpolation="quadratic", green_cache="none",
                            slicing=ob.LongitudinalSlicing(nslices=5, method="normal_quantile"))
    check(run_precision(s, 6000, 4000))


def test_precision_form_source_slice():
    """interaction_grid = :source_slice in the precision form: the union boxes from float32 coordinates."""
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), interaction_grid="source_slice",
                            slicing=ob.LongitudinalSlicing(nslices=5, method="normal_quantile"))
    check(run_precision(s, 6000, 4000, e_sigma=(95e-6, 8.5e-6, 0.7e-2), p_sigma=(95e-6, 8.5e-6, 6e-2)))


@pytest.mark.parametrize("aspect", [1, 5, 11, 25])
def test_field_error_vs_bassetti_erskine_both_forms(aspect):
    import octo_b200 as ob
    from octo_b200.diagnostics import field_error
    sy = 8.5e-6
    for solver in (ob.PICPoissonSolver(grid=(128, 128), interaction_grid="node"),
                   ob.PICPoissonSolver(grid=(128, 128), interaction_grid="node", deposit_method="TSC",
                                       field_derivative="fourth")):
        e64 = field_error(solver, aspect * sy, sy, torch.float64)
        e32 = field_error(solver, aspect * sy, sy, torch.float32)
        assert e64["rms"] < 0.01 and e32["rms"] < 0.01, (e64, e32)
        assert abs(e32["rms"] - e64["rms"]) < 1e-4, (e64, e32)


def test_linear6d_float32_matches_float64():
    import octo_b200 as ob
    pe, _ = _params(ob)
    e, _ = beams(5000, 10)
    b64 = ob.Beam.from_numpy(e, pe)
    b32 = ob.Beam.from_numpy(e, pe, dtype=torch.float32)
    m = ob.Linear6D((0.55, 0.056, 12.7), (0, 0, 0), (0.08, 0.06, -0.069))
    m.track(b64, turns=3)
    m.track(b32, turns=3)
    torch.cuda.synchronize()
    a, b = b64.coords.cpu().numpy(), b32.coords.to(torch.float64).cpu().numpy()
    for row in range(6):
        assert np.max(np.abs(a[row] - b[row])) <= 1e-6 * np.ptp(a[row])


def test_precision_form_rejects_float64_beams():
    import octo_b200 as ob
    pe, pp = _params(ob)
    e, p = beams(1000, 1000)
    s = ob.PICPoissonSolver(grid=(32, 32), slicing=ob.LongitudinalSlicing(nslices=3, method="normal_quantile"))
    ctx = ob.Context(s, 0, torch.float32)
    with pytest.raises(ob.CollisionError) as err:
        ctx.collide(ob.Beam.from_numpy(e, pe), ob.Beam.from_numpy(p, pp))
    assert "float32" in str(err.value)
    ctx.close()


@pytest.mark.parametrize("opts", [
    dict(),
    dict(deposit_method="TSC", field_derivative="fourth"),
    dict(neutralize=False, margin_sigma=0.0, green_cache="none", grid=(48, 48)),
])
def test_precision_form_gaussian_hybrid(opts):
    """GaussianPICPoissonSolver in the precision form: FP32 particles, residual planes and FFTs (the R plane an
    exact int64 difference L - R with the difference of the two reference Gaussians subtracted), FP64 moments,
    reference Gaussians and Bassetti-Erskine add-back; against the oracle's FP64 hybrid under the same bounds."""
    import octo_b200 as ob
    kw = dict(grid=(64, 64), slicing=ob.LongitudinalSlicing(nslices=4, method="normal_quantile"))
    kw.update(opts)
    s = ob.GaussianPICPoissonSolver(**kw)
    check(run_precision(s, 6000, 4000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2)))


def test_precision_form_gaussian_hybrid_coupled():
    """The coupled (rotated) subtraction in the precision form on beams tilted by 0.05 rad."""
    import octo_b200 as ob
    from helpers import tilt
    s = ob.GaussianPICPoissonSolver(grid=(64, 64), slicing=ob.LongitudinalSlicing(nslices=4, method="normal_quantile"),
                                    coupling_tol=0.01)
    check(run_precision(s, 6000, 4000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2),
                        transform=lambda b: tilt(b, 0.05)))
