"""The reference's other slicing methods on the GPU against the oracle: :equal_area (LongitudinalSlicing()'s
default), :equal_count and :equal_width (and the :equal_spaced alias), each inside full collides at the
backend-consistency tolerance (coordinates atol = rtol = 1e-10, luminosity and per-pair trace at 1e-10,
identical Green-cache histories); the zero-width convention of slice 1; and PICPoissonSolver() with every
keyword at its default running and matching the oracle."""
import numpy as np
import pytest

from helpers import beams, oracle_options, oracle_params, E_PARAMS, P_PARAMS
from test_gpu_parity import check, run_both

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,ns,opts", [
    ("equal_area", 7, dict()),
    ("equal_area", 5, dict(interaction_grid="node")),
    ("equal_count", 7, dict()),
    ("equal_count", 4, dict(deposit_method="TSC")),
    ("equal_width", 7, dict()),
    ("equal_spaced", 5, dict(interaction_grid="node")),
])
def test_slicing_method_collides_match_oracle(method, ns, opts):
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), slicing=ob.LongitudinalSlicing(nslices=ns, method=method), **opts)
    check(run_both(s, 30000, 20000, turns=2, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2)))


def test_mixed_methods_and_resolution():
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), slicing1=ob.LongitudinalSlicing(nslices=6, method="equal_area", resolution=37),
                            slicing2=ob.LongitudinalSlicing(nslices=5, method="equal_count"))
    check(run_both(s, 20000, 15000, turns=2))


def test_default_solver_runs_and_matches_oracle():
    """PICPoissonSolver() with the reference's defaults: 128^2, one :equal_area slice, CIC, slice-pair cache."""
    import octo_b200 as ob
    s = ob.PICPoissonSolver()
    assert s.resolved_slicing1.method == "equal_area" and s.resolved_slicing1.nslices == 1
    check(run_both(s, 20000, 20000, turns=2))


@pytest.mark.parametrize("method", ["equal_area", "equal_width", "equal_count"])
def test_zero_width_and_tied_beams(method):
    """Every z equal: :equal_area / :equal_width file all particles into slice 1 (runtests.jl:4540-4560);
    :equal_count splits them by rank.  The collide still matches the oracle."""
    import octo_b200 as ob
    from oracle import oracle as orc
    e, p = beams(4000, 3000)
    e[4] = 1.5e-3
    s = ob.PICPoissonSolver(grid=(32, 32), slicing=ob.LongitudinalSlicing(nslices=4, method=method))
    o = orc.Oracle(oracle_options(s))
    pe, pp = oracle_params()
    be = ob.Beam.from_numpy(e, ob.BeamParams(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"], E_PARAMS["r0"],
                                             E_PARAMS["npart"]))
    bp = ob.Beam.from_numpy(p, ob.BeamParams(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"], P_PARAMS["r0"],
                                             P_PARAMS["npart"]))
    ctx = ob.Context(s, 0)
    lg = ctx.collide(be, bp, turn=1)
    lo = o.collide(e, p, pe, pp)
    assert abs(lg / lo - 1) < 1e-10
    assert np.allclose(be.numpy(), e, rtol=1e-10, atol=1e-10) and np.allclose(bp.numpy(), p, rtol=1e-10, atol=1e-10)
    assert [(a, b) for a, b, _ in ctx.pair_luminosity_trace()] == [(a, b) for a, b, _ in o.pair_trace()]
    ctx.close()
