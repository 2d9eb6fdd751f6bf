"""The plain PIC collide does not depend on the order of particles inside a slice: the working copy grouped by
transverse position (the default, octo_set_particle_order(1)) and the caller order give bit-identical
coordinates, luminosities, per-pair luminosity traces and Green-cache counters, over several turns, for
:slice_pair, :source_slice and :node grids, CIC and TSC, and the float32 precision form."""
import pytest

from helpers import beams, E_PARAMS, P_PARAMS

pytestmark = pytest.mark.gpu


def _run(solver, spatial, dtype, turns=2):
    import torch
    import octo_b200 as ob
    e, p = beams(60000, 30000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2))
    pe = ob.BeamParams(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"], E_PARAMS["r0"], E_PARAMS["npart"])
    pp = ob.BeamParams(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"], P_PARAMS["r0"], P_PARAMS["npart"])
    be = ob.Beam.from_numpy(e, pe, dtype=dtype)
    bp = ob.Beam.from_numpy(p, pp, dtype=dtype)
    ctx = ob.Context(solver, 0, dtype)
    ctx.set_particle_order(spatial)
    out = []
    for t in range(turns):
        lum = ctx.collide(be, bp, turn=t + 1)
        out.append((lum, ctx.pair_luminosity_trace(), ctx.green_cache_stats(), ctx.last_report.dropped))
    res = (be.coords.clone(), bp.coords.clone(), out)
    ctx.close()
    return res


@pytest.mark.parametrize("opts,dtype_name", [
    (dict(), "float64"),
    (dict(interaction_grid="node"), "float64"),
    (dict(deposit_method="TSC", field_derivative="fourth"), "float64"),
    (dict(interaction_grid="node"), "float32"),
    (dict(slice_interpolation="quadratic"), "float32"),
    (dict(interaction_grid="source_slice"), "float64"),
])
def test_spatial_order_is_bit_identical(opts, dtype_name):
    import torch
    import octo_b200 as ob
    dtype = getattr(torch, dtype_name)
    solver = ob.PICPoissonSolver(grid=(64, 64), slicing=ob.LongitudinalSlicing(nslices=7, method="normal_quantile"),
                                 **opts)
    a = _run(solver, True, dtype)
    b = _run(solver, False, dtype)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert a[2] == b[2]
