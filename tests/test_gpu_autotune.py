"""The launch-shape autotuner (octo_pic_autotune): its tuning collides run every candidate shape, and the
beams they leave are bit-identical to the same number of collides in the default shape on another context
(charge sums are exact integers and each particle's kick is its own, so a shape changes only the time);
the Python wrapper tunes on copies and leaves the caller's beams untouched."""
import ctypes as C

import pytest
import torch

from helpers import beams, E_PARAMS, P_PARAMS

pytestmark = pytest.mark.gpu


def _setup():
    import octo_b200 as ob
    e, p = beams(20000, 12000)
    pe = ob.BeamParams(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"], E_PARAMS["r0"], E_PARAMS["npart"])
    pp = ob.BeamParams(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"], P_PARAMS["r0"], P_PARAMS["npart"])
    solver = ob.PICPoissonSolver(grid=(64, 64), interaction_grid="node",
                                 slicing=ob.LongitudinalSlicing(nslices=4, method="normal_quantile"))
    return ob, e, p, pe, pp, solver


def test_autotune_shapes_leave_results_unchanged():
    ob, e, p, pe, pp, solver = _setup()
    from octo_b200 import _lib
    ea, pa = ob.Beam.from_numpy(e, pe), ob.Beam.from_numpy(p, pp)
    eb, pb = ob.Beam.from_numpy(e, pe), ob.Beam.from_numpy(p, pp)
    rt = ob.StrongStrongRuntime()
    ca, cb = rt.context("tuned", solver, 0), rt.context("default", solver, 0)
    b1, b2, p1, p2 = ea.to_c(), pa.to_c(), pe.to_c(), pp.to_c()
    choice = C.c_int32(-1)
    st = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib().octo_pic_autotune(ca._ptr, C.byref(b1), C.byref(b2), C.byref(p1), C.byref(p2), 1,
                                      C.byref(choice), C.c_void_p(st))
    assert rc == _lib.OCTO_OK, _lib.last_error(ca._ptr)
    assert 0 <= choice.value < 4
    for _ in range(5):  # the untimed collide and the four timed shapes of one round
        cb.collide(eb, pb)
    assert torch.equal(ea.coords, eb.coords) and torch.equal(pa.coords, pb.coords)
    la, lb = ca.collide(ea, pa), cb.collide(eb, pb)  # the chosen shape against the default one
    assert la == lb
    assert torch.equal(ea.coords, eb.coords) and torch.equal(pa.coords, pb.coords)
    rt.close()


def test_autotune_wrapper_tunes_on_copies():
    ob, e, p, pe, pp, solver = _setup()
    be, bp = ob.Beam.from_numpy(e, pe), ob.Beam.from_numpy(p, pp)
    e0, p0 = be.coords.clone(), bp.coords.clone()
    rt = ob.StrongStrongRuntime()
    ctx = rt.context("ip", solver, 0)
    k = ctx.autotune(be, bp, rounds=1)
    assert 0 <= k < len(ctx.AUTOTUNE_SHAPES)
    assert torch.equal(be.coords, e0) and torch.equal(bp.coords, p0)
    with pytest.raises(ob.ArgumentError):
        ctx.autotune(be, bp, rounds=0)
    rt.close()
