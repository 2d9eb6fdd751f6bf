"""The learned field correction inside the collide (octo_set_field_correction) and its training data.

- Training pairs from the probe collides are well formed (finite, the interior covered) and, for a plain
  Gaussian slice, the Gaussian-subtracted hybrid's field is already close to the fine plain-PIC field.
- A network whose parameters are all zero adds nothing: collides with and without it are bit-identical, in
  the plain form (float64) and in the precision form (float32, where a plane holds a difference of two
  planes' fields and gets the difference of their corrections).
- A tolerance the correction exceeds makes the learned form fall back to the plain solver, bit-identical to
  a collide of that solver from the same beams.
- The committed trained networks lower the coarse solvers' RMS field error against the fine plain-PIC
  solver on held-out slices (seeds the training never saw), and keep the field within 1 % RMS of exact
  Bassetti-Erskine at aspect ratios 1, 5, 11.2 and 25."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_BEAM = dict(beta=(0.55, 0.056, 0.7e-2 / 5.5e-4), sigma=(95e-6, 8.5e-6, 7e-3), rng_id=1)
P_BEAM = dict(beta=(0.8, 0.072, 6e-2 / 6.6e-4), sigma=(95e-6, 8.5e-6, 6e-2), rng_id=2)


def _beams(ob, n1, n2, dtype):
    import torch
    e = ob.Beam.gaussian(n1, seed=5, charge=-1.0, mc2=ob.EMASS_EV, E0=10e9, npart=1.7e11, **E_BEAM)
    p = ob.Beam.gaussian(n2, seed=5, charge=1.0, mc2=ob.PMASS_EV, E0=275e9, npart=6.9e10, **P_BEAM)
    return e.astype(dtype), p.astype(dtype)


@pytest.mark.parametrize("coarse", ["hybrid", "pic"])
def test_training_pairs_are_well_formed(coarse):
    import torch
    from octo_b200 import learned as L
    X, T, M, F = L.make_dataset(8, seed=77, coarse=coarse)
    assert torch.isfinite(T).all() and torch.isfinite(F).all() and torch.isfinite(X.float()).all()
    interior = (48 - 2 * L.EDGE) ** 2
    # the probes cover the density's box; the hybrid's mesh also spans +-5 sigma of its Gaussian fit
    assert float(M.sum(dim=(1, 2)).min()) > 0.15 * interior
    # a plain Gaussian slice (kind 0): the hybrid subtracts it and adds its field back analytically
    rel = float((T[0] * M[0, ..., None]).norm() / (F[0] * M[0, ..., None]).norm())
    if coarse == "hybrid":
        assert rel < 0.05, rel


@pytest.mark.parametrize("dtype_name", ["float64", "float32"])
def test_zero_network_leaves_the_collide_unchanged(dtype_name):
    import torch
    import octo_b200 as ob
    from octo_b200 import learned as L
    dtype = getattr(torch, dtype_name)
    solver = L.coarse_solver("pic", 32, slicing=ob.LongitudinalSlicing(nslices=5, method="normal_quantile"))
    net = L.FieldCorrectionNet(32, 32, max_batch=32)
    net.set_params(np.zeros(net.num_params, dtype=np.float32))
    e1, p1 = _beams(ob, 20000, 10000, dtype)
    e2, p2 = ob.Beam(e1.coords.clone(), e1.params), ob.Beam(p1.coords.clone(), p1.params)
    plain = ob.Context(solver, 0, dtype)
    form = L.LearnedForm(solver, solver, net, tolerance=1.0, dtype=dtype)
    l1 = plain.collide(e1, p1, turn=1)
    l2 = form.collide(e2, p2, turn=1)
    assert form.fallbacks == 0
    assert l1 == l2
    assert torch.equal(e1.coords, e2.coords) and torch.equal(p1.coords, p2.coords)
    plain.close(); form.close(); net.close()


def test_fallback_runs_the_plain_solver():
    import torch
    import octo_b200 as ob
    from octo_b200 import learned as L
    sl = ob.LongitudinalSlicing(nslices=5, method="normal_quantile")
    coarse = L.coarse_solver("pic", 32, slicing=sl)
    plain_solver = ob.PICPoissonSolver(grid=(64, 64), slicing=sl)
    net = L.FieldCorrectionNet(32, 32, max_batch=32, seed=9)  # random weights: large corrections
    e1, p1 = _beams(ob, 20000, 10000, torch.float64)
    e2, p2 = ob.Beam(e1.coords.clone(), e1.params), ob.Beam(p1.coords.clone(), p1.params)
    form = L.LearnedForm(coarse, plain_solver, net, tolerance=1e-9)
    plain = ob.Context(plain_solver, 0)
    l_form = form.collide(e1, p1, turn=1)
    assert form.fallbacks == 1 and form.planes_over_tolerance() > 0
    l_plain = plain.collide(e2, p2, turn=1)
    assert l_form == l_plain
    assert torch.equal(e1.coords, e2.coords) and torch.equal(p1.coords, p2.coords)
    form.close(); plain.close(); net.close()


@pytest.mark.parametrize("coarse", ["hybrid", "pic"])
def test_trained_network_lowers_the_heldout_field_error(coarse):
    from octo_b200 import learned as L
    net, meta = L.load_net(coarse=coarse, max_batch=64)
    X, T, M, F = L.make_dataset(128, seed=4242, coarse=coarse)  # seeds disjoint from the training run's
    r = L.evaluate(net, X, T, M, F)
    assert r["learned"] < 0.5 * r["hybrid"], r
    net.close()


@pytest.mark.parametrize("coarse", ["hybrid", "pic"])
def test_learned_form_field_error_against_bassetti_erskine(coarse):
    import torch
    import octo_b200 as ob
    from octo_b200 import learned as L
    from octo_b200.diagnostics import field_error
    net, meta = L.load_net(coarse=coarse, max_batch=64)
    solver = L.coarse_solver(coarse, 48)
    sy = 8.5e-6
    for aspect in (1.0, 5.0, 95e-6 / 8.5e-6, 25.0):
        for dtype in (torch.float64, torch.float32) if coarse == "pic" else (torch.float64,):
            err = field_error(solver, aspect * sy, sy, dtype, 0, correction=(net, L.OUT_SCALE, 1e30, L.EDGE))
            assert err["rms"] < 0.01, (coarse, aspect, dtype, err)
    net.close()
