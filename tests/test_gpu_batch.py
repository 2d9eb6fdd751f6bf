"""Independent collides in one batch (octo_pic_collide_batch), the multi-collision form of the batched
scan: seeded cases of uneven particle counts, slice counts, grids (2^a and 3*2^a) and aspect ratios,
each checked against the FP64 oracle at the contract tolerance (atol = rtol = 1e-10, identical
Green-cache histories), a batch shown bit-identical to the same collides run one by one, and a failing
collide shown not to disturb the others."""
import numpy as np
import pytest
import torch

from helpers import beams, oracle_options, oracle_params, within, E_PARAMS, P_PARAMS

pytestmark = pytest.mark.gpu

ATOL = RTOL = 1e-10


def scan_cases(n_cases, seed=20261203, nmax=30000):
    """Seeded draw in the shape of the scan: N log-uniform per beam, S in 3..9, grid in {48, 64, 96, 128},
    sigma_x / sigma_y log-uniform in [1, 25] with sigma_y = 8.5 um (sizes reduced so the oracle runs fast)."""
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(n_cases):
        n1, n2 = (int(np.exp(rng.uniform(np.log(3000), np.log(nmax)))) for _ in range(2))
        s1, s2 = (int(rng.integers(3, 10)) for _ in range(2))
        g = int(rng.choice([48, 64, 96, 128]))
        aspect = float(np.exp(rng.uniform(0, np.log(25))))
        sx = 8.5e-6 * aspect
        cases.append(dict(n1=n1, n2=n2, s1=s1, s2=s2, grid=(g, g), e_sigma=(sx, 8.5e-6, 7e-3),
                          p_sigma=(sx, 8.5e-6, 6e-2), seed=int(rng.integers(1, 2**31))))
    return cases


def _solver(ob, case):
    return ob.PICPoissonSolver(grid=case["grid"],
                               slicing1=ob.LongitudinalSlicing(nslices=case["s1"], method="normal_quantile"),
                               slicing2=ob.LongitudinalSlicing(nslices=case["s2"], method="normal_quantile"))


def _params(ob):
    pe = ob.BeamParams(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"], E_PARAMS["r0"], E_PARAMS["npart"])
    pp = ob.BeamParams(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"], P_PARAMS["r0"], P_PARAMS["npart"])
    return pe, pp


def _setup(ob, cases, dtype=torch.float64):
    pe, pp = _params(ob)
    host, dev, ctxs = [], [], []
    for c in cases:
        e, p = beams(c["n1"], c["n2"], c["e_sigma"], c["p_sigma"], seed=c["seed"])
        if dtype == torch.float32:
            e, p = e.astype(np.float32).astype(np.float64), p.astype(np.float32).astype(np.float64)
        host.append((e, p))
        dev.append((ob.Beam.from_numpy(e, pe, dtype=dtype), ob.Beam.from_numpy(p, pp, dtype=dtype)))
        ctxs.append(ob.Context(_solver(ob, c), 0, dtype))
    return host, dev, ctxs


def test_scan_batch_matches_oracle():
    import octo_b200 as ob
    from oracle import oracle as orc
    cases = scan_cases(6)
    host, dev, ctxs = _setup(ob, cases)
    oracles = [orc.Oracle(oracle_options(_solver(ob, c))) for c in cases]
    ope, opp = oracle_params()
    for turn in (1, 2):
        lums = ob.collide_batch(ctxs, [d[0] for d in dev], [d[1] for d in dev], turn=turn)
        for k, c in enumerate(cases):
            e, p = host[k]
            lo = oracles[k].collide(e, p, ope, opp)
            assert abs(lums[k] / lo - 1) <= 1e-10, (k, c, lums[k], lo)
            assert within(dev[k][0].numpy(), e, ATOL, RTOL) <= 1.0, (k, c)
            assert within(dev[k][1].numpy(), p, ATOL, RTOL) <= 1.0, (k, c)
            assert ctxs[k].green_cache_stats() == oracles[k].cache_stats(), (k, c)
    for c in ctxs:
        c.close()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_batch_is_bit_identical_to_sequential_collides(dtype):
    import octo_b200 as ob
    cases = scan_cases(5, seed=7)
    _, dev_a, ctx_a = _setup(ob, cases, dtype)
    _, dev_b, ctx_b = _setup(ob, cases, dtype)
    for turn in (1, 2):
        lum_a = ob.collide_batch(ctx_a, [d[0] for d in dev_a], [d[1] for d in dev_a], turn=turn)
        lum_b = [ctx_b[k].collide(dev_b[k][0], dev_b[k][1], turn=turn) for k in range(len(cases))]
        assert lum_a == lum_b
        for (a1, a2), (b1, b2) in zip(dev_a, dev_b):
            assert torch.equal(a1.coords, b1.coords) and torch.equal(a2.coords, b2.coords)
    for c in ctx_a + ctx_b:
        c.close()


def test_failing_collide_leaves_the_rest_of_the_batch_intact():
    import octo_b200 as ob
    cases = scan_cases(3, seed=11)
    _, dev, ctxs = _setup(ob, cases)
    _, ref, ctx_ref = _setup(ob, cases)
    dev[1][0].coords[0, 17] = float("nan")
    with pytest.raises(ob.CollisionError) as err:
        ob.collide_batch(ctxs, [d[0] for d in dev], [d[1] for d in dev], turn=3)
    assert err.value.code == 1 and "collide 1" in str(err.value)
    for k in (0, 2):
        ctx_ref[k].collide(ref[k][0], ref[k][1], turn=3)
        assert torch.equal(dev[k][0].coords, ref[k][0].coords) and torch.equal(dev[k][1].coords, ref[k][1].coords)
    for c in ctxs + ctx_ref:
        c.close()
