"""Captured collide graphs (octo_set_collide_graph): once two consecutive collides have the same schedule the
next one is captured, and later collides replay it behind a device guard that checks the slice counts, starts
and collision order and recomputes the slice drifts.  A replayed collide is bit-identical to the ordinary one
-- coordinates, luminosities, per-pair traces, Green-cache counters -- over turns with Linear6D maps between
them, in both forms and on :slice_pair and :node grids; replayed collides match the oracle at the contract's
1e-10; and a collide whose schedule changed is declined by the guard and runs the ordinary path, still at
1e-10 against the oracle given the same history."""
import numpy as np
import pytest

from helpers import beams, oracle_options, oracle_params, within, E_PARAMS, P_PARAMS

pytestmark = pytest.mark.gpu

E_BEAM = dict(beta=(0.55, 0.056, 0.7e-2 / 5.5e-4), alpha=(0.0, 0.0, 0.0), tune=(0.228, 0.21, 0.0))
P_BEAM = dict(beta=(0.8, 0.072, 6e-2 / 6.6e-4), alpha=(0.0, 0.0, 0.0), tune=(0.228, 0.21, 0.0))


def _params(ob):
    pe = ob.BeamParams(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"], E_PARAMS["r0"], E_PARAMS["npart"])
    pp = ob.BeamParams(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"], P_PARAMS["r0"], P_PARAMS["npart"])
    return pe, pp


def _run(solver, graph, dtype_name, turns=6, n1=40000, n2=20000, ztunes=(0.0, 0.0)):
    import torch
    import octo_b200 as ob
    dtype = getattr(torch, dtype_name)
    e, p = beams(n1, n2, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2))
    pe, pp = _params(ob)
    be = ob.Beam.from_numpy(e, pe, dtype=dtype)
    bp = ob.Beam.from_numpy(p, pp, dtype=dtype)
    me = ob.Linear6D(E_BEAM["beta"], E_BEAM["alpha"], E_BEAM["tune"][:2] + (ztunes[0],))
    mp = ob.Linear6D(P_BEAM["beta"], P_BEAM["alpha"], P_BEAM["tune"][:2] + (ztunes[1],))
    ctx = ob.Context(solver, 0, dtype)
    ctx.set_collide_graph(graph)
    out = []
    for t in range(turns):
        lum = ctx.collide(be, bp, turn=t + 1)
        r = ctx.last_report
        out.append((lum, ctx.pair_luminosity_trace(), ctx.green_cache_stats(), r.dropped, r.n_batches))
        out[-1] = out[-1] + (r.replayed,)
        me.track(be)
        mp.track(bp)
    stats = ctx.collide_graph_stats()
    res = (be.coords.clone(), bp.coords.clone(), out, stats)
    ctx.close()
    return res


@pytest.mark.parametrize("opts,dtype_name", [
    (dict(interaction_grid="node"), "float64"),
    (dict(), "float64"),
    (dict(green_cache="none", slice_interpolation="quadratic", deposit_method="TSC"), "float64"),
    (dict(interaction_grid="node"), "float32"),
    (dict(slice_interpolation="quadratic"), "float32"),
])
def test_replayed_collides_are_bit_identical(opts, dtype_name):
    import torch
    import octo_b200 as ob
    solver = ob.PICPoissonSolver(grid=(64, 64), slicing=ob.LongitudinalSlicing(nslices=7, method="normal_quantile"),
                                 **opts)
    a = _run(solver, True, dtype_name)
    b = _run(solver, False, dtype_name)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert [x[:5] for x in a[2]] == [x[:5] for x in b[2]]
    # turns 1-2 ordinary (the second captures), 3-6 replayed
    assert [x[5] for x in a[2]] == [0, 0, 1, 1, 1, 1], a[2]
    assert a[3][:2] == (1, 4) and a[3][2:] == (0, 0), a[3]
    assert [x[5] for x in b[2]] == [0] * 6 and b[3] == (0, 0, 0, 0)


def test_replay_across_reordered_collisions():
    """Longitudinal tunes move the slice centroids every turn, and pairs with nearly equal collision times
    change places in the collision order; as long as the wavefronts are unchanged the guard accepts the graph
    and the host folds the pair luminosities in the new order.  Bit-identical to the ordinary path over 16
    turns, with at least one replayed turn whose order differs from the previous turn's."""
    import torch
    import octo_b200 as ob
    solver = ob.PICPoissonSolver(grid=(64, 64), interaction_grid="node",
                                 slicing=ob.LongitudinalSlicing(nslices=15, method="normal_quantile"))
    a = _run(solver, True, "float64", turns=16, ztunes=(-0.069, -0.01))
    b = _run(solver, False, "float64", turns=16, ztunes=(-0.069, -0.01))
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert [x[:5] for x in a[2]] == [x[:5] for x in b[2]]
    assert a[3][1] >= 1, a[3]
    orders = [[(i, j) for i, j, _ in x[1]] for x in a[2]]
    reordered = [t for t in range(1, 16) if a[2][t][5] and orders[t] != orders[t - 1]]
    assert reordered, (a[3], [x[5] for x in a[2]])


def _oracle_turns(solver, states, ob):
    """Collide each (e, p) pair of states on the GPU (reloaded into the same device buffers) and in the oracle,
    one context each, in order; returns per turn (errors, replayed)."""
    import torch
    from oracle import oracle as orc
    pe, pp = _params(ob)
    e0, p0 = states[0]
    be = ob.Beam.from_numpy(e0, pe)
    bp = ob.Beam.from_numpy(p0, pp)
    ctx = ob.Context(solver, 0, torch.float64)
    oracle = orc.Oracle(oracle_options(solver))
    ope, opp = oracle_params()
    out = []
    for t, (e, p) in enumerate(states):
        e, p = e.copy(), p.copy()
        be.coords.copy_(torch.from_numpy(e))
        bp.coords.copy_(torch.from_numpy(p))
        lum_g = ctx.collide(be, bp, turn=t + 1)
        rep = ctx.last_report.replayed
        lum_o = oracle.collide(e, p, ope, opp)
        out.append(dict(replayed=rep, lum=abs(lum_g / lum_o - 1), e=within(be.numpy(), e, 1e-10, 1e-10),
                        p=within(bp.numpy(), p, 1e-10, 1e-10), cache=(ctx.green_cache_stats(), oracle.cache_stats()),
                        trace=[(a, b) for a, b, _ in ctx.pair_luminosity_trace()] == [(a, b) for a, b, _ in
                                                                                      oracle.pair_trace()]))
    stats = ctx.collide_graph_stats()
    ctx.close()
    return out, stats


def _check(out):
    for r in out:
        assert r["e"] <= 1.0 and r["p"] <= 1.0 and r["lum"] <= 1e-10 and r["trace"], r
        assert r["cache"][0] == r["cache"][1], r


@pytest.mark.parametrize("grid_mode", ["slice_pair", "node"])
def test_replayed_collides_match_the_oracle(grid_mode):
    """Five collides of the same beams: the third to fifth replay the graph (the Green cache keeps counting hits
    as the oracle's does)."""
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), interaction_grid=grid_mode,
                            slicing=ob.LongitudinalSlicing(nslices=5, method="normal_quantile"))
    e, p = beams(6000, 4000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2))
    out, stats = _oracle_turns(s, [(e, p)] * 5, ob)
    _check(out)
    assert [r["replayed"] for r in out] == [0, 0, 1, 1, 1] and stats == (1, 3, 0, 0), (out, stats)


def test_changed_counts_replay_and_a_changed_schedule_is_declined():
    """:equal_width slices: the counts follow the z distribution.  Two collides of one beam pair capture the
    graph.  Another proton sample has other slice counts and starts but the same wavefronts and no empty slice:
    the guard rewrites the ranges, fixed-point scales and kick block map and replays it.  A proton bunch with a
    gap of six sigma in z leaves two of its slices empty, which changes the schedule: the guard declines it, the
    graph is dropped and the ordinary path runs; the next collide repeats that schedule and captures anew.
    Every collide against the oracle at 1e-10."""
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), slicing=ob.LongitudinalSlicing(nslices=6, method="equal_width"))
    e, p = beams(6000, 4000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2))
    _, p2 = beams(6000, 4000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2), seed=7)
    p3 = p.copy()
    p3[4] = np.where(p3[4] > 0, p3[4] + 6 * 6e-2, p3[4])
    out, stats = _oracle_turns(s, [(e, p), (e, p), (e, p2), (e, p3), (e, p3), (e, p3)], ob)
    _check(out)
    assert [r["replayed"] for r in out] == [0, 0, 1, 0, 0, 1], out
    assert stats == (2, 2, 1, 0), stats


def test_slices_that_outgrow_the_graph_are_declined_and_recaptured():
    """The same schedule with an end slice grown seventyfold (1000 protons of the third :equal_width slice moved into
    the first, the bunch's extent unchanged): the kick's block map has no room for it, the guard declines, the
    ordinary path runs and captures the schedule again with room for the new counts, and the next collide replays
    that graph."""
    from oracle import oracle as orc
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(64, 64), slicing=ob.LongitudinalSlicing(nslices=6, method="equal_width"))
    e, p = beams(6000, 4000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2))
    b = orc.slices(p[4], 6, method="equal_width")[0]
    third = np.where((p[4] >= b[2]) & (p[4] < b[3]))[0]
    p5 = p.copy()
    p5[4, third[:1000]] = 0.5 * (b[0] + b[1])
    out, stats = _oracle_turns(s, [(e, p), (e, p), (e, p), (e, p5), (e, p5)], ob)
    _check(out)
    assert [r["replayed"] for r in out] == [0, 0, 1, 0, 1], out
    assert stats == (2, 2, 1, 0), stats


def test_a_nonfinite_coordinate_during_replays_is_reported():
    """A NaN that reaches the beams after the graph was captured: the slicing flags it, the guard declines and
    drops the graph, and the ordinary path reports it as a collide without a graph would (OCTO_ERR_NONFINITE,
    the particle, the turn).  The context then collides clean beams again: the first of them repeats the last
    ordinary schedule and captures anew, the next ones replay."""
    import torch
    import octo_b200 as ob
    s = ob.PICPoissonSolver(grid=(32, 32), slicing=ob.LongitudinalSlicing(nslices=4, method="normal_quantile"))
    e, p = beams(3000, 2000)
    pe, pp = _params(ob)
    be = ob.Beam.from_numpy(e, pe)
    bp = ob.Beam.from_numpy(p, pp)
    ctx = ob.Context(s, 0, torch.float64)
    for t in range(3):
        be.coords.copy_(torch.from_numpy(e))
        bp.coords.copy_(torch.from_numpy(p))
        ctx.collide(be, bp, turn=t + 1)
    assert ctx.last_report.replayed == 1
    bad = e.copy()
    bad[4, 1234] = np.nan
    be.coords.copy_(torch.from_numpy(bad))
    bp.coords.copy_(torch.from_numpy(p))
    with pytest.raises(ob.CollisionError) as err:
        ctx.collide(be, bp, turn=4)
    assert err.value.code == 1 and "1235" in str(err.value) and "turn 4" in str(err.value), str(err.value)
    assert err.value.report.role == 3 and err.value.report.replayed == 0
    out = []
    for t in range(3):
        be.coords.copy_(torch.from_numpy(e))
        bp.coords.copy_(torch.from_numpy(p))
        out.append((ctx.collide(be, bp, turn=5 + t), ctx.last_report.replayed))
    assert all(np.isfinite(l) for l, _ in out) and [r for _, r in out] == [0, 1, 1], out
    assert ctx.collide_graph_stats()[2] == 1
    ctx.close()


def test_two_interaction_points_replay_side_by_side():
    """Two contexts of one runtime (two interaction points, different grids) collided in turn, with Linear6D maps
    between: a buffer reallocated by one context invalidates the other's graph until both have settled, after
    which both replay.  Bit-identical to the same sequence with collide graphs off."""
    import torch
    import octo_b200 as ob

    def run(graph):
        e, p = beams(20000, 10000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2))
        pe, pp = _params(ob)
        be = ob.Beam.from_numpy(e, pe)
        bp = ob.Beam.from_numpy(p, pp)
        me = ob.Linear6D(E_BEAM["beta"], E_BEAM["alpha"], E_BEAM["tune"])
        mp = ob.Linear6D(P_BEAM["beta"], P_BEAM["alpha"], P_BEAM["tune"])
        rt = ob.StrongStrongRuntime()
        sl = ob.LongitudinalSlicing(nslices=5, method="normal_quantile")
        ctx = [rt.context("ip1", ob.PICPoissonSolver(grid=(64, 64), interaction_grid="node", slicing=sl), 0),
               rt.context("ip2", ob.PICPoissonSolver(grid=(32, 32), slicing=sl), 0)]
        for c in ctx:
            c.set_collide_graph(graph)
        lums, replayed = [], []
        for t in range(8):
            for c in ctx:
                lums.append(c.collide(be, bp, turn=t + 1))
                replayed.append(c.last_report.replayed)
                me.track(be)
                mp.track(bp)
        stats = [c.collide_graph_stats() for c in ctx]
        out = (be.coords.clone(), bp.coords.clone(), lums, replayed, stats)
        rt.close()
        return out

    a, b = run(True), run(False)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]) and a[2] == b[2]
    assert a[3][-4:] == [1, 1, 1, 1], a[3]
    assert all(s[1] >= 2 for s in a[4]) and all(s[3] == 0 for s in a[4]), a[4]
    assert b[3] == [0] * 16
