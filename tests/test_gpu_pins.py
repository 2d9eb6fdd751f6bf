"""Pins of the benchmarked path on the GPU against the oracle.

Every piece the benchmark's timed turn runs is checked here on the device, at the benchmark's own sizes
where that matters:
- the seeded beam generator (octo_beam_gaussian) against the oracle's Beam.jl restatement, elementwise;
- the Linear6D one-turn map (octo_linear6d) against linear6d.jl's matrix product;
- the int64 fixed-point charge grids, read back through octo_capture_charge_plane, bit-equal to the
  oracle's fixed-point deposit (CIC / TSC x :slice_pair / :node, every plane of a pair);
- one collide plus both one-turn maps at exactly the benchmark configuration (2.56M / 1.024M, 15
  :normal_quantile centroid slices, 128^2 :node, CIC, luminosity on) at the reference's backend-consistency
  tolerance atol = rtol = 1e-10 (Contracts.jl:99-136), with the per-pair luminosity trace and counters;
- the reference's production golden luminosity 1.0254361754701657e+30
  (docs/history/cpu_benchmark_history.tsv:2,6,10; inputs of profiling/benchmark_collide_cpu.jl:88-126)
  reproduced by the GPU collide, with the cold-cache counters (0 hits, 450 misses, 0 rebuilds)."""
import os

import numpy as np
import pytest

from helpers import beams, oracle_options, oracle_params, within, E_PARAMS, P_PARAMS

pytestmark = pytest.mark.gpu

ATOL = RTOL = 1e-10
SEED = 123456789
# the benchmark workload's beams (flat 95 / 8.5 um for both rings)
BENCH_E = dict(beta=(0.55, 0.056, 0.7e-2 / 5.5e-4), sigma=(95e-6, 8.5e-6, 7e-3))
BENCH_P = dict(beta=(0.8, 0.072, 6e-2 / 6.6e-4), sigma=(95e-6, 8.5e-6, 6e-2))


def _ob():
    import octo_b200 as ob
    return ob


def _params(ob):
    pe = ob.BeamParams(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"], E_PARAMS["r0"], E_PARAMS["npart"])
    pp = ob.BeamParams(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"], P_PARAMS["r0"], P_PARAMS["npart"])
    return pe, pp


@pytest.mark.parametrize("n", [1, 4095, 100_000, 2_560_000])
@pytest.mark.parametrize("which", ["electron", "proton"])
def test_device_beam_generator_matches_oracle(n, which):
    """Beam.jl:475-515 on the device: Philox normals, cutoff, standardisation, Twiss scaling.  The only
    differences are the device's log / sin / cos ulps and the order of the mean and variance sums."""
    import torch
    from oracle import oracle as orc
    ob = _ob()
    spec = dict(beta=(0.55, 0.056, 12.727272727272727), alpha=(0.3, -0.2, 0.0), sigma=(106e-6, 9.5e-6, 7e-3),
                rng_id=1) if which == "electron" else dict(beta=(0.8, 0.072, 90.9090909090909), alpha=(0.0, 0.0, 0.0),
                                                           sigma=(95e-6, 8.5e-6, 6e-2), rng_id=2)
    got = ob.Beam.gaussian(n, seed=SEED, **spec).numpy()
    want = orc.beam_gaussian(n, seed=SEED, **spec)
    assert got.shape == want.shape and np.all(np.isfinite(got))
    if n == 1:  # a single particle standardises to the origin (zero spread), as Beam.jl:148-160 does
        assert np.array_equal(got, want) and not np.any(got)
        return
    scale = np.sqrt(np.mean(want ** 2, axis=1, keepdims=True))
    err = np.abs(got - want) / (scale + np.abs(want))
    assert float(err.max()) < 1e-14, float(err.max())


def test_linear6d_matches_oracle():
    """linear6d.jl:110-121 (x' = M x per particle) against the oracle, three turns per launch, on the
    benchmark's electron beam; the matrix built by the Python mirror equals the oracle's (linear6d.jl:233-280)."""
    import torch
    from oracle import oracle as orc
    ob = _ob()
    beta, alpha, tune = (0.55, 0.056, 12.727272727272727), (0.25, -0.4, 0.0), (0.08, 0.06, -0.069)
    m = ob.Linear6D(beta, alpha, tune)
    m_ref = orc.linear6d_matrix(beta, alpha, tune)
    assert np.allclose(m.matrix, m_ref, rtol=1e-15, atol=1e-15)
    e = orc.beam_gaussian(1_000_003, seed=SEED, rng_id=1, **BENCH_E)
    be = ob.Beam.from_numpy(e, ob.BeamParams())
    m.track(be, turns=3)
    for _ in range(3):
        orc.linear6d(m.matrix, e)
    got = be.numpy()
    scale = np.sqrt(np.mean(e ** 2, axis=1, keepdims=True))
    err = float((np.abs(got - e) / scale).max())
    assert err < 1e-15, err


def _first_pair(solver, e, p):
    """The first slice pair in collision order (it runs in the first wavefront, so both of its source
    slices are still the untouched inputs)."""
    from oracle import oracle as orc
    o = orc.Oracle(oracle_options(solver))
    pe, pp = oracle_params()
    o.collide(e.copy(), p.copy(), pe, pp)
    i, j, _ = o.pair_trace()[0]
    return i, j


@pytest.mark.parametrize("method", ["CIC", "TSC"])
@pytest.mark.parametrize("mode", ["slice_pair", "node"])
def test_charge_grid_bit_exact(method, mode):
    """The int64 fixed-point charge grid of every plane of both directions of the first pair is bit-equal
    to the oracle's fixed-point deposit, on the same mesh (bit-equal origin and size) with the same scale."""
    from oracle import oracle as orc
    ob = _ob()
    solver = ob.PICPoissonSolver(grid=(64, 64), deposit_method=method, interaction_grid=mode,
                                 slicing=ob.LongitudinalSlicing(nslices=7, method="normal_quantile"))
    e, p = beams(40_000, 20_000, e_sigma=(95e-6, 8.5e-6, 7e-3), p_sigma=(95e-6, 8.5e-6, 6e-2))
    i, j = _first_pair(solver, e, p)
    pe, pp = oracle_params()
    ge, gp = _params(ob)
    nplanes = 3  # sL, sR and the third plane (:node Z with the longitudinal kick; none for linear :slice_pair)
    checked = 0
    for direction in (1, 2):
        for plane in range(nplanes if mode == "node" else 2):
            be = ob.Beam.from_numpy(e, ge)
            bp = ob.Beam.from_numpy(p, gp)
            rt = ob.StrongStrongRuntime()
            ctx = rt.context("ip", solver, 0)
            ctx.capture_charge_plane(i, j, direction, plane)
            ctx.collide(be, bp, turn=1)
            q_gpu, mesh_gpu, bits_gpu = ctx.captured_charge_plane()
            rt.close()
            o = orc.Oracle(oracle_options(solver, fixed=True))
            o.capture_plane(i, j, direction, plane)
            o.collide(e.copy(), p.copy(), pe, pp)
            q_ref, mesh_ref, bits_ref = o.captured_plane()
            assert mesh_gpu == mesh_ref, (direction, plane, mesh_gpu, mesh_ref)
            assert bits_gpu == bits_ref
            assert q_ref.any()
            diff = np.argwhere(q_gpu != q_ref)
            assert diff.size == 0, (direction, plane, len(diff), diff[:5].tolist())
            checked += 1
    assert checked == (6 if mode == "node" else 4)


def _oracle_threads():
    return max(1, os.cpu_count() or 1)


def test_benchmark_configuration_collide_and_maps():
    """One turn of the benchmarked workload on the GPU and on the oracle from identical inputs: collide
    (2.56M / 1.024M flat beams, 15 slices, 128^2 :node, CIC, second order, linear, luminosity on) then the
    linear uncoupled one-turn map of each ring."""
    from oracle import oracle as orc
    ob = _ob()
    solver = ob.PICPoissonSolver(grid=(128, 128), interaction_grid="node", deposit_method="CIC",
                                 slicing=ob.LongitudinalSlicing(nslices=15, method="normal_quantile",
                                                                center_position="centroid"))
    e = orc.beam_gaussian(2_560_000, seed=SEED, rng_id=1, **BENCH_E)
    p = orc.beam_gaussian(1_024_000, seed=SEED, rng_id=2, **BENCH_P)
    pe = orc.beam_params(-1.0, orc.EMASS_EV, 10e9, 1.7e11)
    pp = orc.beam_params(1.0, orc.PMASS_EV, 275e9, 6.9e10)
    ge = ob.BeamParams(-1.0, ob.EMASS_EV, 10e9, ob.RE, 1.7e11)
    gp = ob.BeamParams(1.0, ob.PMASS_EV, 275e9, ob.RE * ob.ME0 / ob.PMASS_EV, 6.9e10)
    be, bp = ob.Beam.from_numpy(e, ge), ob.Beam.from_numpy(p, gp)
    me = ob.Linear6D(BENCH_E["beta"], (0, 0, 0), (0.08, 0.06, -0.069))
    mp = ob.Linear6D(BENCH_P["beta"], (0, 0, 0), (0.228, 0.210, -0.01))
    rt = ob.StrongStrongRuntime()
    ctx = rt.context("ip", solver, 0)
    lum_g = ctx.collide(be, bp, turn=1)
    rep = ctx.last_report
    trace_g = ctx.pair_luminosity_trace()
    me.track(be)
    mp.track(bp)
    got_e, got_p = be.numpy(), bp.numpy()
    cache_g = ctx.green_cache_stats()
    rt.close()

    o = orc.Oracle(orc.OracleOptions(grid=(128, 128), interaction_grid="node", nslices1=15, nslices2=15,
                                     nthreads=_oracle_threads()))
    lum_o = o.collide(e, p, pe, pp)
    trace_o = o.pair_trace()
    orc.linear6d(me.matrix, e)
    orc.linear6d(mp.matrix, p)

    assert abs(lum_g / lum_o - 1) <= 1e-10, (lum_g, lum_o)
    assert [(a, b) for a, b, _ in trace_g] == [(a, b) for a, b, _ in trace_o]
    assert len(trace_g) == 225
    for (_, _, lg), (_, _, lo) in zip(trace_g, trace_o):
        assert abs(lg - lo) <= 1e-10 * abs(lo) + 1e-300
    assert within(got_e, e, ATOL, RTOL) <= 1.0
    assert within(got_p, p, ATOL, RTOL) <= 1.0
    assert rep.dropped == o.dropped()
    assert cache_g == o.cache_stats()


def test_reference_golden_luminosity_on_gpu():
    """The reference's production golden collide (profiling/benchmark_collide_cpu.jl:88-126): 2.56M / 1.024M
    seeded beams, 15 :normal_quantile centroid slices, 128^2 :slice_pair grids, CIC, :integrated Green
    function, slice-pair cache 0.5 / 0.25, one cold collide.  Its luminosity is 1.0254361754701657e+30
    (docs/history/cpu_benchmark_history.tsv:2,6,10) and the cache sees 450 misses."""
    ob = _ob()
    from oracle import oracle as orc
    solver = ob.PICPoissonSolver(grid=(128, 128), deposit_method="CIC",
                                 slicing=ob.LongitudinalSlicing(nslices=15, method="normal_quantile",
                                                                center_position="centroid"))
    espec = dict(beta=(0.55, 0.056, 0.7e-2 / 5.5e-4), sigma=(106e-6, 9.5e-6, 0.7e-2))
    pspec = dict(beta=(0.8, 0.072, 6e-2 / 6.6e-4), sigma=(95e-6, 8.5e-6, 6e-2))
    ge = ob.BeamParams(-1.0, ob.EMASS_EV, 10e9, ob.RE, 1.7203e11)
    gp = ob.BeamParams(1.0, ob.PMASS_EV, 275e9, ob.RE * ob.ME0 / ob.PMASS_EV, 0.6881e11)
    golden = 1.0254361754701657e+30
    # beams built as the reference builds them (the oracle's Beam.jl restatement), uploaded
    e = orc.beam_gaussian(2_560_000, seed=SEED, rng_id=1, **espec)
    p = orc.beam_gaussian(1_024_000, seed=SEED, rng_id=2, **pspec)
    rt = ob.StrongStrongRuntime()
    ctx = rt.context("ip", solver, 0)
    lum = ctx.collide(ob.Beam.from_numpy(e, ge), ob.Beam.from_numpy(p, gp), turn=1)
    stats = ctx.green_cache_stats()
    rt.close()
    assert abs(lum / golden - 1) <= 1e-12, lum
    assert stats == (0, 450, 0)
    # the same collide on beams built by the device generator (equal to the reference's up to the device's
    # libm ulps)
    rt = ob.StrongStrongRuntime()
    ctx = rt.context("ip", solver, 0)
    de = ob.Beam.gaussian(2_560_000, seed=SEED, rng_id=1, **espec, charge=-1.0, mc2=ob.EMASS_EV, E0=10e9,
                          npart=1.7203e11)
    dp = ob.Beam.gaussian(1_024_000, seed=SEED, rng_id=2, **pspec, charge=1.0, mc2=ob.PMASS_EV, E0=275e9,
                          npart=0.6881e11)
    lum_d = ctx.collide(de, dp, turn=1)
    rt.close()
    assert abs(lum_d / golden - 1) <= 1e-10, lum_d
