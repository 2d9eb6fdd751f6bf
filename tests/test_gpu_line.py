"""Line tracking on the GPU (octo_track_line through the C ABI) against the oracle.

Tolerance: the element arithmetic is the same FP64 sequence on both sides (the library is built without
fused multiply-add); they differ only in the device's sin / cos / log, within a few ulp.  Every
coordinate must agree to 1e-13 of its component's RMS over the beam, far inside the reference's
backend-consistency contract for these elements (atol = rtol = 1e-10, runtests.jl:7405-7415), and the
radiation case of runtests.jl:450-486 to its 1e-16 absolute bar."""
import ctypes as C
import math

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from helpers import beams

pytestmark = pytest.mark.gpu

RTOL_RMS = 1e-13


def gpu_track(elems, coords, turn=0, turns=1, seed=0, rng_method="philox", dtype=torch.float64):
    import octo_b200 as ob
    beam = ob.Beam.from_numpy(coords, ob.BeamParams(1.0, 1.0, 1.0, 1.0, 1.0), dtype=dtype)
    ob.track(beam, elems, turns, ob.TrackingContext(turn=turn, seed=seed, rng_method=rng_method))
    torch.cuda.synchronize()
    return beam.numpy().astype(np.float64)


def oracle_track(elems, coords, turn=0, turns=1, seed=0, rng_method=1):
    from octo_b200 import line as ln
    return orc.track_line([e.to_c() for e in ln.flatten(elems)], coords, turn=turn, turns=turns, seed=seed,
                          rng_method=rng_method)


def assert_close(got, want, rtol=RTOL_RMS):
    scale = np.sqrt(np.mean(want ** 2, axis=1))
    err = np.max(np.abs(got - want), axis=1)
    assert np.all(err <= rtol * scale), (err / scale)


def all_elements():
    from octo_b200 import line as ln
    return [
        ln.Linear6DSpec(beta1=(0.55, 0.056, 12.7), beta2=(150.0, 30.0, 12.7), alpha1=(0.1, -0.2, 0.0),
                        dmu=(math.pi / 2, 0.3, 0.01), zeta1=(0.01, -0.02, 0.0, 0.03), eta1=(0.1, 0.02, -0.01, 0.0),
                        R1=(0.02, 0.01, -0.01, 0.03)),
        ln.ThinCrabCavitySpec(197e6, N=3, strengthX=(0.01, -0.003, 0.001), strengthY=(0.002, 0.0, 0.001),
                              phase=(0.1, 0.0, -0.2)),
        ln.LorentzBoostSpec(12.5e-3),
        ln.RevLorentzBoostSpec(-7.0e-3),
        ln.ChromaticityKickSpec(xi=(2.0, 1.5), beta=(0.8, 0.07, 90.0), alpha=(0.3, -0.2, 0.0),
                                zeta=(0.01, -0.02, 0.03, -0.04), eta=(0.05, -0.06, 0.07, -0.08),
                                R=(0.01, 0.02, -0.015, 0.005)),
        ln.LumpedRadSpec(damping_turns=(4000.0, 4000.0, 2000.0), beta=(0.55, 0.056, 12.7),
                         alpha=(0.1, -0.2, 0.0), sigma=(106e-6, 9.5e-6, 0.7e-2), zeta=(0.01, -0.02, 0.03, -0.04),
                         eta=(0.05, -0.06, 0.07, -0.08), R=(0.01, 0.02, -0.015, 0.005), rng_id=103),
        ln.CrabDispersionSpec(0.01, -0.02, 0.03, -0.04),
        ln.MomentumDispersionSpec(0.05, -0.06, 0.07, -0.08),
        ln.XYCouplingSpec(0.01, 0.02, -0.015, 0.005, mode="A"),
        ln.XYCouplingSpec(0.01, 0.02, -0.015, 0.005, mode="B"),
        ln.XYCouplingSpec(0.3, 0.2, 0.1, 0.4, mode="undef"),
    ]


@pytest.mark.parametrize("k", range(11))
def test_each_element_matches_oracle(k):
    e, _ = beams(50_000, 16)
    elem = all_elements()[k]
    got = gpu_track([elem], e, turn=5, turns=2, seed=0x12345678)
    assert_close(got, oracle_track([elem], e, turn=5, turns=2, seed=0x12345678))


@pytest.mark.parametrize("method", ["philox", "splitmix"])
@pytest.mark.parametrize("beam", ["electron", "proton"])
def test_example_line_matches_oracle(beam, method):
    """Both segments of the strong-strong example's ring (examples/strong_strong_tracking.jl:206-262):
    11 (electron) / 10 (proton) elements, more than one launch program, so the turns run one by one."""
    from octo_b200 import line as ln
    e, p = beams(200_000, 100_000)
    coords = e if beam == "electron" else p
    segs = ln.eic_like_segments(beam)
    code = 1 if method == "philox" else 2
    got = gpu_track(segs, coords, turn=3, turns=3, seed=123456789, rng_method=method)
    assert_close(got, oracle_track(segs, coords, turn=3, turns=3, seed=123456789, rng_method=code))


def test_segments_one_launch_each_match_oracle():
    """Each segment fits one launch program: all turns run inside the kernel."""
    from octo_b200 import line as ln
    e, _ = beams(100_000, 16)
    before, after = ln.eic_like_segments("electron")
    for seg in (before, after):
        got = gpu_track(seg, e, turn=0, turns=4, seed=99)
        assert_close(got, oracle_track(seg, e, turn=0, turns=4, seed=99))


def test_radiation_matches_host_reference_case():
    """runtests.jl:450-486: seed 777 Philox, 4096 particles of s(scale, phase) = scale sin(0.7 i + phase),
    3 turns from turn 0; GPU and host agree to 1e-16 absolute, and two runs are bitwise equal."""
    from octo_b200 import line as ln
    spec = ln.LumpedRadSpec(damping_turns=(20.0, 25.0, 30.0), beta=(0.7, 0.9, 1.1), alpha=(0.2, -0.1, 0.05),
                            sigma=(1.2e-3, 0.8e-3, 2.0e-3), rng_id=0x1234)
    i = np.arange(1, 4097)
    s = lambda scale, phase: scale * np.sin(0.7 * i + phase)
    rep = np.stack([s(1e-4, 0.0), s(1e-5, 0.3), s(1e-4, 0.9), s(1e-5, 1.2), s(1e-3, 2.1), s(1e-4, 2.5)])
    g1 = gpu_track([spec], rep, turn=0, turns=3, seed=777)
    g2 = gpu_track([spec], rep, turn=0, turns=3, seed=777)
    assert np.array_equal(g1, g2)
    ref = oracle_track([spec], rep, turn=0, turns=3, seed=777)
    assert np.max(np.abs(g1 - ref)) <= 1e-16


def test_chunked_equals_continuous_on_gpu():
    from octo_b200 import line as ln
    e, _ = beams(100_000, 16)
    before, after = ln.eic_like_segments("electron")
    for seg in (after, (before, after)):
        cont = gpu_track(seg, e, turn=0, turns=7, seed=0x5EED)
        part = gpu_track(seg, e, turn=0, turns=3, seed=0x5EED)
        part = gpu_track(seg, part, turn=3, turns=4, seed=0x5EED)
        assert np.array_equal(cont, part)


def test_float32_beam():
    """FP32 coordinates are widened on load, tracked in FP64 and rounded once on store."""
    from octo_b200 import line as ln
    e, _ = beams(100_000, 16)
    e32 = e.astype(np.float32).astype(np.float64)
    seg = ln.eic_like_segments("electron")[1]
    got = gpu_track(seg, e32, turns=2, seed=5, dtype=torch.float32)
    want = oracle_track(seg, e32, turns=2, seed=5).astype(np.float32).astype(np.float64)
    # both sides round an FP64 result to FP32 once: at most one FP32 ulp apart where the FP64 values straddle
    # a rounding boundary
    scale = np.sqrt(np.mean(want ** 2, axis=1, keepdims=True))
    assert np.all(np.abs(got - want) <= 1.2e-7 * np.abs(want) + 1e-13 * scale)


def test_abi_errors_and_empty_beam():
    import octo_b200 as ob
    from octo_b200 import _lib
    from octo_b200.api import _scratch_ctx
    from octo_b200 import line as ln
    ctx = _scratch_ctx(0)
    L = _lib.lib()
    coords = torch.zeros((6, 10), dtype=torch.float64, device="cuda:0")
    b = ob.Beam(coords, ob.BeamParams(1.0, 1.0, 1.0, 1.0, 1.0)).to_c()
    arr = (_lib.OctoElement * 1)()
    arr[0] = ln.ThinCrabCavitySpec(1e8, N=1, strengthX=(0.1,)).to_c()
    arr[0].p[0] = 0.0  # frequency 0: rejected as the constructor does
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.octo_track_line(ctx, C.byref(b), arr, 1, 0, 1, 0, 1, st) == _lib.OCTO_ERR_ARG
    assert "frequency" in _lib.last_error(ctx)
    arr[0] = ln.LorentzBoostSpec(0.01).to_c()
    assert L.octo_track_line(ctx, C.byref(b), arr, 1, 0, 1, 0, 3, st) == _lib.OCTO_ERR_ARG  # RNG method 3
    assert L.octo_track_line(ctx, C.byref(b), arr, 1, -1, 1, 0, 1, st) == _lib.OCTO_ERR_ARG  # negative turn
    arr[0].kind = 42
    assert L.octo_track_line(ctx, C.byref(b), arr, 1, 0, 1, 0, 1, st) == _lib.OCTO_ERR_ARG
    arr[0] = ln.Linear6DSpec(matrix=np.eye(6)).to_c()
    arr[0].p[2] = 0.3  # not symplectic
    assert L.octo_track_line(ctx, C.byref(b), arr, 1, 0, 1, 0, 1, st) == _lib.OCTO_ERR_ARG
    empty = ob.Beam(torch.zeros((6, 0), dtype=torch.float64, device="cuda:0"), ob.BeamParams(1, 1, 1, 1, 1))
    ob.track(empty, [ln.LorentzBoostSpec(0.01)], 3)
    with pytest.raises(ob.ArgumentError):
        ob.track(empty, [ln.LorentzBoostSpec(0.01)], 1, ob.TrackingContext(turn=-1))


def test_nonfinite_particles_spread_as_oracle():
    """Dropped zero harmonics and skipped all-zero frame transforms are exact shortcuts: particles with a
    NaN or Inf coordinate take the full arithmetic, so the non-finite pattern equals the oracle's."""
    from octo_b200 import line as ln
    e, _ = beams(4096, 16)
    bad = e.copy()
    rng = np.random.default_rng(7)
    for k in range(6):
        idx = rng.choice(4096, 40, replace=False)
        bad[k, idx[:20]] = np.nan
        bad[k, idx[20:30]] = np.inf
        bad[k, idx[30:]] = -np.inf
    before, after = ln.eic_like_segments("electron")
    np.seterr(invalid="ignore")
    for seg in (before, after, [after[2]], [after[5]], [after[6]]):
        got = gpu_track(seg, bad, turn=2, turns=2, seed=11)
        want = oracle_track(seg, bad, turn=2, turns=2, seed=11)
        assert np.array_equal(np.isnan(got), np.isnan(want))
        assert np.array_equal(np.isposinf(got), np.isposinf(want))
        fin = np.isfinite(want)
        scale = np.sqrt(np.mean(np.where(fin, want, 0.0) ** 2, axis=1, keepdims=True))
        assert np.all(np.abs(np.where(fin, got - want, 0.0)) <= RTOL_RMS * scale)
