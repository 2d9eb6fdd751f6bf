"""Moment rows on the device (octo_beam_moments through MomentObserver) against the oracle's restatement of
the reference's moment row (src/tasks/BeamObservers.jl:1013-1040, 1254-1271).  Tolerance: each moment to
1e-12 of its natural scale prod_d sigma_d^p_d (the two sides sum in different orders)."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from helpers import beams

pytestmark = pytest.mark.gpu


def observe(coords, turn=0, dtype=torch.float64, **kw):
    import octo_b200 as ob
    beam = ob.Beam.from_numpy(coords, ob.BeamParams(1.0, 1.0, 1.0, 1.0, 1.0), dtype=dtype)
    obs = ob.MomentObserver("ip", **kw)
    obs.observe(turn, beam)
    return obs, obs.rows()[0]


def assert_row(got, coords, moments, turn, mask_lost=False):
    want = orc.moment_row(coords, moments, turn, mask_lost)
    assert got[0] == want[0]
    b = coords[:, np.all(np.isfinite(coords), axis=0)] if mask_lost else coords
    sig = b.std(axis=1)
    for k, m in enumerate(moments):
        scale = np.prod([sig[d] ** m[d] for d in range(6)])
        assert abs(got[1 + k] - want[1 + k]) <= 1e-12 * scale, (m, got[1 + k], want[1 + k])


@pytest.mark.parametrize("kw", [dict(), dict(orders=(1, 2, 3), extra="m000004"),
                                dict(orders=2, extra=["m100000", "m000001"], exclude=["m200000", "m000011"])])
def test_rows_match_oracle(kw):
    e, _ = beams(300_000, 16)
    obs, row = observe(e, turn=7, **kw)
    assert len(row) == 1 + len(obs.moments)
    assert_row(row, e, obs.moments, 7)


def test_lost_particles():
    e, _ = beams(100_000, 16)
    bad = e.copy()
    bad[1, 5] = np.nan
    bad[4, 77] = np.inf
    bad[0, 99_999] = -np.inf
    obs, row = observe(bad, turn=3, mask_lost=True)
    assert_row(row, bad, obs.moments, 3, mask_lost=True)
    obs, row = observe(bad, turn=3)
    want = orc.moment_row(bad, obs.moments, 3)
    assert row[0] == 3
    np.testing.assert_array_equal(np.isnan(row), np.isnan(want))
    assert np.isnan(row[1:]).any()
    dead = np.full((6, 1000), np.nan)
    obs, row = observe(dead, turn=9, mask_lost=True)
    assert row[0] == 9 and np.all(np.isnan(row[1:]))


def test_float32_beam():
    e, _ = beams(100_000, 16)
    e32 = e.astype(np.float32).astype(np.float64)
    obs, row = observe(e32, turn=1, dtype=torch.float32)
    assert_row(row, e32, obs.moments, 1)


def test_buffer_flush_and_tracking_turns():
    """Rows recorded across a capacity flush, with line tracking between observations, equal the oracle's
    rows of the same turns."""
    import octo_b200 as ob
    from octo_b200 import line as ln
    e, _ = beams(50_000, 16)
    beam = ob.Beam.from_numpy(e, ob.BeamParams(1.0, 1.0, 1.0, 1.0, 1.0))
    obs = ob.MomentObserver("electron", capacity=3)
    seg = ln.eic_like_segments("electron")[1]
    host = e.copy()
    wants = []
    for t in range(7):
        ob.track(beam, seg, 1, ob.TrackingContext(turn=t, seed=5))
        host = beam.numpy()
        obs.observe(t, beam)
        wants.append(host)
    rows = obs.rows()
    assert rows.shape == (7, 28) and obs.record_count == 7
    for t in range(7):
        assert_row(rows[t], wants[t], obs.moments, t)
    np.testing.assert_array_equal(obs.column("turn"), np.arange(7))


def test_abi_errors():
    import octo_b200 as ob
    from octo_b200 import _lib
    from octo_b200.api import _scratch_ctx
    ctx = _scratch_ctx(0)
    coords = torch.zeros((6, 10), dtype=torch.float64, device="cuda:0")
    b = ob.Beam(coords, ob.BeamParams(1.0, 1.0, 1.0, 1.0, 1.0)).to_c()
    row = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = _lib.lib()
    for powers in ([0] * 6, [33, 0, 0, 0, 0, 0], [1, 0, 0, 0, 0, 0] * 2, [-1, 2, 0, 0, 0, 0]):
        arr = (C.c_int32 * len(powers))(*powers)
        assert L.octo_beam_moments(ctx, C.byref(b), arr, len(powers) // 6, 0, 0,
                                   C.c_void_p(row.data_ptr()), st) == _lib.OCTO_ERR_ARG
