"""The allocation-free beam constructor, octo_beam_gaussian_noalloc, against octo_beam_gaussian.

octo_beam_gaussian_noalloc serves callers that cannot call cudaMalloc -- hosts whose device memory
belongs to a pool allocator (CUDA.jl, PyTorch) and services that forbid allocation after start-up.
Its reduction scratch is a fixed static device array in the library, so it needs no context.  This
test drives both entry points through the C ABI on the same seeds and checks the coordinates agree
within the parity tolerance (atol = rtol = 1e-10) on two calls in a row, and with the oracle's restatement
of the reference's generator; and that a beam larger than the fixed scratch allows is rejected.  The file name sorts last so a stop-at-first-failure run has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ATOL = RTOL = 1e-10


def _beam_struct(ob, coords):
    return ob.Beam(coords, ob.BeamParams()).to_c()


def _noalloc(ob, n, rng_id, beta, sigma, stream):
    import torch
    from octo_b200 import _lib
    coords = torch.empty((6, n), dtype=torch.float64, device="cuda:0")
    b = _beam_struct(ob, coords)
    d3 = C.c_double * 3
    err = C.create_string_buffer(256)
    rc = _lib.lib().octo_beam_gaussian_noalloc(0, C.byref(b), 123456789, rng_id, d3(*beta), d3(0.0, 0.0, 0.0),
                                               d3(*sigma), 5.0, C.c_void_p(stream), err, len(err))
    assert rc == _lib.OCTO_OK, err.value
    return coords


def test_noalloc_beam_matches_context_beam_on_two_calls():
    import torch
    import octo_b200 as ob
    from oracle import oracle as orc
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(100_000, 1, (0.55, 0.056, 12.727272727272727), (95e-6, 8.5e-6, 7e-3)),
             (70_001, 2, (0.8, 0.072, 90.9090909090909), (95e-6, 8.5e-6, 6e-2))]
    for n, rng_id, beta, sigma in cases:
        device_before = torch.cuda.current_device()
        got = _noalloc(ob, n, rng_id, beta, sigma, stream)
        assert torch.cuda.current_device() == device_before  # the caller's current device is left as it was
        ref = ob.Beam.gaussian(n, beta=beta, sigma=sigma, rng_id=rng_id, seed=123456789)
        torch.cuda.synchronize()
        a, b = got.cpu().numpy(), ref.coords.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert np.all(np.abs(a - b) <= ATOL + RTOL * np.abs(b)), float(np.abs(a - b).max())
        # and against the oracle's restatement of Beam.jl's generator (device libm ulps and sum order apart)
        want = orc.beam_gaussian(n, seed=123456789, rng_id=rng_id, beta=beta, sigma=sigma)
        scale = np.sqrt(np.mean(want ** 2, axis=1, keepdims=True))
        assert float((np.abs(a - want) / (scale + np.abs(want))).max()) < 1e-14


def test_noalloc_rejects_beams_beyond_its_scratch():
    import torch
    from octo_b200 import _lib
    n = (8192 * 4094) + 1
    # a real allocation of the full size, so the rejection is the size check's and never a stray launch
    coords = torch.zeros((6, n), dtype=torch.float64, device="cuda:0")
    b = _lib.OctoBeam()
    b.n = n
    for k, name in enumerate(("x", "px", "y", "py", "z", "pz")):
        setattr(b, name, C.c_void_p(coords[k].data_ptr()))
    d3 = C.c_double * 3
    err = C.create_string_buffer(256)
    rc = _lib.lib().octo_beam_gaussian_noalloc(0, C.byref(b), 1, 1, d3(1, 1, 1), d3(0, 0, 0), d3(1, 1, 1), 5.0,
                                               None, err, len(err))
    assert rc == _lib.OCTO_ERR_ARG
    assert b"scratch limit" in err.value
    torch.cuda.synchronize()
    assert not torch.any(coords)  # nothing was written
    del coords
    torch.cuda.empty_cache()
