"""``collide`` -- the drop-in for Octopus.jl's ``collide!(::PICPoissonSolver, beam1, beam2, backend[, ctx])``
(interface.jl:13-74, 508-509), running on libocto_b200.

The bare call builds a fresh context (cold Green cache) per call, as the reference's public
``collide!`` does (pic_cpu.jl:1-21).  Passing a ``StrongStrongRuntime`` keeps the context and
its slice-pair Green cache across calls, as ``task.runtime_cache`` does on the task path
(pic_cpu.jl:23-32, 499-515).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from . import _lib
from . import line as _line
from .beam import Beam
from .solver import ArgumentError, LongitudinalSlicing, PICPoissonSolver


class CUDABackend:
    """Backend tag (src/Octopus.jl:10-25)."""


class CollisionError(ArgumentError):
    """Raised for a failed collide; ``code`` is the OCTO_* status, ``report`` the collide report."""

    def __init__(self, code: int, message: str, report=None):
        super().__init__(message)
        self.code = code
        self.report = report


@dataclass
class TrackingContext:
    """TrackingContext (src/track/Track.jl:3-22): the turn (collision messages and schedules; the turn of
    the counter-RNG draws of line tracking) and the seed and method of the global counter RNG, taken when
    the context is made.  turn = -1 marks a collide outside a turn loop."""
    turn: int = -1
    seed: int = field(default_factory=_line.global_rng_seed)
    rng_method: str = field(default_factory=_line.global_rng_method)


def with_turn(ctx: TrackingContext, turn: int) -> TrackingContext:
    """with_turn (src/track/Track.jl:24-32)."""
    return TrackingContext(turn=int(turn), seed=ctx.seed, rng_method=ctx.rng_method)


class Context:
    """One libocto_b200 context: device workspaces plus the slice-pair Green cache."""

    def __init__(self, solver: PICPoissonSolver, device: int = 0, dtype: torch.dtype = torch.float64):
        """dtype is the beams' element type: float64 runs the plain form, float32 the precision form
        (FP32 particles, field planes and FFTs; FP64 Green function, statistics and luminosity)."""
        if dtype not in (torch.float64, torch.float32):
            raise ArgumentError("beam element type must be Float64 or Float32")
        self.solver = solver
        self.device = device
        self.dtype = dtype
        self._opts = solver.to_c()
        self._opts.precision = 1 if dtype == torch.float32 else 0
        self._ptr = _lib.lib().octo_create(int(device), C.byref(self._opts))
        if not self._ptr:
            raise RuntimeError("octo_create failed")
        self.last_report = None

    def close(self):
        if getattr(self, "_ptr", None):
            _lib.lib().octo_destroy(self._ptr)
            self._ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ptr(self):
        return self._ptr

    def collide(self, beam1: Beam, beam2: Beam, turn: int = -1, compute_luminosity: bool = True,
                stream: Optional[torch.cuda.Stream] = None) -> float:
        b1, b2 = beam1.to_c(), beam2.to_c()
        p1, p2 = beam1.params.to_c(), beam2.params.to_c()
        lum = C.c_double(float("nan"))
        rep = _lib.OctoCollideReport()
        st = (stream or torch.cuda.current_stream(beam1.coords.device)).cuda_stream
        rc = _lib.lib().octo_pic_collide(self._ptr, C.byref(b1), C.byref(b2), C.byref(p1), C.byref(p2), int(turn),
                                         int(bool(compute_luminosity)), C.byref(lum), C.byref(rep), C.c_void_p(st))
        self.last_report = rep
        if rc != _lib.OCTO_OK:
            raise CollisionError(rc, f"{_lib.ERROR_NAMES.get(rc, rc)}: {_lib.last_error(self._ptr)}", rep)
        return lum.value

    AUTOTUNE_SHAPES = ((1, 1), (2, 1), (1, 2), (2, 2))  # (deposit waves, kick block-slot multiple)

    def autotune(self, beam1: Beam, beam2: Beam, rounds: int = 2,
                 stream: Optional[torch.cuda.Stream] = None) -> int:
        """Pick this context's launch shape by timing collides of copies of beam1 and beam2 (the beams
        themselves are untouched); later collides give the same results in any shape, only faster.
        Returns the chosen shape's index into AUTOTUNE_SHAPES."""
        c1 = Beam(beam1.coords.clone(), beam1.params)
        c2 = Beam(beam2.coords.clone(), beam2.params)
        b1, b2 = c1.to_c(), c2.to_c()
        p1, p2 = c1.params.to_c(), c2.params.to_c()
        choice = C.c_int32(-1)
        st = (stream or torch.cuda.current_stream(beam1.coords.device)).cuda_stream
        rc = _lib.lib().octo_pic_autotune(self._ptr, C.byref(b1), C.byref(b2), C.byref(p1), C.byref(p2), int(rounds),
                                          C.byref(choice), C.c_void_p(st))
        if rc != _lib.OCTO_OK:
            raise CollisionError(rc, f"{_lib.ERROR_NAMES.get(rc, rc)}: {_lib.last_error(self._ptr)}", None)
        return choice.value

    def set_particle_order(self, spatial: bool = True):
        """Plain PIC: keep each slice's particles grouped by transverse position (default) or in caller order;
        results are bit-identical either way, only the speed differs."""
        rc = _lib.lib().octo_set_particle_order(self._ptr, 1 if spatial else 0)
        if rc != _lib.OCTO_OK:
            raise CollisionError(rc, "octo_set_particle_order failed")

    def set_collide_graph(self, enable: bool = True):
        """Plain PIC: replay each collide as a captured CUDA graph once its schedule repeats (default), or always
        run the ordinary host-scheduled path; results are bit-identical either way."""
        rc = _lib.lib().octo_set_collide_graph(self._ptr, 1 if enable else 0)
        if rc != _lib.OCTO_OK:
            raise CollisionError(rc, f"octo_set_collide_graph failed: {_lib.last_error(self._ptr)}")

    def collide_graph_stats(self) -> Tuple[int, int, int, int]:
        """(graphs captured, collides replayed, replays the device guard declined, capture failures)."""
        out = (C.c_int64 * 4)()
        _lib.lib().octo_collide_graph_stats(self._ptr, out)
        return tuple(out)

    def green_cache_stats(self) -> Tuple[int, int, int]:
        h, m, r = C.c_int64(), C.c_int64(), C.c_int64()
        _lib.lib().octo_green_cache_stats(self._ptr, C.byref(h), C.byref(m), C.byref(r))
        return h.value, m.value, r.value

    def capture_charge_plane(self, pair_i: int, pair_j: int, direction: int, plane: int = 0):
        """Arm a copy of one field-solve charge grid of the next collide (a test hook): slice pair (i, j),
        direction 1 or 2, plane 0 (sL), 1 (sR) or 2 (the midpoint / :node Z plane)."""
        rc = _lib.lib().octo_capture_charge_plane(self._ptr, int(pair_i), int(pair_j), int(direction), int(plane))
        if rc != _lib.OCTO_OK:
            raise CollisionError(rc, _lib.last_error(self._ptr))

    def captured_charge_plane(self, with_field_mesh: bool = False):
        """The captured int64 grid as an (ny, nx) array (row iy-1 holds nodes (1..nx, iy)), the mesh
        (x0, y0, width, height) and the fixed-point bits; with_field_mesh: also the interaction's field mesh."""
        nx, ny = self.solver.grid
        q = np.zeros(nx * ny, dtype=np.int64)
        mesh = (C.c_double * 4)()
        fmesh = (C.c_double * 4)()
        bits = C.c_int32()
        rc = _lib.lib().octo_captured_charge_plane(self._ptr, q.ctypes.data_as(C.POINTER(C.c_int64)), mesh, fmesh,
                                                   C.byref(bits))
        if rc != _lib.OCTO_OK:
            raise CollisionError(rc, _lib.last_error(self._ptr))
        if with_field_mesh:
            return q.reshape(ny, nx), tuple(mesh), tuple(fmesh), bits.value
        return q.reshape(ny, nx), tuple(mesh), bits.value

    def set_timing(self, enable: bool = True, phases=None):
        """Per-phase device timing (the reference's pic_timing diagnostics); enabling clears it.  phases: the
        names of the phases to time (default all); each timed launch group records two CUDA events."""
        mask = 0xFFFFFFFF if phases is None else sum(1 << _lib.PHASES.index(p) for p in phases)
        _lib.lib().octo_set_timing_phases(self._ptr, mask)
        _lib.lib().octo_set_timing(self._ptr, int(bool(enable)))

    def timing_report(self):
        """{phase: (device ms, launches, algorithmic bytes)} accumulated since set_timing(True)."""
        n = len(_lib.PHASES)
        ms = (C.c_double * n)(); la = (C.c_int64 * n)(); by = (C.c_double * n)()
        _lib.lib().octo_timing_report(self._ptr, ms, la, by)
        return {name: (ms[k], la[k], by[k]) for k, name in enumerate(_lib.PHASES)}

    def pair_luminosity_trace(self):
        cap = 1 << 14
        pi = (C.c_int32 * cap)(); pj = (C.c_int32 * cap)(); lum = (C.c_double * cap)()
        n = _lib.lib().octo_pair_luminosity_trace(self._ptr, pi, pj, lum, cap)
        return [(pi[k], pj[k], lum[k]) for k in range(min(n, cap))]


class StrongStrongRuntime:
    """Twin of task.runtime_cache: one persistent context per (label, solver, element type), the key
    of pic_cpu.jl:499-515."""

    def __init__(self):
        self._ctx: Dict[tuple, Context] = {}

    def context(self, label: str, solver: PICPoissonSolver, device: int, dtype: torch.dtype = torch.float64) -> Context:
        key = (label, solver, device, dtype)
        ctx = self._ctx.get(key)
        if ctx is None:
            ctx = Context(solver, device, dtype)
            self._ctx[key] = ctx
        return ctx

    def close(self):
        for c in self._ctx.values():
            c.close()
        self._ctx.clear()


def compute_luminosity(solver: PICPoissonSolver, ctx: Optional[TrackingContext]) -> bool:
    """_pic_compute_luminosity (interface.jl:2596-2630): every turn unless a schedule says otherwise."""
    sched = solver.luminosity_schedule
    if ctx is None or sched is None:
        return True
    return bool(sched(ctx.turn)) if callable(sched) else True


def collide(solver: PICPoissonSolver, beam1: Beam, beam2: Beam, backend=CUDABackend,
            ctx: Optional[TrackingContext] = None, runtime: Optional[StrongStrongRuntime] = None,
            label: str = "ip") -> float:
    """collide!(solver, beam1, beam2, backend[, ctx]) -> luminosity (Float64; NaN when not scheduled).

    Kicks both beams in place.  Raises ``CollisionError`` (an ``ArgumentError``) with the reference's
    non-finite / extent / unsupported-option messages."""
    if backend is not CUDABackend:
        raise ArgumentError("this backend implements collide! for CUDABackend beams only")
    if beam1.coords.device != beam2.coords.device:
        raise ArgumentError("both beams must be on the same device (interface.jl:2461-2464)")
    if beam1.dtype != beam2.dtype:
        raise ArgumentError("both beams must have the same element type")
    device = beam1.coords.device.index or 0
    turn = -1 if ctx is None else int(ctx.turn)
    lum_on = compute_luminosity(solver, ctx)
    if runtime is None:
        c = Context(solver, device, beam1.dtype)
        try:
            return c.collide(beam1, beam2, turn=turn, compute_luminosity=lum_on)
        finally:
            c.close()
    return runtime.context(label, solver, device, beam1.dtype).collide(beam1, beam2, turn=turn,
                                                                       compute_luminosity=lum_on)


def collide_batch(contexts, beams1, beams2, turn: int = -1, compute_luminosity: bool = True, streams=None):
    """Independent collides, one per context, overlapped on their own streams (octo_pic_collide_batch):
    the parameter-scan and multi-collision-point form of collide!.  Returns the luminosities; raises
    CollisionError for the first failing collide after all of them have run."""
    n = len(contexts)
    if not (len(beams1) == len(beams2) == n):
        raise ArgumentError("collide_batch needs one beam pair per context")
    if streams is None:
        streams = [torch.cuda.Stream(device=b.coords.device) for b in beams1]
    cb1 = [b.to_c() for b in beams1]
    cb2 = [b.to_c() for b in beams2]
    cp1 = [b.params.to_c() for b in beams1]
    cp2 = [b.params.to_c() for b in beams2]
    P = C.POINTER
    arr = lambda T, items: (T * max(n, 1))(*items)
    ctxs = arr(C.c_void_p, [c.ptr for c in contexts])
    a1 = arr(P(_lib.OctoBeam), [C.pointer(b) for b in cb1])
    a2 = arr(P(_lib.OctoBeam), [C.pointer(b) for b in cb2])
    q1 = arr(P(_lib.OctoBeamParams), [C.pointer(p) for p in cp1])
    q2 = arr(P(_lib.OctoBeamParams), [C.pointer(p) for p in cp2])
    lum = (C.c_double * max(n, 1))()
    reps = (_lib.OctoCollideReport * max(n, 1))()
    status = (C.c_int32 * max(n, 1))()
    sts = arr(C.c_void_p, [s.cuda_stream for s in streams])
    # the caller's current stream work on the beams precedes the batch's streams
    for s, b in zip(streams, beams1):
        s.wait_stream(torch.cuda.current_stream(b.coords.device))
    rc = _lib.lib().octo_pic_collide_batch(n, ctxs, a1, a2, q1, q2, int(turn), int(bool(compute_luminosity)), lum, reps,
                                           status, sts)
    for c, r in zip(contexts, reps):
        c.last_report = r
    for b, s in zip(beams1, streams):
        torch.cuda.current_stream(b.coords.device).wait_stream(s)
    if rc != _lib.OCTO_OK:
        k = next(i for i in range(n) if status[i] != _lib.OCTO_OK)
        raise CollisionError(rc, f"collide {k}: {_lib.ERROR_NAMES.get(rc, rc)}: {_lib.last_error(contexts[k].ptr)}",
                             reps[k])
    return [lum[k] for k in range(n)]


_scratch: Dict[int, int] = {}


def _scratch_ctx(device: int):
    """A small context used for beam construction and one-turn maps."""
    if device not in _scratch:
        s = PICPoissonSolver(grid=(8, 8), slicing=LongitudinalSlicing(nslices=1, method="normal_quantile"))
        c = Context(s, device)
        _scratch[device] = c
    return _scratch[device].ptr


class Linear6D:
    """Linear 6D one-turn map (linear6d.jl:85-123, 233-280) for an uncoupled lattice without dispersion:
    per-plane rotation by 2*pi*tune with equal Twiss parameters at both ends."""

    def __init__(self, beta, alpha, tune):
        m = np.zeros(36)
        for i in range(3):
            mu = 2.0 * math.pi * tune[i]
            s, c = math.sin(mu), math.cos(mu)
            b1 = b2 = float(beta[i]); a1 = a2 = float(alpha[i])
            r = 2 * i
            m[r * 6 + r] = math.sqrt(b2 / b1) * (c + a1 * s)
            m[r * 6 + r + 1] = math.sqrt(b2 * b1) * s
            m[(r + 1) * 6 + r] = (-(1.0 + a1 * a2) * s + (a1 - a2) * c) / math.sqrt(b1 * b2)
            m[(r + 1) * 6 + r + 1] = math.sqrt(b1 / b2) * (c - a2 * s)
        self.matrix = m

    def track(self, beam: Beam, turns: int = 1, stream=None):
        b = beam.to_c()
        m = (C.c_double * 36)(*self.matrix.tolist())
        st = (stream or torch.cuda.current_stream(beam.coords.device)).cuda_stream
        ctx = _scratch_ctx(beam.coords.device.index or 0)
        rc = _lib.lib().octo_linear6d(ctx, C.byref(b), m, int(turns), C.c_void_p(st))
        if rc != _lib.OCTO_OK:
            raise RuntimeError(_lib.last_error(ctx))
        return beam


def track(beam: Beam, elems, turns: int = 1, context: Optional[TrackingContext] = None, stream=None) -> Beam:
    """track!(rep, elems, turns; context) (src/track/phase6d_track.jl:10-35, 197-212) for a line of zero-length
    element specs (octo_b200.line), nested tuples expanded as fusedTrack does: one fused device pass applies
    every element to every particle, `turns` times.  Turn t of the call draws the radiation noise of
    context turn ``context.turn + t`` for particle i as id i + 1, so chunked runs equal one run bit for bit.
    The default context is TrackingContext(turn=0) with the global seed and method."""
    ctx = context if context is not None else TrackingContext(turn=0)
    if ctx.turn < 0:
        raise ArgumentError("line tracking needs a context turn >= 0")
    if int(turns) < 0:
        raise ArgumentError("turns must be non-negative")
    arr, n = _line.compile_line(elems)
    b = beam.to_c()
    st = (stream or torch.cuda.current_stream(beam.coords.device)).cuda_stream
    cptr = _scratch_ctx(beam.coords.device.index or 0)
    rc = _lib.lib().octo_track_line(cptr, C.byref(b), arr, n, int(ctx.turn), int(turns), int(ctx.seed),
                                    _line.rng_method_code(ctx.rng_method), C.c_void_p(st))
    if rc != _lib.OCTO_OK:
        raise ArgumentError(_lib.last_error(cptr))
    return beam
