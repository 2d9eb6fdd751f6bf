"""Beam moment output fed from device reductions.

``MomentObserver`` mirrors the reference's moment observer (src/tasks/BeamObservers.jl:488-720, 830-838,
1000-1060, 1254-1271): the same moment selection (orders, ``extra``, ``exclude``), canonical column order
and names (``turn``, ``m100000``, ...), means for order 1 and central moments above.  Each observation is
one ``octo_beam_moments`` call that writes its row into a device record buffer without synchronising the
host; rows come back to the host in one copy when the buffer fills or is read, as the reference's row
buffer flushes to its run artifact at capacity.
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, List, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .solver import ArgumentError

Powers = Tuple[int, int, int, int, int, int]
COORDS = ("x", "px", "y", "py", "z", "pz")


def moment(*powers, **named) -> Powers:
    """Moment(x, px, y, py, z, pz) / Moment(; x=.., ...) / Moment("m110000") (BeamObservers.jl:488-520)."""
    if len(powers) == 1 and isinstance(powers[0], str):
        return parse_moment(powers[0])
    if len(powers) == 1 and isinstance(powers[0], tuple):
        powers = powers[0]
    if powers and named:
        raise ArgumentError("give moment powers positionally or by name, not both")
    if named:
        unknown = set(named) - set(COORDS)
        if unknown:
            raise ArgumentError(f"unknown coordinates {sorted(unknown)}")
        powers = tuple(int(named.get(c, 0)) for c in COORDS)
    if len(powers) != 6:
        raise ArgumentError("a moment has six powers")
    powers = tuple(int(p) for p in powers)
    if any(p < 0 for p in powers):
        raise ArgumentError("moment powers must be nonnegative integers")
    return powers


def parse_moment(text: str) -> Powers:
    """Moment(raw::AbstractString) (BeamObservers.jl:502-519): "m110000" or "m1_10_0_0_0_0"."""
    if not text.startswith("m"):
        raise ArgumentError(f"moment name must start with `m`: {text}")
    body = text[1:]
    if not body:
        raise ArgumentError(f"moment name has no powers: {text}")
    if "_" in body:
        parts = body.split("_")
        if len(parts) != 6:
            raise ArgumentError(f"separated moment name must contain six powers: {text}")
        return moment(*(int(p) for p in parts))
    if len(body) != 6:
        raise ArgumentError(f"compact moment name must contain six powers: {text}")
    return moment(*(int(ch) for ch in body))


def moment_name(powers: Powers) -> str:
    """name(moment) (BeamObservers.jl:545-551): compact when every power is one digit."""
    if all(0 <= p <= 9 for p in powers):
        return "m" + "".join(str(p) for p in powers)
    return "m" + "_".join(str(p) for p in powers)


def _order_key(powers: Powers):
    """isless of Moment (BeamObservers.jl:523-524): by order, then by descending powers."""
    return (sum(powers), tuple(-p for p in powers))


def _moments_for_order(order: int) -> List[Powers]:
    out: List[Powers] = []
    pw = [0] * 6

    def rec(remaining, dim):
        if dim == 5:
            pw[dim] = remaining
            out.append(tuple(pw))
            return
        for p in range(remaining, -1, -1):
            pw[dim] = p
            rec(remaining - p, dim + 1)
        pw[dim] = 0

    if order > 0:
        rec(order, 0)
    return out


def _flatten_orders(orders) -> List[int]:
    if isinstance(orders, int):
        return [orders]
    out = []
    for o in orders:
        out += _flatten_orders(o)
    return out


def _moment_list(items) -> List[Powers]:
    if items is None:
        return []
    if isinstance(items, str):
        return [parse_moment(items)]
    if isinstance(items, tuple) and len(items) == 6 and all(isinstance(p, int) for p in items):
        return [moment(items)]
    return [moment(i) if not isinstance(i, str) else parse_moment(i) for i in items]


def selected_moments(orders=(1, 2), extra=(), exclude=()) -> Tuple[Powers, ...]:
    """_selected_moments (BeamObservers.jl:619-628): every moment of the given orders, plus extra, minus
    exclude (exclude wins), order 0 dropped, sorted canonically."""
    ords = sorted(set(o for o in _flatten_orders(orders) if o > 0))
    ms: List[Powers] = []
    for o in ords:
        ms += _moments_for_order(o)
    ms += _moment_list(extra)
    excluded = set(_moment_list(exclude))
    seen, out = set(), []
    for m in ms:
        if m in seen:
            continue
        seen.add(m)
        if sum(m) > 0 and m not in excluded:
            out.append(m)
    return tuple(sorted(out, key=_order_key))


class MomentObserver:
    """MomentObserver(; name, orders=1:2, extra=(), exclude=()) (BeamObservers.jl:707-720) with a device record
    buffer of ``capacity`` rows.  ``observe(turn, beam)`` records one row on the device (no host sync);
    ``rows()`` returns every recorded row as a (records, 1 + moments) float64 array, column 0 the turn.
    ``mask_lost`` is allow_lost_particles(): reduce over the particles whose six coordinates are finite."""

    def __init__(self, name: str, orders=(1, 2), extra=(), exclude=(), capacity: int = 1024, mask_lost: bool = False,
                 device: int = 0):
        if not str(name):
            raise ArgumentError("the artifact-view MomentObserver needs a nonempty name")
        if capacity < 1:
            raise ArgumentError("capacity must be positive")
        self.name = str(name)
        self.moments = selected_moments(orders, extra, exclude)
        if len(self.moments) > _lib.MOMENTS_MAX:
            raise ArgumentError(f"a moment row holds at most {_lib.MOMENTS_MAX} moments")
        self.column_names = ["turn"] + [moment_name(m) for m in self.moments]
        self.capacity = int(capacity)
        self.mask_lost = bool(mask_lost)
        self.device = device
        self._powers = (C.c_int32 * max(6 * len(self.moments), 1))(*[p for m in self.moments for p in m])
        self._buffer = torch.full((self.capacity, len(self.column_names)), float("nan"), dtype=torch.float64,
                                  device=f"cuda:{device}")
        self._length = 0
        self._host: List[np.ndarray] = []
        self.record_count = 0

    def observe(self, turn: int, beam, stream=None) -> None:
        from .api import _scratch_ctx
        if self._length == self.capacity:
            self.flush()
        b = beam.to_c()
        st = (stream or torch.cuda.current_stream(beam.coords.device)).cuda_stream
        ctx = _scratch_ctx(beam.coords.device.index or 0)
        row = C.c_void_p(self._buffer[self._length].data_ptr())
        rc = _lib.lib().octo_beam_moments(ctx, C.byref(b), self._powers, len(self.moments), int(self.mask_lost),
                                          int(turn), row, C.c_void_p(st))
        if rc != _lib.OCTO_OK:
            raise ArgumentError(_lib.last_error(ctx))
        self._length += 1

    def flush(self) -> None:
        """_flush_moment_observer! (BeamObservers.jl:1000-1011): one device-to-host copy of the buffered rows."""
        if self._length == 0:
            return
        self._host.append(self._buffer[: self._length].cpu().numpy())
        self.record_count += self._length
        self._length = 0

    def rows(self) -> np.ndarray:
        self.flush()
        if not self._host:
            return np.zeros((0, len(self.column_names)))
        return np.concatenate(self._host, axis=0)

    def column(self, item) -> np.ndarray:
        key = item if item == "turn" else moment_name(moment(item) if not isinstance(item, str) else parse_moment(item))
        return self.rows()[:, self.column_names.index(key)]
