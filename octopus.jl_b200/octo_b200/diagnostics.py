"""Field accuracy of the collide path against the exact Bassetti-Erskine field.

The measurement follows the reference's solver review (81 x 81 probe points over +-4 sigma, RMS error
normalised by the largest exact field, no fitted constant): a deterministic Gaussian quantile lattice
is the source slice, an 81 x 81 lattice of probe particles with zero momenta is the field slice, and
one ``collide`` with kbb = 1 kicks every probe by 2 E(x, y), E being the field of a unit-charge
Gaussian in the units of the PIC Green function (E -> r/|r|^2 far away).  The probes therefore read
the field through the same deposition, convolution, derivative and interpolation as production
collides, in the plain (float64) or the precision (float32) form.
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np
import torch


def bassetti_erskine(x: np.ndarray, y: np.ndarray, sx: float, sy: float) -> Tuple[np.ndarray, np.ndarray]:
    """(Ex, Ey) of a unit-charge bi-Gaussian (sigma sx, sy) in units where a point charge gives r/|r|^2.

    sx != sy: Bassetti & Erskine (CERN-ISR-TH/80-06) through the Faddeeva function w(z):
    Ey + i Ex = sqrt(pi / (2 (sx^2 - sy^2))) [w(z1) - exp(-x^2/2sx^2 - y^2/2sy^2) w(z2)], with
    z1 = (x + i y) / sqrt(2 (sx^2 - sy^2)) and z2 = (x sy/sx + i y sx/sy) / sqrt(2 (sx^2 - sy^2)),
    evaluated for sx > sy on |x|, |y| and signed back; sx < sy by exchanging the axes.  sx == sy: the
    round closed form (1 - exp(-r^2 / 2 s^2)) r / r^2."""
    from scipy.special import wofz

    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if math.isclose(sx, sy, rel_tol=1e-12):
        r2 = x * x + y * y
        with np.errstate(invalid="ignore", divide="ignore"):
            f = np.where(r2 > 0, (1.0 - np.exp(-r2 / (2 * sx * sx))) / r2, 0.0)
        return f * x, f * y
    if sx < sy:
        ey, ex = bassetti_erskine(y, x, sy, sx)
        return ex, ey
    ax, ay = np.abs(x), np.abs(y)
    d = math.sqrt(2.0 * (sx * sx - sy * sy))
    z1 = (ax + 1j * ay) / d
    z2 = (ax * (sy / sx) + 1j * ay * (sx / sy)) / d
    v = math.sqrt(math.pi) / d * (wofz(z1) - np.exp(-ax * ax / (2 * sx * sx) - ay * ay / (2 * sy * sy)) * wofz(z2))
    return np.sign(x) * v.imag, np.sign(y) * v.real


def quantile_lattice(n: int, sx: float, sy: float) -> Tuple[np.ndarray, np.ndarray]:
    """n x n deterministic Gaussian source: the product of the 1D normal quantiles at (k - 1/2)/n."""
    from scipy.special import erfinv

    u = (np.arange(1, n + 1) - 0.5) / n
    q = math.sqrt(2.0) * erfinv(2 * u - 1)
    return np.repeat(sx * q, n), np.tile(sy * q, n)


def field_error(solver, sx: float, sy: float, dtype: torch.dtype = torch.float64, device: int = 0,
                n_source: int = 400, n_probe: int = 81, extent: float = 4.0, correction=None) -> Dict[str, float]:
    """RMS and max field error of one collide of `solver` (slice_pair or node grid, any deposit and
    derivative) against exact Bassetti-Erskine, for an (sx, sy) Gaussian source slice.  correction: a learned
    field correction to attach, (network, out_scale, tolerance, edge) (octo_b200.learned)."""
    from dataclasses import replace

    from .api import Context
    from .beam import Beam, BeamParams
    from .solver import LongitudinalSlicing

    changes = dict(kbb1=1.0, kbb2=1.0, luminosity_scale=1.0,
                   slicing=LongitudinalSlicing(nslices=1, method="normal_quantile"), slicing1=None, slicing2=None)
    s = solver.replace(**changes) if hasattr(solver, "margin_sigma") else replace(solver, **changes)
    xs, ys = quantile_lattice(n_source, sx, sy)
    g = np.linspace(-extent, extent, n_probe)
    px_, py_ = np.meshgrid(g * sx, g * sy, indexing="ij")
    xp, yp = px_.ravel(), py_.ravel()
    src = np.zeros((6, xs.size))
    src[0], src[2] = xs, ys
    prb = np.zeros((6, xp.size))
    prb[0], prb[2] = xp, yp
    dev = f"cuda:{device}"
    p = BeamParams(1.0, 1.0, 1.0, 1.0, 1.0)
    b1 = Beam.from_numpy(src, p, device=dev, dtype=dtype)
    b2 = Beam.from_numpy(prb, p, device=dev, dtype=dtype)
    ctx = Context(s, device, dtype)
    try:
        if correction is not None:
            from . import _lib
            net, out_scale, tol, edge = correction
            rc = _lib.lib().octo_set_field_correction(ctx.ptr, net.ptr, float(out_scale), float(tol), int(edge))
            if rc != _lib.OCTO_OK:
                raise RuntimeError(_lib.last_error(ctx.ptr))
        ctx.collide(b1, b2, turn=1, compute_luminosity=False)
    finally:
        if correction is not None:
            from . import _lib
            _lib.lib().octo_set_field_correction(ctx.ptr, None, 1.0, 1.0, 0)
        ctx.close()
    out = b2.coords.to(torch.float64).cpu().numpy()
    # kick = 2 kbb2 / n1 * sum_taps w E(n1 unit charges) = 2 E_unit
    ex = (out[1] - 0.0) / 2.0
    ey = (out[3] - 0.0) / 2.0
    bx, by = bassetti_erskine(xp, yp, sx, sy)
    err = np.hypot(ex - bx, ey - by)
    norm = float(np.max(np.hypot(bx, by)))
    return {"rms": float(np.sqrt(np.mean(err * err)) / norm), "max": float(err.max() / norm),
            "aspect": sx / sy, "points": int(xp.size)}


def emittances(beam) -> Tuple[float, float, float]:
    """RMS emittances sqrt(<u^2><u'^2> - <u u'>^2) of the (x, px), (y, py), (z, pz) planes with population
    moments, as beam_statistics reports them (Beam.jl:650-734); reduced in FP64 on the beam's device."""
    c = beam.coords.to(torch.float64)
    c = c - c.mean(dim=1, keepdim=True)
    out = []
    for k in range(3):
        u, v = c[2 * k], c[2 * k + 1]
        a, b, d = (u * u).mean(), (v * v).mean(), (u * v).mean()
        out.append(float(torch.sqrt(torch.clamp(a * b - d * d, min=0.0))))
    return tuple(out)
