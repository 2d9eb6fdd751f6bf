"""Line tracking between collisions.

The zero-length elements the production strong-strong lines place around the collision point
(examples/strong_strong_tracking.jl:206-262) and ``track``, which applies a line of them to every
particle of a beam in one fused device pass: the twin of ``track!(rep, elems, turns; context)`` with
``fusedTrack`` (src/track/phase6d_track.jl:25-35, 197-212; src/track/fused_track.jl:53-77).

The spec classes mirror the reference's friendly constructors (names, keyword meaning, defaults,
validation with ``ArgumentError``); ``to_c()`` is their ``compile_runtime`` step into the C ABI's
``octo_element``.  The counter-RNG state (global seed and method, stream-id counter) mirrors
src/math/counter_rng.jl:23-96.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .solver import ArgumentError

CLIGHT = 299_792_458.0  # src/constants/Constants.jl:8

# ---------------------------------------------------------------- counter-RNG state (counter_rng.jl:23-96)
_rng_lock = threading.Lock()
_rng_state = {"seed": 0, "method": "philox", "id_counter": 0}


def rng_method_code(method) -> int:
    """rng_method_code (counter_rng.jl:88-93): :philox -> 1, :splitmix -> 2."""
    if isinstance(method, int):
        if method in (_lib.RNG_PHILOX, _lib.RNG_SPLITMIX):
            return method
        raise ArgumentError(f"unknown RNG method code {method}")
    m = str(method).lower().lstrip(":")
    if m == "philox":
        return _lib.RNG_PHILOX
    if m == "splitmix":
        return _lib.RNG_SPLITMIX
    raise ArgumentError(f"unknown RNG method {method}; use :philox or :splitmix")


def set_global_rng(seed: Optional[int] = None, method=None):
    """set_global_rng! (counter_rng.jl:34-38)."""
    with _rng_lock:
        if seed is not None:
            _rng_state["seed"] = int(seed) & 0xFFFFFFFFFFFFFFFF
        if method is not None:
            rng_method_code(method)
            _rng_state["method"] = str(method).lower().lstrip(":")
        return _rng_state["seed"], _rng_state["method"]


def global_rng_seed() -> int:
    return _rng_state["seed"]


def global_rng_method() -> str:
    return _rng_state["method"]


def next_rng_id() -> int:
    """next_rng_id! (counter_rng.jl:50-56): the next automatically assigned stream id."""
    with _rng_lock:
        _rng_state["id_counter"] += 1
        return _rng_state["id_counter"]


def claim_rng_id(rng_id: int) -> int:
    """claim_rng_id! (counter_rng.jl:58-81): record an explicit id so automatic ids skip past it."""
    with _rng_lock:
        if rng_id > 0:
            _rng_state["id_counter"] = max(_rng_state["id_counter"], int(rng_id))
        return int(rng_id)


def reset_rng_id_counter(value: int = 0) -> int:
    with _rng_lock:
        _rng_state["id_counter"] = int(value)
        return _rng_state["id_counter"]


# ---------------------------------------------------------------- element specs
def _tuple(values, n: int, name: str = "values"):
    values = tuple(values)
    if len(values) != n:
        raise ArgumentError(f"expected {n} values, got {len(values)}")
    return tuple(float(v) for v in values)


def _element(kind: int) -> _lib.OctoElement:
    e = _lib.OctoElement()
    e.kind = kind
    return e


def _mat_identity():
    return [[1.0 if i == j else 0.0 for j in range(6)] for i in range(6)]


def _mmul66(a, b):
    """_mmul66 (linear6d.jl:216-222): left-to-right sums over the inner index."""
    out = [[0.0] * 6 for _ in range(6)]
    for i in range(6):
        for j in range(6):
            s = a[i][0] * b[0][j]
            for l in range(1, 6):
                s = s + a[i][l] * b[l][j]
            out[i][j] = s
    return out


def _mzeta66(z):
    m = _mat_identity()
    for i in range(4):
        m[i][4] = z[i]
    m[5][0], m[5][1], m[5][2], m[5][3] = z[1], -z[0], z[3], -z[2]
    return m


def _meta66(e):
    m = _mat_identity()
    for i in range(4):
        m[i][5] = e[i]
    m[4][0], m[4][1], m[4][2], m[4][3] = -e[1], e[0], -e[3], e[2]
    return m


def _mR66(c):
    m = _mat_identity()
    g = math.sqrt(1.0 - c[0] * c[3] + c[1] * c[2])
    for i in range(4):
        m[i][i] = g
    m[0][2], m[0][3], m[1][2], m[1][3] = c[0], c[1], c[2], c[3]
    m[2][0], m[2][1], m[3][0], m[3][1] = -c[3], c[1], c[2], -c[0]
    return m


def _minv66(m):
    return np.linalg.inv(np.array(m, dtype=np.float64)).tolist()


def linear6d_symplectic_ratio(m: Sequence[float]) -> float:
    """_linear6d_symplectic_error (linear6d.jl:147-204): worst row residual of M^T J M - J over its
    componentwise forward-error bound 64 eps max(1, row scale); > 1 is not symplectic."""
    m = [float(v) for v in m]
    if not all(math.isfinite(v) for v in m):
        return math.inf
    worst = 0.0
    eps = np.finfo(np.float64).eps
    for i in range(6):
        row_res = row_scale = 0.0
        for j in range(6):
            value = pscale = 0.0
            for q in (0, 2, 4):
                pos = m[q * 6 + i] * m[(q + 1) * 6 + j]
                neg = m[(q + 1) * 6 + i] * m[q * 6 + j]
                if not (math.isfinite(pos) and math.isfinite(neg)):
                    return math.inf
                value = (value + pos) - neg
                pscale += abs(pos) + abs(neg)
            target = 1.0 if (i % 2 == 0 and j == i + 1) else (-1.0 if (i % 2 == 1 and j == i - 1) else 0.0)
            row_res += abs(value - target)
            row_scale += max(abs(target), pscale)
        tol = 64.0 * eps * max(1.0, row_scale)
        if not (math.isfinite(row_res) and math.isfinite(tol)):
            return math.inf
        ratio = row_res / tol if tol > 0 else (0.0 if row_res == 0 else math.inf)
        worst = max(worst, ratio)
    return worst


class Linear6DSpec:
    """Linear6DSpec (linear6d.jl:27-61): either ``matrix`` (6x6 or 36 row-major, canonical symplectic) or
    optics ``beta1, dmu`` with ``beta2=beta1, alpha1=(0,0,0), alpha2=alpha1`` and the dispersion /
    coupling tuples ``zeta1, eta1, R1`` (``zeta2, eta2, R2`` default to them), composed as
    Z(zeta2) E(eta2) R(R2) B R(R1)^-1 E(eta1)^-1 Z(zeta1)^-1 (linear6d.jl:233-275)."""

    def __init__(self, matrix=None, beta1=None, dmu=None, beta2=None, alpha1=(0.0, 0.0, 0.0), alpha2=None,
                 zeta1=(0.0,) * 4, eta1=(0.0,) * 4, R1=(0.0,) * 4, zeta2=None, eta2=None, R2=None):
        if matrix is not None:
            m = np.asarray(matrix, dtype=np.float64).reshape(-1)
            if m.size != 36:
                raise ArgumentError(f"Linear6D matrix must have 36 entries, got {m.size}")
            ratio = linear6d_symplectic_ratio(m)
            if not ratio <= 1.0:
                raise ArgumentError("Linear6DSpec matrix must be finite and canonical symplectic in "
                                    f"(x, px, y, py, z, pz) order: ratio={ratio}.")
            self.matrix = [float(v) for v in m]
            return
        if beta1 is None:
            raise ArgumentError("Linear6DSpec requires either matrix or beta1")
        if dmu is None:
            raise ArgumentError("Linear6DSpec requires either matrix or dmu")
        beta2 = beta1 if beta2 is None else beta2
        alpha2 = alpha1 if alpha2 is None else alpha2
        zeta2 = zeta1 if zeta2 is None else zeta2
        eta2 = eta1 if eta2 is None else eta2
        R2 = R1 if R2 is None else R2
        b1, b2 = _tuple(beta1, 3), _tuple(beta2, 3)
        a1, a2 = _tuple(alpha1, 3), _tuple(alpha2, 3)
        mu = _tuple(dmu, 3)
        B = [[0.0] * 6 for _ in range(6)]
        for i in range(3):
            s, c = math.sin(mu[i]), math.cos(mu[i])
            r = 2 * i
            B[r][r] = math.sqrt(b2[i] / b1[i]) * (c + a1[i] * s)
            B[r][r + 1] = math.sqrt(b2[i] * b1[i]) * s
            B[r + 1][r] = (-(1.0 + a1[i] * a2[i]) * s + (a1[i] - a2[i]) * c) / math.sqrt(b1[i] * b2[i])
            B[r + 1][r + 1] = math.sqrt(b1[i] / b2[i]) * (c - a2[i] * s)
        z1, e1, r1 = _tuple(zeta1, 4), _tuple(eta1, 4), _tuple(R1, 4)
        z2, e2, r2 = _tuple(zeta2, 4), _tuple(eta2, 4), _tuple(R2, 4)
        left = _mmul66(_mmul66(_mmul66(_mmul66(_mzeta66(z2), _meta66(e2)), _mR66(r2)), B), _minv66(_mR66(r1)))
        right = _mmul66(_minv66(_meta66(e1)), _minv66(_mzeta66(z1)))
        m = _mmul66(left, right)
        self.matrix = [m[i][j] for i in range(6) for j in range(6)]

    def inverse(self) -> "Linear6DSpec":
        """Linear6DSpec(matrix = inv(Matrix(Linear6D(spec)))), as the production lines build their
        inverse transports (examples/strong_strong_tracking.jl:210, 215)."""
        return Linear6DSpec(matrix=np.linalg.inv(np.array(self.matrix).reshape(6, 6)))

    def to_c(self) -> _lib.OctoElement:
        e = _element(_lib.ELEM_LINEAR6D)
        for k, v in enumerate(self.matrix):
            e.p[k] = v
        return e


class ThinCrabCavitySpec:
    """ThinCrabCavitySpec{N}(frequency; strengthX, strengthY, phase) (crab_cavity.jl:14-45): N harmonics,
    omitted tuples filled with zeros; frequency finite and nonzero."""

    def __init__(self, frequency, N: Optional[int] = None, strengthX=(), strengthY=(), phase=()):
        f = float(frequency)
        if not (math.isfinite(f) and f != 0.0):
            raise ArgumentError(f"thin crab-cavity frequency must be finite and nonzero; got {f}")
        if N is None:
            N = max(len(tuple(strengthX)), len(tuple(strengthY)), len(tuple(phase)), 1)
        N = int(N)
        if not 1 <= N <= _lib.CRAB_MAX_HARMONICS:
            raise ArgumentError(f"thin crab-cavity harmonic count must be 1..{_lib.CRAB_MAX_HARMONICS}")

        def harm(values):
            values = tuple(values)
            if len(values) == 0:
                return (0.0,) * N
            if len(values) != N:
                raise ArgumentError(f"expected {N} harmonic values, got {len(values)}")
            return tuple(float(v) for v in values)

        self.frequency, self.N = f, N
        self.strengthX, self.strengthY, self.phase = harm(strengthX), harm(strengthY), harm(phase)

    @property
    def kcc(self) -> float:
        return 2.0 * math.pi * self.frequency / CLIGHT

    def to_c(self) -> _lib.OctoElement:
        e = _element(_lib.ELEM_THIN_CRAB_CAVITY)
        e.nharm = self.N
        e.p[0] = self.frequency
        for h in range(self.N):
            e.p[1 + h], e.p[9 + h], e.p[17 + h] = self.strengthX[h], self.strengthY[h], self.phase[h]
        return e


class LorentzBoostSpec:
    """LorentzBoostSpec(angle) (lorentz_boost.jl:18-25): angle is HALF the full crossing angle."""
    kind = _lib.ELEM_LORENTZ_BOOST

    def __init__(self, angle):
        self.angle = float(angle)

    def to_c(self) -> _lib.OctoElement:
        if not math.isfinite(self.angle):
            raise ArgumentError("Lorentz boost angle must be finite")
        e = _element(self.kind)
        e.p[0] = self.angle
        return e


class RevLorentzBoostSpec(LorentzBoostSpec):
    """RevLorentzBoostSpec(angle) (lorentz_boost.jl:34-38), the exact inverse of LorentzBoostSpec."""
    kind = _lib.ELEM_REV_LORENTZ_BOOST


def _transverse(values, name):
    values = tuple(values)
    if len(values) not in (2, 3):
        raise ArgumentError(f"{name} must contain 2 or 3 values, got {len(values)}")
    return float(values[0]), float(values[1])


class ChromaticityKickSpec:
    """ChromaticityKickSpec(; xi, beta, alpha=(0,0,0), zeta, eta, R) (chromaticity_kick.jl:17-39): beta and
    alpha take 2 or 3 values, only the transverse pair is used."""

    def __init__(self, xi, beta, alpha=(0.0, 0.0, 0.0), zeta=(0.0,) * 4, eta=(0.0,) * 4, R=(0.0,) * 4):
        self.xi = _tuple(xi, 2)
        self.beta = _transverse(beta, "beta")
        self.alpha = _transverse(alpha, "alpha")
        self.zeta, self.eta, self.R = _tuple(zeta, 4), _tuple(eta, 4), _tuple(R, 4)
        _check_coupling(self.R)

    def to_c(self) -> _lib.OctoElement:
        e = _element(_lib.ELEM_CHROMATICITY_KICK)
        vals = self.xi + self.beta + self.alpha + self.zeta + self.eta + self.R
        for k, v in enumerate(vals):
            e.p[k] = v
        return e


def _check_coupling(r):
    """The XYCoupling constructor's check (linear_maps.jl:296-310)."""
    det = 1.0 + r[0] * r[3] - r[1] * r[2]
    if math.isfinite(det) and det <= 0:
        raise ArgumentError(f"XYCoupling is not invertible: 1 + r1*r4 - r2*r3 = {det} must be positive, because the "
                            f"map scales by 1/sqrt of it. Got r1={r[0]}, r2={r[1]}, r3={r[2]}, r4={r[3]}.")


RADIATION_METHODS = {"radiation": _lib.RAD_RADIATION, "damping": _lib.RAD_DAMPING, "diffusion": _lib.RAD_DIFFUSION}


@dataclass
class LumpedRad:
    """The compiled runtime of LumpedRadSpec (radiation.jl:71-131): effective components, per-plane damping
    factors exp(-1/tau) and the nine excitation amplitudes."""
    method: str
    is_damping: bool
    is_excitation: bool
    damping: tuple
    excitation: tuple
    rng_id: int


class LumpedRadSpec:
    """LumpedRadSpec(; damping_turns, beta=(1,1,1), alpha=(0,0,0), sigma=(-1,-1,-1), zeta, eta, R,
    is_damping=True, is_excitation=True, tracking_method="radiation", rng_id=0) (radiation.jl:19-51).
    tracking_method: "radiation" (Radiation6DMap), "damping" (Damping6DMap) or "diffusion"
    (Diffusion6DMap); rng_id 0 auto-assigns a unique stream id, an explicit id is claimed."""

    def __init__(self, damping_turns, beta=(1.0, 1.0, 1.0), alpha=(0.0, 0.0, 0.0), sigma=(-1.0, -1.0, -1.0),
                 zeta=(0.0,) * 4, eta=(0.0,) * 4, R=(0.0,) * 4, is_damping=True, is_excitation=True,
                 tracking_method="radiation", rng_id=0):
        self.damping_turns = _tuple(damping_turns, 3)
        self.beta, self.alpha, self.sigma = _tuple(beta, 3), _tuple(alpha, 3), _tuple(sigma, 3)
        self.zeta, self.eta, self.R = _tuple(zeta, 4), _tuple(eta, 4), _tuple(R, 4)
        self.is_damping, self.is_excitation = bool(is_damping), bool(is_excitation)
        if tracking_method not in RADIATION_METHODS:
            raise ArgumentError("LumpedRad supports Radiation6DMap, Damping6DMap, or Diffusion6DMap; "
                                f"got {tracking_method}")
        self.tracking_method = tracking_method
        rid = int(rng_id)
        self.rng_id = next_rng_id() if rid == 0 else claim_rng_id(rid)

    def compile_runtime(self, tracking_method: Optional[str] = None) -> LumpedRad:
        """LumpedRad(spec, method) (radiation.jl:83-171), with its validation."""
        method = tracking_method or self.tracking_method
        if method not in RADIATION_METHODS:
            raise ArgumentError(f"LumpedRad supports Radiation6DMap, Damping6DMap, or Diffusion6DMap; got {method}")
        for i, v in enumerate(self.damping_turns):
            if not v > 0:
                raise ArgumentError(f"damping_turns[{i + 1}] must be positive, got {v}")
        for name, values in (("beta", self.beta), ("alpha", self.alpha), ("sigma", self.sigma),
                             ("zeta", self.zeta), ("eta", self.eta), ("R", self.R)):
            for i, v in enumerate(values):
                if not math.isfinite(v):
                    raise ArgumentError(f"{name}[{i + 1}] must be finite, got {v}")
        for i, v in enumerate(self.beta):
            if not v > 0:
                raise ArgumentError(f"beta[{i + 1}] must be positive, got {v}")
        enabled = all(v >= 0 for v in self.sigma)
        if not (enabled or all(v < 0 for v in self.sigma)):
            raise ArgumentError("sigma must be nonnegative in all three planes to enable excitation or negative in "
                                "all three planes to disable it")
        _check_coupling(self.R)
        damping = tuple(math.exp(-1.0 / t) for t in self.damping_turns)
        scale = tuple(math.sqrt(-math.expm1(-2.0 / t)) for t in self.damping_turns)
        exc = []
        for i in range(3):
            if self.sigma[i] < 0:
                exc += [0.0, 0.0, 0.0]
                continue
            amp = self.sigma[i] * scale[i]
            slope = amp / self.beta[i]
            exc += [amp, slope, -slope * self.alpha[i]]
        is_damping = self.is_damping and method != "diffusion"
        is_excitation = self.is_excitation and enabled and method != "damping"
        return LumpedRad(method, is_damping, is_excitation, damping, tuple(exc), self.rng_id)

    def to_c(self, tracking_method: Optional[str] = None) -> _lib.OctoElement:
        method = tracking_method or self.tracking_method
        self.compile_runtime(method)
        e = _element(_lib.ELEM_LUMPED_RAD)
        vals = self.damping_turns + self.beta + self.alpha + self.sigma + self.zeta + self.eta + self.R
        for k, v in enumerate(vals):
            e.p[k] = v
        e.mode = RADIATION_METHODS[method]
        e.is_damping, e.is_excitation = int(self.is_damping), int(self.is_excitation)
        e.rng_id = self.rng_id
        return e


class CrabDispersionSpec:
    """CrabDispersionSpec(; zeta1..zeta4) (linear_maps.jl:49-75, map :125-132)."""

    def __init__(self, zeta1=0.0, zeta2=0.0, zeta3=0.0, zeta4=0.0):
        self.zeta = (float(zeta1), float(zeta2), float(zeta3), float(zeta4))

    def to_c(self) -> _lib.OctoElement:
        e = _element(_lib.ELEM_CRAB_DISPERSION)
        for k, v in enumerate(self.zeta):
            e.p[k] = v
        return e


class MomentumDispersionSpec:
    """MomentumDispersionSpec(; eta1..eta4) (linear_maps.jl:138-163, map :213-220)."""

    def __init__(self, eta1=0.0, eta2=0.0, eta3=0.0, eta4=0.0):
        self.eta = (float(eta1), float(eta2), float(eta3), float(eta4))

    def to_c(self) -> _lib.OctoElement:
        e = _element(_lib.ELEM_MOMENTUM_DISPERSION)
        for k, v in enumerate(self.eta):
            e.p[k] = v
        return e


XY_MODES = {"undef": 0, "A": 1, "B": 2}


class XYCouplingSpec:
    """XYCouplingSpec(; r1..r4, mode="A") (linear_maps.jl:240-266, map :355-373); mode "undef" is the identity."""

    def __init__(self, r1=0.0, r2=0.0, r3=0.0, r4=0.0, mode="A"):
        if mode not in XY_MODES:
            raise ArgumentError(f"XYCoupling mode must be one of {tuple(XY_MODES)}")
        self.r = (float(r1), float(r2), float(r3), float(r4))
        self.mode = mode
        if mode != "undef":
            _check_coupling(self.r)

    def to_c(self) -> _lib.OctoElement:
        e = _element(_lib.ELEM_XY_COUPLING)
        for k, v in enumerate(self.r):
            e.p[k] = v
        e.mode = XY_MODES[self.mode]
        return e


def flatten(elems) -> list:
    """fusedTrack's compile-time expansion of nested tuples of elements (fused_track.jl:28-51)."""
    out = []
    if isinstance(elems, (list, tuple)):
        for e in elems:
            out += flatten(e)
    else:
        out.append(elems)
    return out


def compile_line(elems) -> "C.Array":
    flat = flatten(elems)
    if len(flat) > _lib.LINE_MAX_ELEMENTS:
        raise ArgumentError(f"a line holds at most {_lib.LINE_MAX_ELEMENTS} elements")
    arr = (_lib.OctoElement * max(len(flat), 1))()
    for k, e in enumerate(flat):
        if not hasattr(e, "to_c"):
            raise ArgumentError(f"line element {k + 1} ({type(e).__name__}) is not a line element spec")
        arr[k] = e.to_c()
    return arr, len(flat)


# ---------------------------------------------------------------- the strong-strong example's lines
EIC_CROSSING_HALF_ANGLE = 12.5e-3
EIC_OPTICS = {
    "electron": dict(beta=(0.55, 0.056, 0.7e-2 / 5.5e-4), alpha=(0.0, 0.0, 0.0), sigma=(106.0e-6, 9.5e-6, 0.7e-2),
                     crab_beta=(150.0, 30.0, 0.7e-2 / 5.5e-4), tune=(0.08, 0.14, -0.069), chromaticity=(1.0, 1.0),
                     crab_frequency=394.0e6,
                     crab_strength_x=(math.tan(12.5e-3) / math.sqrt(150.0 * 0.55), 0.0, 0.0),
                     radiation_damping_turns=(4000.0, 4000.0, 2000.0), rng_id=3),
    "proton": dict(beta=(0.8, 0.072, 6.0e-2 / 6.6e-4), alpha=(0.0, 0.0, 0.0), sigma=(95.0e-6, 8.5e-6, 6.0e-2),
                   crab_beta=(1300.0, 30.0, 6.0e-2 / 6.6e-4), tune=(0.228, 0.210, -0.01), chromaticity=(2.0, 2.0),
                   crab_frequency=197.0e6,
                   crab_strength_x=(math.tan(12.5e-3) / math.sqrt(1300.0 * 0.8) * 4.0 / 3.0,
                                    -math.tan(12.5e-3) / math.sqrt(1300.0 * 0.8) / 3.0, 0.0)),
}


def eic_like_segments(beam: str, crossing_half_angle: float = EIC_CROSSING_HALF_ANGLE):
    """The two line segments of one ring of the strong-strong example (examples/strong_strong_tracking.jl:55-110
    parameters, 206-262 lines) around its collision: before it, the inverse crab-to-IP transport, the crab
    cavity, the crab-to-IP transport and the Lorentz boost; after it, the reverse boost, the IP-to-crab
    transport, the second crab cavity, its inverse transport, the one-turn map, the chromaticity kick and
    (electrons) lumped radiation.  Returns (before, after)."""
    o = EIC_OPTICS[beam]
    tccb2ip = Linear6DSpec(beta1=o["crab_beta"], beta2=o["beta"], alpha1=o["alpha"], alpha2=o["alpha"],
                           dmu=(math.pi / 2.0, 0.0, 0.0))
    ip2tcca = Linear6DSpec(beta1=o["beta"], beta2=o["crab_beta"], alpha1=o["alpha"], alpha2=o["alpha"],
                           dmu=(math.pi / 2.0, 0.0, 0.0))
    crab = ThinCrabCavitySpec(o["crab_frequency"], N=3, strengthX=o["crab_strength_x"], strengthY=(0.0,) * 3,
                              phase=(0.0,) * 3)
    one_turn = Linear6DSpec(beta1=o["beta"], beta2=o["beta"], alpha1=o["alpha"], alpha2=o["alpha"],
                            dmu=tuple(2.0 * math.pi * t for t in o["tune"]))
    chrom = ChromaticityKickSpec(xi=o["chromaticity"], beta=o["beta"], alpha=o["alpha"])
    before = (tccb2ip.inverse(), crab, tccb2ip, LorentzBoostSpec(crossing_half_angle))
    after = [RevLorentzBoostSpec(crossing_half_angle), ip2tcca, crab, ip2tcca.inverse(), one_turn, chrom]
    if "radiation_damping_turns" in o:
        after.append(LumpedRadSpec(damping_turns=o["radiation_damping_turns"], beta=o["beta"], alpha=o["alpha"],
                                   sigma=o["sigma"], is_damping=True, is_excitation=True, rng_id=o["rng_id"]))
    return before, tuple(after)
