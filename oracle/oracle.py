"""ctypes binding of the FP64 CPU oracle (oracle/octo_oracle.cpp) -- TEST INFRASTRUCTURE.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module, as the checker.  The product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboctooracle.so")

OK, ERR_NONFINITE, ERR_UNSUPPORTED, ERR_EXTENT, ERR_ARG = 0, 1, 2, 3, 4

# Physical constants (src/constants/Constants.jl:11-20).
RE = 2.8179403205e-15
EMASS_EV = 0.51099895069e6
ME0 = EMASS_EV
PMASS_EV = 938.27208943e6


class OOElement(C.Structure):
    """oo_element: the layout of the product's octo_element."""
    _fields_ = [("kind", C.c_int32), ("nharm", C.c_int32), ("mode", C.c_int32), ("is_damping", C.c_int32),
                ("is_excitation", C.c_int32), ("reserved", C.c_int32), ("rng_id", C.c_uint64),
                ("p", C.c_double * 40)]


def build() -> str:
    src = os.path.join(HERE, "octo_oracle.cpp")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


class OOOptions(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("deposit_method", C.c_int32), ("lum_deposit_method", C.c_int32),
        ("lum_nx", C.c_int32), ("lum_ny", C.c_int32),
        ("green_type", C.c_int32), ("green_cache", C.c_int32),
        ("field_derivative", C.c_int32), ("slice_interpolation", C.c_int32),
        ("interaction_grid", C.c_int32), ("grid_extent", C.c_int32),
        ("grid_extent_sigma", C.c_double),
        ("min_extent_x", C.c_double), ("min_extent_y", C.c_double),
        ("grid_quantize", C.c_double),
        ("green_min_ratio", C.c_double), ("green_growth", C.c_double),
        ("longitudinal_kick", C.c_int32),
        ("slicing_method1", C.c_int32), ("slicing_method2", C.c_int32),
        ("nslices1", C.c_int32), ("nslices2", C.c_int32),
        ("center_position1", C.c_int32), ("center_position2", C.c_int32),
        ("positions1", C.POINTER(C.c_double)), ("positions2", C.POINTER(C.c_double)),
        ("has_kbb1", C.c_int32), ("has_kbb2", C.c_int32), ("has_lum_scale", C.c_int32),
        ("kbb1", C.c_double), ("kbb2", C.c_double), ("lum_scale", C.c_double),
        ("fixed_point_deposit", C.c_int32),
        ("nthreads", C.c_int32),
        ("gaussian", C.c_int32), ("neutralize", C.c_int32),
        ("margin_sigma", C.c_double),
        ("resolution1", C.c_int32), ("resolution2", C.c_int32),
        ("coupling_tol", C.c_double),
    ]


class OOBeamParams(C.Structure):
    _fields_ = [("charge", C.c_double), ("mc2", C.c_double), ("E0", C.c_double),
                ("r0", C.c_double), ("npart", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        d, i32, i64, u64, vp = C.c_double, C.c_int32, C.c_int64, C.c_uint64, C.c_void_p
        P = C.POINTER
        L = _lib
        L.oo_philox4x32_block.argtypes = [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]
        L.oo_counter_uint64.restype = u64
        L.oo_counter_uint64.argtypes = [u64] * 5
        L.oo_normal.restype = d
        L.oo_normal.argtypes = [u64] * 5
        L.oo_beam_gaussian.argtypes = [i64, u64, u64, P(d), P(d), P(d), d] + [P(d)] * 6
        L.oo_erfinv.restype = d
        L.oo_erfinv.argtypes = [d]
        L.oo_faddeeva.argtypes = [d, d, P(d)]
        L.oo_be_response.argtypes = [d, d, d, d, d, P(d)]
        L.oo_gaussian_profile.argtypes = [i32, d, d, d, d, i32, P(d)]
        L.oo_kernel_integral.restype = d
        L.oo_kernel_integral.argtypes = [d, d]
        L.oo_atan_ratio.restype = d
        L.oo_atan_ratio.argtypes = [d, d]
        L.oo_cic_weights.argtypes = [d, i32, P(i32), P(d)]
        L.oo_tsc_weights.argtypes = [d, i32, P(i32), P(d)]
        L.oo_green_table.argtypes = [i32, d, d, d, d, d, d, i32, i32, P(d)]
        L.oo_fft2.argtypes = [P(d), P(d), i32, i32, i32]
        L.oo_field.argtypes = [P(d), i32, i32, d, d, i32, P(d), P(d)]
        L.oo_fixed_scale_bits.restype = i32
        L.oo_fixed_scale_bits.argtypes = [i64]
        L.oo_deposit_drifted.argtypes = [i32, P(d), P(d), P(d), P(d), i64, d, d, d, d, d, i32, i32, i32,
                                         P(d), P(i64)]
        L.oo_solve_field.argtypes = [P(OOOptions), P(d), P(d), i64, d, d, d, d, d, d, P(d), P(d), P(d)]
        L.oo_interpolation_grids.argtypes = [P(OOOptions), P(d), P(d)]
        L.oo_interpolate.argtypes = [P(OOOptions), P(d), d, d] + [P(d)] * 9 + [i32, d, P(d)]
        L.oo_luminosity.restype = d
        L.oo_luminosity.argtypes = [P(OOOptions), P(d), P(d), i64, P(d), P(d), i64, d, P(d), P(d)]
        L.oo_slices.restype = C.c_int
        L.oo_slices.argtypes = [i32, i32, i32, P(d), P(d), i64, P(d), P(d), P(d), P(i64), P(i64), i32]
        L.oo_julia_range.restype = None
        L.oo_julia_range.argtypes = [d, d, i64, P(d)]
        L.oo_pair_batches.restype = i32
        L.oo_pair_batches.argtypes = [P(d), i32, P(d), i32, P(i32), P(i32), P(i32), P(i32), P(i32)]
        L.oo_union_bounds.restype = i32
        L.oo_union_bounds.argtypes = [P(P(d)), i64, d, P(P(d)), i64, P(d), P(i32)]
        L.oo_create.restype = vp
        L.oo_create.argtypes = [P(OOOptions)]
        L.oo_destroy.argtypes = [vp]
        L.oo_collide.restype = C.c_int
        L.oo_collide.argtypes = [vp, P(P(d)), i64, P(P(d)), i64, P(OOBeamParams), P(OOBeamParams), i32, P(d)]
        L.oo_cache_stats.argtypes = [vp, P(i64)]
        L.oo_dropped.restype = i64
        L.oo_dropped.argtypes = [vp]
        L.oo_pair_trace.restype = i64
        L.oo_pair_trace.argtypes = [vp, P(i32), P(i32), P(d), i64]
        L.oo_last_error.restype = C.c_char_p
        L.oo_last_error.argtypes = [vp]
        L.oo_capture_plane.argtypes = [vp, i32, i32, i32, i32]
        L.oo_capture_plane.restype = None
        L.oo_captured_plane.argtypes = [vp, P(i64), P(d), P(i32)]
        L.oo_captured_plane.restype = i32
        L.oo_linear6d.argtypes = [P(d)] + [P(d)] * 6 + [i64]
        L.oo_linear6d_matrix.argtypes = [P(d), P(d), P(d), P(d)]
        L.oo_gaussian_collide.argtypes = [P(OOOptions), d, i32, i32, i32, i32, i32, P(P(d)), i64, P(P(d)), i64,
                                          P(OOBeamParams), P(OOBeamParams), P(d)]
        L.oo_gaussian_collide.restype = C.c_int
        L.oo_gaussian_last_error.restype = C.c_char_p
        L.oo_be_near_round_L.argtypes = [d, d, d, d, d, P(d)]
        L.oo_be_principal_L.argtypes = [d, d, d, d, d, P(d)]
        L.oo_be_elliptic.argtypes = [d, d, d, d, P(d)]
        L.oo_track_line.argtypes = [P(OOElement), i32, i64, i32, C.c_uint64, i32] + [P(d)] * 6 + [i64]
        L.oo_track_line.restype = None
        L.oo_octopus_normal.argtypes = [C.c_uint64, i32, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]
        L.oo_octopus_normal.restype = d
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


_SYM = {
    "deposit_method": {"CIC": 0, "TSC": 1},
    "green_type": {"integrated": 0, "standard": 1},
    "green_cache": {"none": 0, "slice_pair": 1},
    "field_derivative": {"second": 2, "fourth": 4},
    "slice_interpolation": {"linear": 0, "quadratic": 1},
    "interaction_grid": {"slice_pair": 0, "source_slice": 1, "node": 2},
    "grid_extent": {"extrema": 0, "sigma": 1},
    "method": {"normal_quantile": 0, "gaussian": 0, "Gaussian": 0, "specified": 1, "equal_area": 2,
               "equal_count": 3, "equal_width": 4, "equal_spaced": 4},
    "center_position": {"centroid": 0, "midpoint": 1},
}


@dataclass
class OracleOptions:
    """Keyword twin of PICPoissonSolver (interface.jl:1384-1411) for the oracle."""
    grid: tuple = (128, 128)
    deposit_method: str = "CIC"
    luminosity_deposit_method: Optional[str] = None
    luminosity_grid: Optional[tuple] = None
    green_type: str = "integrated"
    green_cache: str = "slice_pair"
    field_derivative: str = "second"
    slice_interpolation: str = "linear"
    interaction_grid: str = "slice_pair"
    grid_extent: str = "extrema"
    grid_extent_sigma: float = 6.0
    min_transverse_extent: tuple = (0.0, 0.0)
    grid_quantize: float = 0.0
    slice_pair_green_min_ratio: float = 0.5
    slice_pair_green_growth: float = 0.25
    longitudinal_kick: bool = True
    nslices1: int = 1
    nslices2: int = 1
    method1: str = "normal_quantile"
    method2: str = "normal_quantile"
    center_position1: str = "centroid"
    center_position2: str = "centroid"
    positions1: Sequence[float] = field(default_factory=list)
    positions2: Sequence[float] = field(default_factory=list)
    kbb1: Optional[float] = None
    kbb2: Optional[float] = None
    luminosity_scale: Optional[float] = None
    fixed_point_deposit: bool = False
    nthreads: int = 1
    gaussian: bool = False          # GaussianPICPoissonSolver (the Gaussian-subtracted hybrid)
    neutralize: bool = True
    margin_sigma: float = 5.0
    resolution1: int = 100
    resolution2: int = 100
    coupling_tol: float = float("inf")  # hybrid: coupled (rotated) subtraction above this |r_xy|

    def to_c(self) -> OOOptions:
        o = OOOptions()
        o.nx, o.ny = int(self.grid[0]), int(self.grid[1])
        o.deposit_method = _SYM["deposit_method"][self.deposit_method]
        o.lum_deposit_method = -1 if self.luminosity_deposit_method is None else \
            _SYM["deposit_method"][self.luminosity_deposit_method]
        lg = self.luminosity_grid or (0, 0)
        o.lum_nx, o.lum_ny = int(lg[0]), int(lg[1])
        o.green_type = _SYM["green_type"][self.green_type]
        o.green_cache = _SYM["green_cache"][self.green_cache]
        o.field_derivative = _SYM["field_derivative"][self.field_derivative]
        o.slice_interpolation = _SYM["slice_interpolation"][self.slice_interpolation]
        o.interaction_grid = _SYM["interaction_grid"][self.interaction_grid]
        o.grid_extent = _SYM["grid_extent"][self.grid_extent]
        o.grid_extent_sigma = self.grid_extent_sigma
        o.min_extent_x, o.min_extent_y = map(float, self.min_transverse_extent)
        o.grid_quantize = self.grid_quantize
        o.green_min_ratio = self.slice_pair_green_min_ratio
        o.green_growth = self.slice_pair_green_growth
        o.longitudinal_kick = int(bool(self.longitudinal_kick))
        o.slicing_method1 = _SYM["method"][self.method1]
        o.slicing_method2 = _SYM["method"][self.method2]
        o.nslices1, o.nslices2 = int(self.nslices1), int(self.nslices2)
        o.center_position1 = _SYM["center_position"][self.center_position1]
        o.center_position2 = _SYM["center_position"][self.center_position2]
        self._p1 = np.ascontiguousarray(self.positions1, dtype=np.float64)
        self._p2 = np.ascontiguousarray(self.positions2, dtype=np.float64)
        o.positions1 = _dp(self._p1) if self._p1.size else None
        o.positions2 = _dp(self._p2) if self._p2.size else None
        o.has_kbb1 = int(self.kbb1 is not None)
        o.has_kbb2 = int(self.kbb2 is not None)
        o.has_lum_scale = int(self.luminosity_scale is not None)
        o.kbb1 = self.kbb1 or 0.0
        o.kbb2 = self.kbb2 or 0.0
        o.lum_scale = self.luminosity_scale or 0.0
        o.fixed_point_deposit = int(bool(self.fixed_point_deposit))
        o.nthreads = int(self.nthreads)
        o.gaussian = int(bool(self.gaussian))
        o.neutralize = int(bool(self.neutralize))
        o.margin_sigma = float(self.margin_sigma)
        o.resolution1, o.resolution2 = int(self.resolution1), int(self.resolution2)
        o.coupling_tol = float(self.coupling_tol)
        return o


def faddeeva(z: complex) -> complex:
    out = (C.c_double * 2)()
    lib().oo_faddeeva(C.c_double(z.real), C.c_double(z.imag), out)
    return complex(out[0], out[1])


def be_response(kbb, sigx, sigy, x, y):
    """(Kx, Ky, Hxx, Hyy): Bassetti-Erskine kick and kbb-scaled potential Hessians of a (sigx, sigy) Gaussian."""
    out = (C.c_double * 4)()
    lib().oo_be_response(C.c_double(kbb), C.c_double(sigx), C.c_double(sigy), C.c_double(x), C.c_double(y), out)
    return tuple(out)


def gaussian_profile(method, x0, h, mu, sigma, n):
    g = np.zeros(n)
    lib().oo_gaussian_profile(int(_SYM["deposit_method"][method]), C.c_double(x0), C.c_double(h), C.c_double(mu),
                              C.c_double(sigma), int(n), _dp(g))
    return g


def philox4x32_block(c, k):
    ci = (C.c_uint32 * 4)(*c)
    ki = (C.c_uint32 * 2)(*k)
    out = (C.c_uint32 * 4)()
    lib().oo_philox4x32_block(ci, ki, out)
    return tuple(out)


def beam_gaussian(n, *, seed=123456789, rng_id, beta, alpha=(0.0, 0.0, 0.0), sigma, cutoff=5.0):
    """Seeded 6D Gaussian beam as Beam(n, CPUThreadsBackend, Float64; ...) builds it (Beam.jl:475-515)."""
    out = np.empty((6, int(n)), dtype=np.float64)
    b = np.asarray(beta, np.float64); a = np.asarray(alpha, np.float64); s = np.asarray(sigma, np.float64)
    lib().oo_beam_gaussian(int(n), int(seed), int(rng_id), _dp(b), _dp(a), _dp(s), float(cutoff),
                           *[_dp(out[k]) for k in range(6)])
    return out


def beam_params(charge, mass, energy, npart, r0=None):
    return OOBeamParams(charge, mass, energy, RE * ME0 / mass if r0 is None else r0, npart)


def erfinv(x):
    return lib().oo_erfinv(float(x))


class Oracle:
    """A collide context holding the slice-pair Green cache across calls (task.runtime_cache)."""

    def __init__(self, options: OracleOptions):
        self.options = options
        self._copt = options.to_c()
        self._ctx = lib().oo_create(C.byref(self._copt))

    def __del__(self):
        if getattr(self, "_ctx", None):
            lib().oo_destroy(self._ctx)
            self._ctx = None

    def collide(self, beam1: np.ndarray, beam2: np.ndarray, p1: OOBeamParams, p2: OOBeamParams,
                compute_luminosity=True) -> float:
        """In-place collide of (6, n) float64 beams; returns the luminosity (NaN if not computed)."""
        P = C.POINTER(C.c_double)
        a1 = (P * 6)(*[_dp(beam1[k]) for k in range(6)])
        a2 = (P * 6)(*[_dp(beam2[k]) for k in range(6)])
        lum = C.c_double(np.nan)
        rc = lib().oo_collide(self._ctx, a1, beam1.shape[1], a2, beam2.shape[1], C.byref(p1), C.byref(p2),
                              int(bool(compute_luminosity)), C.byref(lum))
        if rc != OK:
            raise OracleErrorPy(rc, lib().oo_last_error(self._ctx).decode())
        return lum.value

    def cache_stats(self):
        out = (C.c_int64 * 3)()
        lib().oo_cache_stats(self._ctx, out)
        return tuple(out)

    def dropped(self):
        return lib().oo_dropped(self._ctx)

    def capture_plane(self, i: int, j: int, direction: int, plane: int = 0):
        """Arm a copy of one field-solve charge grid of the next collide (needs fixed_point_deposit)."""
        lib().oo_capture_plane(self._ctx, int(i), int(j), int(direction), int(plane))

    def captured_plane(self):
        """(int64 grid as (ny, nx), mesh (x0, y0, width, height), fixed-point bits) of the captured plane."""
        nx, ny = self.options.grid
        q = np.zeros(nx * ny, dtype=np.int64)
        mesh = (C.c_double * 4)()
        bits = C.c_int32()
        rc = lib().oo_captured_plane(self._ctx, q.ctypes.data_as(C.POINTER(C.c_int64)), mesh, C.byref(bits))
        if rc != OK:
            raise OracleErrorPy(rc, "no charge plane was captured")
        return q.reshape(ny, nx), tuple(mesh), bits.value

    def pair_trace(self):
        cap = 4096
        pi = (C.c_int32 * cap)(); pj = (C.c_int32 * cap)(); lum = (C.c_double * cap)()
        n = lib().oo_pair_trace(self._ctx, pi, pj, lum, cap)
        return [(pi[k], pj[k], lum[k]) for k in range(min(n, cap))]


class OracleErrorPy(Exception):
    def __init__(self, code, msg):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


def julia_range(start, stop, length):
    out = np.empty(int(length))
    lib().oo_julia_range(float(start), float(stop), int(length), _dp(out))
    return out


def slices(z, ns, method="normal_quantile", center_position="centroid", positions=(), resolution=100):
    z = np.ascontiguousarray(z, dtype=np.float64)
    n = z.size
    b = np.empty(ns + 1); c = np.empty(ns); w = np.empty(ns)
    cnt = np.empty(ns, np.int64); order = np.empty(n, np.int64)
    pos = np.ascontiguousarray(positions, np.float64)
    rc = lib().oo_slices(_SYM["method"][method], ns, _SYM["center_position"][center_position],
                         _dp(pos) if pos.size else None, _dp(z), n, _dp(b), _dp(c), _dp(w),
                         cnt.ctypes.data_as(C.POINTER(C.c_int64)), order.ctypes.data_as(C.POINTER(C.c_int64)),
                         int(resolution))
    if rc != OK:
        raise OracleErrorPy(rc, "slicing")
    return b, c, w, cnt, order


def union_bounds(source, center, partner):
    """The :source_slice union box (pic_cpu.jl:665-712) of a source slice, rows (x, px, y, py), against a
    partner, rows (x, px, y, py, z): ((sxmin, sxmax, symin, symax), (fxmin, fxmax, fymin, fymax)), or None when
    the partner has no finite z."""
    P = C.POINTER(C.c_double)
    src = [np.ascontiguousarray(source[k], np.float64) for k in range(4)]
    par = [np.ascontiguousarray(partner[k], np.float64) for k in range(5)]
    a = (P * 4)(*[_dp(v) for v in src])
    b = (P * 5)(*[_dp(v) for v in par])
    out = (C.c_double * 8)()
    valid = C.c_int32()
    rc = lib().oo_union_bounds(a, src[0].size, float(center), b, par[0].size, out, C.byref(valid))
    if rc != OK:
        raise OracleErrorPy(rc, "source-slice union bounds")
    return (tuple(out[:4]), tuple(out[4:])) if valid.value else None


def pair_batches(c1, c2):
    c1 = np.ascontiguousarray(c1, np.float64); c2 = np.ascontiguousarray(c2, np.float64)
    m = c1.size * c2.size
    I32 = C.POINTER(C.c_int32)
    arrs = [np.empty(m, np.int32) for _ in range(5)]
    nb = lib().oo_pair_batches(_dp(c1), c1.size, _dp(c2), c2.size, *[a.ctypes.data_as(I32) for a in arrs])
    batch_of, pi, pj, oi, oj = arrs
    batches = [[] for _ in range(nb)]
    for b, i, j in zip(batch_of, pi, pj):
        batches[b].append((int(i), int(j)))
    return batches, list(zip(oi.tolist(), oj.tolist()))


def linear6d_matrix(beta, alpha, tune):
    m = np.empty(36)
    lib().oo_linear6d_matrix(_dp(np.asarray(beta, np.float64)), _dp(np.asarray(alpha, np.float64)),
                             _dp(np.asarray(tune, np.float64)), _dp(m))
    return m


def linear6d(m, beam):
    lib().oo_linear6d(_dp(np.ascontiguousarray(m, np.float64)), *[_dp(beam[k]) for k in range(6)], beam.shape[1])


def solve_field(options: OracleOptions, x, y, source_grid, field_grid):
    """One field solve on the oracle: returns (phi, Ex, Ey) as (nx, ny) column-major arrays."""
    nx, ny = options.grid
    x = np.ascontiguousarray(x, np.float64); y = np.ascontiguousarray(y, np.float64)
    phi = np.empty(nx * ny); ex = np.empty(nx * ny); ey = np.empty(nx * ny)
    o = options.to_c()
    sx0, sy0, sw, sh = source_grid
    fx0, fy0 = field_grid[0], field_grid[1]
    lib().oo_solve_field(C.byref(o), _dp(x), _dp(y), x.size, sx0, sy0, sw, sh, fx0, fy0, _dp(phi), _dp(ex), _dp(ey))
    f = lambda a: a.reshape(ny, nx).T.copy()  # column-major (i fastest) -> [i, j]
    return f(phi), f(ex), f(ey)


def interaction_grids(options: OracleOptions, sxmin, sxmax, symin, symax, fxmin, fxmax, fymin, fymax):
    o = options.to_c()
    b = np.array([sxmin, sxmax, symin, symax, fxmin, fxmax, fymin, fymax], np.float64)
    out = np.empty(8)
    lib().oo_interpolation_grids(C.byref(o), _dp(b), _dp(out))
    return tuple(out[:4]), tuple(out[4:])


def interpolate(options: OracleOptions, grid, x, y, L, R, param, M=None):
    """Two-node (M is None, param = zL) or three-node (param = t) kick interpolation; planes are
    (phi, Ex, Ey) tuples of (nx, ny) arrays indexed [i, j]."""
    o = options.to_c()
    g = np.asarray(grid, np.float64)
    cm = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).T)  # [i, j] -> column-major memory
    Ls = [cm(a) for a in L]; Rs = [cm(a) for a in R]; Ms = [cm(a) for a in (M if M is not None else L)]
    out = np.empty(3)
    lib().oo_interpolate(C.byref(o), _dp(g), float(x), float(y), *[_dp(a) for a in Ls], *[_dp(a) for a in Ms],
                         *[_dp(a) for a in Rs], int(M is not None), float(param), _dp(out))
    return tuple(out)


def luminosity(options: OracleOptions, x1, y1, x2, y2, klum):
    o = options.to_c()
    nx, ny = options.luminosity_grid or options.grid
    q1 = np.empty((nx + 1) * (ny + 1)); q2 = np.empty_like(q1)
    a = [np.ascontiguousarray(v, np.float64) for v in (x1, y1, x2, y2)]
    lum = lib().oo_luminosity(C.byref(o), _dp(a[0]), _dp(a[1]), a[0].size, _dp(a[2]), _dp(a[3]), a[2].size,
                              float(klum), _dp(q1), _dp(q2))
    f = lambda q: q.reshape(ny + 1, nx + 1).T.copy()
    return lum, f(q1), f(q2)


def as_oo_elements(elems):
    """Copies C element structs of the same layout (the product's octo_element) into oo_element."""
    arr = (OOElement * max(len(elems), 1))()
    for k, e in enumerate(elems):
        C.memmove(C.byref(arr[k]), C.byref(e), C.sizeof(OOElement))
    return arr


def track_line(elems, beam, turn=0, turns=1, seed=0, rng_method=1):
    """oo_track_line on a (6, n) float64 array (copied); elems: octo_element / oo_element structs."""
    b = np.ascontiguousarray(beam, dtype=np.float64).copy()
    arr = as_oo_elements(list(elems))
    lib().oo_track_line(arr, len(elems), int(turn), int(turns), C.c_uint64(seed), int(rng_method),
                        *[_dp(b[k]) for k in range(6)], b.shape[1])
    return b


def octopus_normal(seed, rng_method, turn, rng_id, particle, component):
    return lib().oo_octopus_normal(seed, rng_method, turn, rng_id, particle, component)


def moment_row(beam, moments, turn, mask_lost=False):
    """_moment_observer_row (src/tasks/BeamObservers.jl:1013-1040, 1254-1271) on a (6, n) float64 array:
    [turn, moments...]; order 1 the mean of its coordinate, higher orders the central moment with term
    1.0 * prod_d (c_d - mean_d)^p_d, summed in particle order.  mask_lost: only particles whose six
    coordinates are finite count; a beam without them gives NaN moments."""
    b = np.asarray(beam, dtype=np.float64)
    if mask_lost:
        b = b[:, np.all(np.isfinite(b), axis=0)]
    n = b.shape[1]
    row = [float(turn)]
    if n == 0:
        return np.array(row + [np.nan] * len(moments))
    means = [_seq_sum(b[d]) / n for d in range(6)]
    for m in moments:
        if sum(m) == 1:
            row.append(means[m.index(1)])
            continue
        term = np.ones(n)
        for d in range(6):
            if m[d]:
                dv = b[d] - means[d]
                t = dv.copy()
                for _ in range(1, m[d]):
                    t = t * dv
                term = term * t
        row.append(_seq_sum(term) / n)
    return np.array(row)


def _seq_sum(v):
    """Sequential left-to-right sum (the reference's CPU loop)."""
    s = 0.0
    for a in np.asarray(v, dtype=np.float64).tolist():
        s += a
    return s


def gaussian_collide(options: "OracleOptions", beam1: np.ndarray, beam2: np.ndarray, p1, p2, min_sigma=0.0,
                     gaussian_when_luminosity=2, ignore_centroid1=False, ignore_centroid2=False,
                     virtual_drift="hirata", include_sigma_xy=False) -> float:
    """collide!(::GaussianPoissonSolver, ...) (src/tasks/strongstrong/gaussian.jl) in place on (6, n) float64
    beams; options gives the slicings, kbb / luminosity-scale overrides and longitudinal_kick."""
    P = C.POINTER(C.c_double)
    a1 = (P * 6)(*[_dp(beam1[k]) for k in range(6)])
    a2 = (P * 6)(*[_dp(beam2[k]) for k in range(6)])
    copt = options.to_c()
    lum = C.c_double(np.nan)
    rc = lib().oo_gaussian_collide(C.byref(copt), float(min_sigma), int(gaussian_when_luminosity),
                                   int(bool(ignore_centroid1)), int(bool(ignore_centroid2)),
                                   {"hirata": 0, "chromatic": 1, "exact": 2}[virtual_drift], int(bool(include_sigma_xy)),
                                   a1, beam1.shape[1], a2,
                                   beam2.shape[1], C.byref(p1), C.byref(p2), C.byref(lum))
    if rc != OK:
        raise OracleErrorPy(rc, lib().oo_gaussian_last_error().decode())
    return lum.value


def be_near_round_L(kbb, v, eta, x, y):
    out = (C.c_double * 5)()
    lib().oo_be_near_round_L(kbb, v, eta, x, y, out)
    return tuple(out)


def be_principal_L(kbb, s1, s2, x, y):
    out = (C.c_double * 5)()
    lib().oo_be_principal_L(kbb, s1, s2, x, y, out)
    return tuple(out)


def be_elliptic(s1, s2, x, y):
    out = (C.c_double * 2)()
    lib().oo_be_elliptic(s1, s2, x, y, out)
    return tuple(out)
