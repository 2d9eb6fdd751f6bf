"""Keyword mirror of the reference's solver and slicing configuration.

``PICPoissonSolver`` follows interface.jl:1384-1507 (keywords, defaults and eager
validation) and ``LongitudinalSlicing`` interface.jl:816-831.  Invalid values raise
``ArgumentError`` with the reference's wording; combinations this GPU backend does not
implement are rejected when the solver is bound to the backend (the reference's
``_require_cuda_pic_options``, pic_cpu.jl:730-777), never silently ignored.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

from . import _lib


class ArgumentError(ValueError):
    """Raised where the reference raises Julia's ArgumentError."""


_SLICING_METHODS = ("equal_area", "equal_count", "equal_width", "equal_spaced", "normal_quantile", "gaussian",
                    "Gaussian", "specified")


# OCTO_SLICING_* codes (the aliases of interface.jl:793-797 map to their methods)
_METHOD_CODE = {"normal_quantile": 0, "gaussian": 0, "Gaussian": 0, "specified": 1, "equal_area": 2,
                "equal_count": 3, "equal_width": 4, "equal_spaced": 4}


@dataclass(frozen=True)
class LongitudinalSlicing:
    """LongitudinalSlicing(; nslices=1, method=:equal_area, resolution=100, center_position=:centroid,
    positions=Float64[]) -- interface.jl:816-831."""
    nslices: int = 1
    method: str = "equal_area"
    resolution: int = 100
    center_position: str = "centroid"
    positions: Tuple[float, ...] = ()

    def __post_init__(self):
        if self.nslices <= 0:
            raise ArgumentError("nslices must be positive")
        if self.resolution <= 0:
            raise ArgumentError("slicing resolution must be positive")
        if self.method not in _SLICING_METHODS:
            raise ArgumentError(f"unsupported longitudinal slicing method :{self.method}")
        if self.center_position not in ("centroid", "midpoint"):
            raise ArgumentError("center_position must be :centroid or :midpoint")
        object.__setattr__(self, "positions", tuple(float(p) for p in self.positions))
        if self.method == "specified" and len(self.positions) != self.nslices - 1:
            raise ArgumentError("specified slicing requires nslices-1 internal positions")


@dataclass(frozen=True)
class PICPoissonSolver:
    """PICPoissonSolver(; ...) -- the keyword surface of interface.jl:1384-1411."""
    kbb1: Optional[float] = None
    kbb2: Optional[float] = None
    luminosity_scale: Optional[float] = None
    grid: Tuple[int, int] = (128, 128)
    deposit_method: str = "CIC"
    green_type: str = "integrated"
    green_cache: str = "slice_pair"
    field_derivative: str = "second"
    slice_interpolation: str = "linear"
    interaction_grid: str = "slice_pair"
    grid_extent: str = "extrema"
    grid_extent_sigma: float = 6.0
    min_transverse_extent: Tuple[float, float] = (0.0, 0.0)
    grid_quantize: float = 0.0
    slice_pair_green_min_ratio: float = 0.50
    slice_pair_green_growth: float = 0.25
    longitudinal_kick: bool = True
    batch_mode: str = "wavefront"
    cuda_async: bool = True
    cuda_batch_fft: bool = True
    cuda_wavefront_fft: bool = True
    cuda_indexed_wavefront: bool = True
    luminosity_grid: Optional[Tuple[int, int]] = None
    luminosity_deposit_method: Optional[str] = None
    luminosity_schedule: Optional[object] = None
    slicing: LongitudinalSlicing = field(default_factory=LongitudinalSlicing)
    slicing1: Optional[LongitudinalSlicing] = None
    slicing2: Optional[LongitudinalSlicing] = None

    def __post_init__(self):
        if not (0.0 < self.slice_pair_green_min_ratio <= 1.0):
            raise ArgumentError(
                f"slice_pair_green_min_ratio must be in (0, 1]; got {self.slice_pair_green_min_ratio}.")
        if not (self.slice_pair_green_growth >= 0.0):
            raise ArgumentError(f"slice_pair_green_growth must be non-negative; got {self.slice_pair_green_growth}.")
        g = (int(self.grid[0]), int(self.grid[1]))
        if min(g) < 5:
            raise ArgumentError(f"PICPoissonSolver grid dimensions must both be at least 5; got {self.grid}.")
        object.__setattr__(self, "grid", g)
        _choice("deposit_method", self.deposit_method, ("CIC", "TSC"))
        _choice("green_type", self.green_type, ("integrated", "standard", "lattice"))
        _choice("green_cache", self.green_cache, ("none", "slice_pair"))
        _choice("field_derivative", self.field_derivative, ("second", "fourth"))
        _choice("slice_interpolation", self.slice_interpolation, ("linear", "quadratic"))
        _choice("grid_extent", self.grid_extent, ("extrema", "sigma"))
        if not self.grid_extent_sigma > 0:
            raise ArgumentError(f"grid_extent_sigma must be positive; got {self.grid_extent_sigma}.")
        mte = self.min_transverse_extent
        if isinstance(mte, (int, float)):
            mte = (float(mte), float(mte))
        mte = (float(mte[0]), float(mte[1]))
        if not all(v >= 0 and v == v and v != float("inf") for v in mte):
            raise ArgumentError(f"min_transverse_extent must be finite and non-negative; got {self.min_transverse_extent}.")
        object.__setattr__(self, "min_transverse_extent", mte)
        if not self.grid_quantize >= 0:
            raise ArgumentError(f"grid_quantize must be non-negative (0 disables); got {self.grid_quantize}.")
        _choice("interaction_grid", self.interaction_grid, ("slice_pair", "source_slice", "node"))
        if self.interaction_grid != "slice_pair" and self.grid_extent != "extrema":
            raise ArgumentError(
                f"grid_extent = :{self.grid_extent} is not implemented for interaction_grid = "
                f":{self.interaction_grid}: that mode sizes its mesh from the union/per-node extrema of its own "
                "particle sets and applies no extent estimator, so a non-default value would be silently ignored. "
                "Use interaction_grid = :slice_pair, or set grid_extent = :extrema.")
        _choice("batch_mode", self.batch_mode, ("sequential", "wavefront"))
        if self.luminosity_grid is not None:
            lg = (int(self.luminosity_grid[0]), int(self.luminosity_grid[1]))
            if min(lg) < 3:
                raise ArgumentError(f"luminosity_grid dimensions must both be at least 3; got {self.luminosity_grid}.")
            object.__setattr__(self, "luminosity_grid", lg)
        if self.luminosity_deposit_method not in (None, "CIC", "TSC"):
            raise ArgumentError("luminosity_deposit_method must be nothing, :CIC, or :TSC; got "
                                f":{self.luminosity_deposit_method}.")
        if self.interaction_grid == "node" and self.slice_interpolation != "linear":
            raise ArgumentError(
                f"slice_interpolation = :{self.slice_interpolation} is not implemented for interaction_grid = :node: "
                "the node-plane path applies its own interpolation. Use interaction_grid = :slice_pair for "
                ":quadratic, or slice_interpolation = :linear.")

    @property
    def resolved_slicing1(self) -> LongitudinalSlicing:
        return self.slicing1 if self.slicing1 is not None else self.slicing

    @property
    def resolved_slicing2(self) -> LongitudinalSlicing:
        return self.slicing2 if self.slicing2 is not None else self.slicing

    def to_c(self) -> "_lib.OctoPicOptions":
        """Bind to the GPU backend: the POD options, rejecting what this backend does not implement."""
        _require_gpu_options(self)
        o = _lib.OctoPicOptions()
        o.nx, o.ny = self.grid
        o.deposit_method = 0 if self.deposit_method == "CIC" else 1
        o.lum_deposit_method = -1 if self.luminosity_deposit_method is None else \
            (0 if self.luminosity_deposit_method == "CIC" else 1)
        lg = self.luminosity_grid or (0, 0)
        o.lum_nx, o.lum_ny = lg
        o.green_type = {"integrated": 0, "standard": 1}[self.green_type]
        o.green_cache = {"none": 0, "slice_pair": 1}[self.green_cache]
        o.field_derivative = 2 if self.field_derivative == "second" else 4
        o.slice_interpolation = 0 if self.slice_interpolation == "linear" else 1
        o.interaction_grid = {"slice_pair": 0, "source_slice": 1, "node": 2}[self.interaction_grid]
        o.grid_extent = 0 if self.grid_extent == "extrema" else 1
        o.grid_extent_sigma = float(self.grid_extent_sigma)
        o.min_extent_x, o.min_extent_y = self.min_transverse_extent
        o.grid_quantize = float(self.grid_quantize)
        o.green_min_ratio = float(self.slice_pair_green_min_ratio)
        o.green_growth = float(self.slice_pair_green_growth)
        o.longitudinal_kick = int(bool(self.longitudinal_kick))
        keep = []
        for k, s in ((1, self.resolved_slicing1), (2, self.resolved_slicing2)):
            setattr(o, f"slicing_method{k}", _METHOD_CODE[s.method])
            setattr(o, f"resolution{k}", int(s.resolution))
            setattr(o, f"nslices{k}", int(s.nslices))
            setattr(o, f"center_position{k}", 0 if s.center_position == "centroid" else 1)
            if s.method == "specified" and s.positions:
                arr = (C.c_double * len(s.positions))(*s.positions)
                keep.append(arr)
                setattr(o, f"positions{k}", C.cast(arr, C.POINTER(C.c_double)))
        o.has_kbb1 = int(self.kbb1 is not None)
        o.has_kbb2 = int(self.kbb2 is not None)
        o.has_lum_scale = int(self.luminosity_scale is not None)
        o.kbb1 = float(self.kbb1 or 0.0)
        o.kbb2 = float(self.kbb2 or 0.0)
        o.lum_scale = float(self.luminosity_scale or 0.0)
        o.precision = 0
        o.coupling_tol = math.inf  # read by the hybrid only
        o._keep = keep  # positions arrays must outlive octo_create
        return o


def _choice(name, value, allowed):
    if value not in allowed:
        opts = ", ".join(":" + a for a in allowed)
        raise ArgumentError(f"{name} must be one of {opts}; got :{value}.")


def _require_gpu_options(s: PICPoissonSolver):
    """The GPU backend's route checks (the reference CUDA backend's, pic_cpu.jl:730-777)."""
    if s.green_type == "lattice":
        raise ArgumentError("green_type = :lattice (an experimental CPU study kernel) is not implemented by the GPU "
                            "PIC backend; use :integrated or :standard.")
    for k, sl in ((1, s.resolved_slicing1), (2, s.resolved_slicing2)):
        if sl.method == "equal_area" and sl.nslices * sl.resolution > 16384:
            raise ArgumentError("the GPU PIC backend's :equal_area histogram holds at most 16384 bins "
                                "(nslices * resolution)")
        if sl.nslices > 64:
            raise ArgumentError("the GPU PIC backend supports at most 64 slices per beam")
    def fft_ok(n):
        m = n // 3 if n % 3 == 0 else n
        return m & (m - 1) == 0 and 8 <= n <= 512
    if not all(fft_ok(n) for n in s.grid) or s.grid[1] % 8:
        raise ArgumentError("the GPU PIC backend's FFT needs grid dimensions of the form 2^a or 3*2^a in 8..512, "
                            f"ny a multiple of 8; got {s.grid}")


class GaussianPICPoissonSolver:
    """GaussianPICPoissonSolver(; margin_sigma=5.0, neutralize=true, coupling_tol=Inf, kwargs...)
    (gaussian_pic.jl:87-112): a PICPoissonSolver built from the remaining keywords, whose slice-pair
    interactions subtract the drifted reference Gaussian of each source slice before the solve and add its
    Bassetti-Erskine kick back analytically.  The PIC options the hybrid does not read must keep their
    defaults (gaussian_pic.jl:162-164).  A finite coupling_tol subtracts the tilted (coupled) reference Gaussian of
    slices whose drifted |r_xy| exceeds it and adds the rotated Bassetti-Erskine kick back (gaussian_pic.jl:240-372,
    837-854); Inf, the default, always subtracts the separable Gaussian."""

    def __init__(self, margin_sigma: float = 5.0, neutralize: bool = True, coupling_tol: float = math.inf,
                 **kwargs):
        pic = kwargs.pop("pic", None) or PICPoissonSolver(**kwargs)
        if not float(margin_sigma) >= 0.0:
            raise ArgumentError(f"margin_sigma must be non-negative; got {margin_sigma}.")
        if not float(coupling_tol) >= 0.0:
            raise ArgumentError(f"coupling_tol must be non-negative; got {coupling_tol}.")
        self.pic = pic
        self.margin_sigma = float(margin_sigma)
        self.neutralize = bool(neutralize)
        self.coupling_tol = float(coupling_tol)

    def __getattr__(self, name):  # the embedded PIC solver's options
        if name == "pic":
            raise AttributeError(name)
        return getattr(self.pic, name)

    def _key(self):
        return (self.pic, self.margin_sigma, self.neutralize, self.coupling_tol)

    def __eq__(self, other):
        return isinstance(other, GaussianPICPoissonSolver) and self._key() == other._key()

    def __hash__(self):
        return hash(("GaussianPICPoissonSolver",) + self._key())

    def replace(self, **pic_changes) -> "GaussianPICPoissonSolver":
        from dataclasses import replace
        return GaussianPICPoissonSolver(self.margin_sigma, self.neutralize, self.coupling_tol,
                                        pic=replace(self.pic, **pic_changes))

    def to_c(self) -> "_lib.OctoPicOptions":
        p = self.pic
        if p.slice_interpolation != "linear" or p.interaction_grid != "slice_pair" or p.grid_extent != "extrema":
            raise ArgumentError(
                "GaussianPICPoissonSolver does not read slice_interpolation, interaction_grid or grid_extent: it "
                "interpolates linearly on its own :slice_pair box (gaussian_pic.jl:162-164); keep their defaults.")
        o = p.to_c()
        o.gaussian = 1
        o.margin_sigma = self.margin_sigma
        o.neutralize = int(self.neutralize)
        o.coupling_tol = self.coupling_tol
        return o


@dataclass(frozen=True)
class GaussianPoissonSolver:
    """GaussianPoissonSolver(; ...) -- the soft-Gaussian strong-strong solver (interface.jl:949-1020,
    src/tasks/strongstrong/gaussian.jl): each slice pair kicks each slice with the Bassetti-Erskine field of a
    Gaussian carrying the other slice's transverse moments, uncoupled or with the full transverse covariance
    (include_sigma_xy), with the :hirata, :chromatic and :exact virtual drifts, on float64 or float32 beams (the
    latter stored in float and computed in FP64, as the reference promotes them against its Float64 moments)."""
    kbb1: Optional[float] = None
    kbb2: Optional[float] = None
    luminosity_scale: Optional[float] = None
    slicing: LongitudinalSlicing = field(default_factory=LongitudinalSlicing)
    slicing1: Optional[LongitudinalSlicing] = None
    slicing2: Optional[LongitudinalSlicing] = None
    min_sigma: float = 0.0
    gaussian_when_luminosity: int = 2
    ignore_centroid1: bool = False
    ignore_centroid2: bool = False
    longitudinal_kick: bool = True
    virtual_drift: str = "hirata"
    include_sigma_xy: bool = False
    batch_mode: str = "wavefront"
    luminosity_schedule: Optional[object] = None

    def __post_init__(self):
        ms = float(self.min_sigma)
        if not (math.isfinite(ms) and ms >= 0):
            raise ArgumentError(f"min_sigma must be finite and nonnegative; got {self.min_sigma}.")
        if self.gaussian_when_luminosity not in (1, 2):
            raise ArgumentError("gaussian_when_luminosity must be 1 or 2")
        _choice("batch_mode", self.batch_mode, ("sequential", "wavefront"))
        _choice("virtual_drift", self.virtual_drift, ("hirata", "chromatic", "exact"))

    @property
    def resolved_slicing1(self) -> LongitudinalSlicing:
        return self.slicing1 if self.slicing1 is not None else self.slicing

    @property
    def resolved_slicing2(self) -> LongitudinalSlicing:
        return self.slicing2 if self.slicing2 is not None else self.slicing

    def to_c(self) -> "_lib.OctoPicOptions":
        # the PIC fields are unused by this solver; a valid small grid keeps the context's setup cheap
        o = PICPoissonSolver(grid=(8, 8), kbb1=self.kbb1, kbb2=self.kbb2, luminosity_scale=self.luminosity_scale,
                             slicing=self.slicing, slicing1=self.slicing1, slicing2=self.slicing2,
                             longitudinal_kick=self.longitudinal_kick).to_c()
        o.solver = _lib.SOLVER_SOFT_GAUSSIAN
        o.gaussian_when_luminosity = int(self.gaussian_when_luminosity)
        o.ignore_centroid1 = int(bool(self.ignore_centroid1))
        o.ignore_centroid2 = int(bool(self.ignore_centroid2))
        o.virtual_drift = {"hirata": 0, "chromatic": 1, "exact": 2}[self.virtual_drift]
        o.include_sigma_xy = int(bool(self.include_sigma_xy))
        o.min_sigma = float(self.min_sigma)
        return o
