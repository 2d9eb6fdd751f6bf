"""ctypes binding of libocto_b200.so (include/octo_b200.h).

The library is built in-tree (``octopus.jl_b200/build/libocto_b200.so``) by
``octopus.jl_b200/build.py``.  Loading fails loudly when it is missing: there is no
CPU fallback for the collision.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "build", "libocto_b200.so")

OCTO_OK, OCTO_ERR_NONFINITE, OCTO_ERR_UNSUPPORTED, OCTO_ERR_EXTENT, OCTO_ERR_ARG, OCTO_ERR_CUDA, OCTO_ERR_TIMEOUT = range(7)

ERROR_NAMES = {
    OCTO_ERR_NONFINITE: "NONFINITE", OCTO_ERR_UNSUPPORTED: "UNSUPPORTED", OCTO_ERR_EXTENT: "EXTENT",
    OCTO_ERR_ARG: "ARG", OCTO_ERR_CUDA: "CUDA", OCTO_ERR_TIMEOUT: "TIMEOUT",
}

# Every symbol include/octo_b200.h declares.
EXPORTS = (
    "octo_create", "octo_destroy", "octo_pic_collide", "octo_green_cache_stats",
    "octo_pair_luminosity_trace", "octo_linear6d", "octo_beam_gaussian", "octo_last_error",
    "octo_normal_quantile", "octo_erfinv", "octo_version", "octo_set_timing", "octo_timing_report",
    "octo_beam_gaussian_noalloc", "octo_pic_collide_batch", "octo_set_timing_phases", "octo_pic_autotune",
    "octo_track_line", "octo_beam_moments", "octo_capture_charge_plane", "octo_captured_charge_plane",
    "octo_gemm_bf16", "octo_cnn_create", "octo_cnn_destroy", "octo_cnn_num_params", "octo_cnn_get_params",
    "octo_cnn_set_params", "octo_cnn_forward", "octo_cnn_train_step", "octo_set_field_correction",
    "octo_field_correction_report", "octo_set_particle_order", "octo_set_collide_graph", "octo_collide_graph_stats",
)

PHASES = ("slicing", "bounds", "plan", "green", "luminosity", "deposit", "fft", "field", "kick", "unsort", "node")


class OctoBeam(C.Structure):
    _fields_ = [("n", C.c_int64), ("dtype", C.c_int32), ("reserved", C.c_int32),
                ("x", C.c_void_p), ("px", C.c_void_p), ("y", C.c_void_p),
                ("py", C.c_void_p), ("z", C.c_void_p), ("pz", C.c_void_p)]


# Line elements (OCTO_ELEM_* kinds of include/octo_b200.h).
ELEM_LINEAR6D, ELEM_THIN_CRAB_CAVITY, ELEM_LORENTZ_BOOST, ELEM_REV_LORENTZ_BOOST, ELEM_CHROMATICITY_KICK, \
    ELEM_LUMPED_RAD, ELEM_CRAB_DISPERSION, ELEM_MOMENTUM_DISPERSION, ELEM_XY_COUPLING = range(1, 10)
RAD_RADIATION, RAD_DAMPING, RAD_DIFFUSION = range(3)
RNG_PHILOX, RNG_SPLITMIX = 1, 2
CRAB_MAX_HARMONICS = 8
MOMENTS_MAX = 256
LINE_MAX_ELEMENTS = 32


class OctoElement(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nharm", C.c_int32), ("mode", C.c_int32), ("is_damping", C.c_int32),
                ("is_excitation", C.c_int32), ("reserved", C.c_int32), ("rng_id", C.c_uint64),
                ("p", C.c_double * 40)]


class OctoBeamParams(C.Structure):
    _fields_ = [("charge", C.c_double), ("mc2", C.c_double), ("E0", C.c_double),
                ("r0", C.c_double), ("npart", C.c_double)]


class OctoPicOptions(C.Structure):
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
        ("precision", C.c_int32),
        ("gaussian", C.c_int32),
        ("margin_sigma", C.c_double),
        ("neutralize", C.c_int32),
        ("solver", C.c_int32), ("gaussian_when_luminosity", C.c_int32),
        ("ignore_centroid1", C.c_int32), ("ignore_centroid2", C.c_int32),
        ("virtual_drift", C.c_int32), ("include_sigma_xy", C.c_int32),
        ("min_sigma", C.c_double),
        ("resolution1", C.c_int32), ("resolution2", C.c_int32),
        ("coupling_tol", C.c_double),
    ]


SOLVER_PIC, SOLVER_SOFT_GAUSSIAN = 0, 1


class OctoCollideReport(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("role", C.c_int32), ("pair_i", C.c_int32), ("pair_j", C.c_int32),
        ("direction", C.c_int32), ("n_batches", C.c_int32), ("turn", C.c_int64), ("first_index", C.c_int64),
        ("dropped", C.c_int64), ("green_hits", C.c_int64), ("green_misses", C.c_int64),
        ("green_rebuilds", C.c_int64), ("kernel_launches", C.c_int64), ("replayed", C.c_int32), ("pad", C.c_int32),
    ]


class OctoGemmDesc(C.Structure):
    _fields_ = [("M", C.c_int32), ("N", C.c_int32), ("K", C.c_int32), ("a_mode", C.c_int32), ("H", C.c_int32),
                ("W", C.c_int32), ("C", C.c_int32), ("splits", C.c_int32), ("relu", C.c_int32), ("pad", C.c_int32),
                ("A", C.c_void_p), ("lda", C.c_int64), ("B", C.c_void_p), ("ldb", C.c_int64),
                ("out", C.c_void_p), ("ldc", C.c_int64), ("bias", C.c_void_p), ("out_bf16", C.c_void_p),
                ("ldo", C.c_int64)]


_lib = None


def lib():
    """Load libocto_b200.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libocto_b200.so not found at {LIB_PATH}; build it with `python octopus.jl_b200/build.py` "
            "(the collision has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, d, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_uint64
    P = C.POINTER
    L.octo_create.restype = vp
    L.octo_create.argtypes = [i32, P(OctoPicOptions)]
    L.octo_destroy.restype = None
    L.octo_destroy.argtypes = [vp]
    L.octo_pic_collide.restype = i32
    L.octo_pic_collide.argtypes = [vp, P(OctoBeam), P(OctoBeam), P(OctoBeamParams), P(OctoBeamParams), i64, i32,
                                   P(d), P(OctoCollideReport), vp]
    L.octo_pic_collide_batch.restype = i32
    L.octo_pic_collide_batch.argtypes = [i32, P(vp), P(P(OctoBeam)), P(P(OctoBeam)), P(P(OctoBeamParams)),
                                         P(P(OctoBeamParams)), i64, i32, P(d), P(OctoCollideReport), P(i32), P(vp)]
    L.octo_pic_autotune.restype = i32
    L.octo_pic_autotune.argtypes = [vp, P(OctoBeam), P(OctoBeam), P(OctoBeamParams), P(OctoBeamParams), i32, P(i32), vp]
    L.octo_green_cache_stats.restype = i32
    L.octo_green_cache_stats.argtypes = [vp, P(i64), P(i64), P(i64)]
    L.octo_pair_luminosity_trace.restype = i64
    L.octo_pair_luminosity_trace.argtypes = [vp, P(i32), P(i32), P(d), i64]
    L.octo_beam_moments.restype = i32
    L.octo_beam_moments.argtypes = [vp, P(OctoBeam), P(i32), i32, i32, i64, vp, vp]
    L.octo_track_line.restype = i32
    L.octo_track_line.argtypes = [vp, P(OctoBeam), P(OctoElement), i32, i64, i32, u64, i32, vp]
    L.octo_linear6d.restype = i32
    L.octo_linear6d.argtypes = [vp, P(OctoBeam), P(d), i32, vp]
    L.octo_beam_gaussian.restype = i32
    L.octo_beam_gaussian.argtypes = [vp, P(OctoBeam), u64, u64, P(d), P(d), P(d), d, vp]
    L.octo_last_error.restype = i32
    L.octo_last_error.argtypes = [vp, C.c_char_p, i64]
    L.octo_normal_quantile.restype = d
    L.octo_normal_quantile.argtypes = [i32, i32]
    L.octo_erfinv.restype = d
    L.octo_erfinv.argtypes = [d]
    L.octo_version.restype = i32
    L.octo_version.argtypes = []
    L.octo_beam_gaussian_noalloc.restype = i32
    L.octo_beam_gaussian_noalloc.argtypes = [i32, P(OctoBeam), u64, u64, P(d), P(d), P(d), d, vp, C.c_char_p, i64]
    L.octo_capture_charge_plane.restype = i32
    L.octo_capture_charge_plane.argtypes = [vp, i32, i32, i32, i32]
    L.octo_captured_charge_plane.restype = i32
    L.octo_captured_charge_plane.argtypes = [vp, P(i64), P(d), P(d), P(i32)]
    L.octo_gemm_bf16.restype = i32
    L.octo_gemm_bf16.argtypes = [i32, P(OctoGemmDesc), vp]
    L.octo_cnn_create.restype = vp
    L.octo_cnn_create.argtypes = [i32, i32, i32, i32, u64]
    L.octo_cnn_destroy.restype = None
    L.octo_cnn_destroy.argtypes = [vp]
    L.octo_cnn_num_params.restype = i64
    L.octo_cnn_num_params.argtypes = [vp]
    L.octo_cnn_get_params.restype = i32
    L.octo_cnn_get_params.argtypes = [vp, P(C.c_float), i64]
    L.octo_cnn_set_params.restype = i32
    L.octo_cnn_set_params.argtypes = [vp, P(C.c_float), i64]
    L.octo_cnn_forward.restype = i32
    L.octo_cnn_forward.argtypes = [vp, vp, i32, vp, vp]
    L.octo_cnn_train_step.restype = i32
    L.octo_cnn_train_step.argtypes = [vp, vp, vp, vp, i32, C.c_float, i32, P(d), P(C.c_float), vp]
    L.octo_set_field_correction.restype = i32
    L.octo_set_field_correction.argtypes = [vp, vp, C.c_float, C.c_float, i32]
    L.octo_field_correction_report.restype = i32
    L.octo_field_correction_report.argtypes = [vp, P(i32)]
    L.octo_set_particle_order.restype = i32
    L.octo_set_particle_order.argtypes = [vp, i32]
    L.octo_set_collide_graph.restype = i32
    L.octo_set_collide_graph.argtypes = [vp, i32]
    L.octo_collide_graph_stats.restype = i32
    L.octo_collide_graph_stats.argtypes = [vp, C.POINTER(C.c_int64)]
    L.octo_set_timing_phases.restype = i32
    L.octo_set_timing_phases.argtypes = [vp, C.c_uint32]
    L.octo_set_timing.restype = i32
    L.octo_set_timing.argtypes = [vp, i32]
    L.octo_timing_report.restype = i32
    L.octo_timing_report.argtypes = [vp, P(d), P(i64), P(d)]
    _lib = L
    return L


def last_error(ctx) -> str:
    buf = C.create_string_buffer(1024)
    lib().octo_last_error(ctx, buf, len(buf))
    return buf.value.decode(errors="replace")
