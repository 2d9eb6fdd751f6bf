"""octo_b200 -- B200-native backend for Octopus.jl's strong-strong PIC collision.

Host mirror of the reference API for this one path: ``PICPoissonSolver``,
``LongitudinalSlicing``, ``Beam``, ``collide`` (``collide!``), ``Linear6D``.  All
compute runs in libocto_b200.so (hand-written sm_100a kernels behind a C ABI).
"""
from ._lib import OCTO_OK, EXPORTS, lib  # noqa: F401
from .api import (CUDABackend, Context, CollisionError, Linear6D, StrongStrongRuntime,  # noqa: F401
                  TrackingContext, collide, collide_batch)
from .beam import EMASS_EV, ME0, PMASS_EV, RE, Beam, BeamParams  # noqa: F401
from .solver import ArgumentError, GaussianPICPoissonSolver, LongitudinalSlicing, PICPoissonSolver  # noqa: F401

__all__ = ["PICPoissonSolver", "GaussianPICPoissonSolver", "LongitudinalSlicing", "Beam", "BeamParams", "collide", "collide_batch", "Context",
           "StrongStrongRuntime", "TrackingContext", "CUDABackend", "Linear6D", "ArgumentError",
           "CollisionError", "RE", "ME0", "EMASS_EV", "PMASS_EV"]
