"""octo_b200 -- B200-native backend for Octopus.jl's strong-strong PIC collision.

Host mirror of the reference API for this one path: ``PICPoissonSolver``,
``LongitudinalSlicing``, ``Beam``, ``collide`` (``collide!``), ``Linear6D``, and the line elements
around the collision with ``track`` (``track!``).  All
compute runs in libocto_b200.so (hand-written sm_100a kernels behind a C ABI).
"""
from ._lib import OCTO_OK, EXPORTS, lib  # noqa: F401
from .api import (CUDABackend, Context, CollisionError, Linear6D, StrongStrongRuntime,  # noqa: F401
                  TrackingContext, collide, collide_batch, track, with_turn)
from .line import (ChromaticityKickSpec, CrabDispersionSpec, Linear6DSpec, LorentzBoostSpec,  # noqa: F401
                   LumpedRadSpec, MomentumDispersionSpec, RevLorentzBoostSpec, ThinCrabCavitySpec,
                   XYCouplingSpec, claim_rng_id, global_rng_method, global_rng_seed, next_rng_id,
                   reset_rng_id_counter, set_global_rng)
from .observers import MomentObserver, moment, moment_name, selected_moments  # noqa: F401
from .beam import EMASS_EV, ME0, PMASS_EV, RE, Beam, BeamParams  # noqa: F401
from .solver import (ArgumentError, GaussianPICPoissonSolver, GaussianPoissonSolver,  # noqa: F401
                     LongitudinalSlicing, PICPoissonSolver)

__all__ = ["PICPoissonSolver", "GaussianPICPoissonSolver", "LongitudinalSlicing", "Beam", "BeamParams", "collide", "collide_batch", "Context",
           "StrongStrongRuntime", "TrackingContext", "CUDABackend", "Linear6D", "ArgumentError",
           "CollisionError", "RE", "ME0", "EMASS_EV", "PMASS_EV", "track", "with_turn", "Linear6DSpec",
           "ThinCrabCavitySpec", "LorentzBoostSpec", "RevLorentzBoostSpec", "ChromaticityKickSpec",
           "LumpedRadSpec", "CrabDispersionSpec", "MomentumDispersionSpec", "XYCouplingSpec",
           "set_global_rng", "global_rng_seed", "global_rng_method", "next_rng_id", "claim_rng_id",
           "reset_rng_id_counter", "GaussianPoissonSolver", "MomentObserver", "moment", "moment_name", "selected_moments"]
