"""Device-resident beams: ``Beam`` holds the six SoA coordinates (Phase6DRep, Beam.jl:45-55)
as CUDA float64 tensors (or float32 for the precision form, the reference's Beam{CUDABackend, Float32})
and the ``BeamParams`` (Beam.jl:29-35)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import numpy as np
import torch

from . import _lib

# src/constants/Constants.jl:11-20
RE = 2.8179403205e-15
EMASS_EV = 0.51099895069e6
ME0 = EMASS_EV
PMASS_EV = 938.27208943e6

COORDS = ("x", "px", "y", "py", "z", "pz")


@dataclass
class BeamParams:
    charge: float = 0.0
    mc2: float = 0.0
    E0: float = 0.0
    r0: float = 0.0
    npart: float = 0.0

    def to_c(self) -> _lib.OctoBeamParams:
        return _lib.OctoBeamParams(self.charge, self.mc2, self.E0, self.r0, self.npart)


_DTYPE_CODE = {torch.float64: 0, torch.float32: 1}


class Beam:
    """A beam on one CUDA device: ``coords`` is a (6, n) float64 (plain form) or float32 (precision
    form) tensor, rows x, px, y, py, z, pz."""

    def __init__(self, coords: torch.Tensor, params: BeamParams):
        if coords.dim() != 2 or coords.shape[0] != 6:
            raise ValueError("coords must have shape (6, n)")
        if coords.dtype not in _DTYPE_CODE or not coords.is_cuda:
            raise ValueError("coords must be a CUDA float64 or float32 tensor")
        self.coords = coords.contiguous()
        self.params = params

    @property
    def dtype(self) -> torch.dtype:
        return self.coords.dtype

    def astype(self, dtype: torch.dtype) -> "Beam":
        """A copy of the beam with coordinates of another element type (rounded once)."""
        return Beam(self.coords.to(dtype), BeamParams(**vars(self.params)))

    @property
    def n(self) -> int:
        return int(self.coords.shape[1])

    def __len__(self):
        return self.n

    @classmethod
    def from_numpy(cls, arr: np.ndarray, params: BeamParams, device="cuda:0", dtype=torch.float64) -> "Beam":
        np_dtype = np.float64 if dtype == torch.float64 else np.float32
        return cls(torch.from_numpy(np.ascontiguousarray(arr, dtype=np_dtype)).to(device), params)

    def numpy(self) -> np.ndarray:
        return self.coords.cpu().numpy()

    def to_c(self) -> _lib.OctoBeam:
        b = _lib.OctoBeam()
        b.n = self.n
        b.dtype = _DTYPE_CODE[self.coords.dtype]
        for k, name in enumerate(COORDS):
            setattr(b, name, C.c_void_p(self.coords[k].data_ptr()))
        return b

    @classmethod
    def gaussian(cls, n: int, *, beta: Sequence[float], alpha: Sequence[float] = (0.0, 0.0, 0.0),
                 sigma: Sequence[float], cutoff: float = 5.0, rng_id: int, seed: int = 123456789,
                 charge=0.0, mc2=0.0, E0=0.0, r0=None, npart=None, device="cuda:0",
                 dtype=torch.float64) -> "Beam":
        """Seeded counter-RNG Gaussian beam, built on the device like
        Beam(n, backend, Float64; beta, alpha, sigma, cutoff, rng_id, charge, mc2, E0, r0, npart).
        dtype=torch.float32 builds the float64 beam and rounds it once to float32."""
        from .api import _scratch_ctx
        dev = torch.device(device)
        coords = torch.empty((6, int(n)), dtype=torch.float64, device=dev)
        params = BeamParams(charge, mc2, E0, (RE * ME0 / mc2 if mc2 else 0.0) if r0 is None else r0,
                            float(n) if npart is None else npart)
        beam = cls(coords, params)
        b = beam.to_c()
        d3 = C.c_double * 3
        ctx = _scratch_ctx(dev.index or 0)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = _lib.lib().octo_beam_gaussian(ctx, C.byref(b), int(seed), int(rng_id), d3(*beta), d3(*alpha),
                                           d3(*sigma), float(cutoff), C.c_void_p(stream))
        if rc != _lib.OCTO_OK:
            raise RuntimeError(_lib.last_error(ctx))
        return beam if dtype == torch.float64 else beam.astype(dtype)
