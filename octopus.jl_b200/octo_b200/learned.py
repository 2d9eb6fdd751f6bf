"""The learned field correction: a BF16 tensor-core CNN that restores fine-grid field quality to the coarse
Gaussian-subtracted hybrid solver (GaussianPICPoissonSolver, src/tasks/strongstrong/gaussian_pic.jl).  No
counterpart in the reference.

``FieldCorrectionNet`` wraps libocto_b200's network (octo_cnn_*): a 4-level U-Net of 3x3 convolutions, 32 base
channels, 641k parameters, whose convolutions, gradients and Adam update run on the GPU in the library's own
tcgen05 kernels.  Inputs are NHWC bf16 [batch, height, width, 8]; outputs fp32 [batch, height, width, 2].
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np
import torch

from . import _lib


class FieldCorrectionNet:
    def __init__(self, height: int = 48, width: int = 48, max_batch: int = 64, device: int = 0, seed: int = 1234):
        self.height, self.width, self.max_batch, self.device = int(height), int(width), int(max_batch), int(device)
        self._ptr = _lib.lib().octo_cnn_create(self.device, self.height, self.width, self.max_batch, int(seed))
        if not self._ptr:
            raise RuntimeError("octo_cnn_create failed (height and width must be multiples of 8, >= 16)")

    def close(self):
        if getattr(self, "_ptr", None):
            _lib.lib().octo_cnn_destroy(self._ptr)
            self._ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ptr(self):
        return self._ptr

    @property
    def num_params(self) -> int:
        return int(_lib.lib().octo_cnn_num_params(self._ptr))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.num_params, dtype=np.float32)
        rc = _lib.lib().octo_cnn_get_params(self._ptr, p.ctypes.data_as(C.POINTER(C.c_float)), p.size)
        if rc != _lib.OCTO_OK:
            raise RuntimeError(f"octo_cnn_get_params failed: {rc}")
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        rc = _lib.lib().octo_cnn_set_params(self._ptr, p.ctypes.data_as(C.POINTER(C.c_float)), p.size)
        if rc != _lib.OCTO_OK:
            raise RuntimeError(f"octo_cnn_set_params failed: {rc}")

    def _check(self, x: torch.Tensor):
        if x.dtype != torch.bfloat16 or not x.is_cuda or tuple(x.shape[1:]) != (self.height, self.width, 8):
            raise ValueError("input must be a CUDA bf16 tensor [batch, height, width, 8]")
        if not 1 <= x.shape[0] <= self.max_batch:
            raise ValueError("batch out of range")
        return x.contiguous()

    def forward(self, x: torch.Tensor, stream=None) -> torch.Tensor:
        x = self._check(x)
        out = torch.empty((x.shape[0], self.height, self.width, 2), dtype=torch.float32, device=x.device)
        st = (stream or torch.cuda.current_stream(x.device)).cuda_stream
        rc = _lib.lib().octo_cnn_forward(self._ptr, C.c_void_p(x.data_ptr()), int(x.shape[0]), C.c_void_p(out.data_ptr()),
                                         C.c_void_p(st))
        if rc != _lib.OCTO_OK:
            raise RuntimeError(f"octo_cnn_forward failed: {rc}")
        return out

    def train_step(self, x: torch.Tensor, target: torch.Tensor, mask: Optional[torch.Tensor] = None, lr: float = 1e-3,
                   update: bool = True, want_grads: bool = False, stream=None):
        """One forward + backward (+ Adam step when update); returns the loss (and the gradients)."""
        x = self._check(x)
        target = target.to(torch.float32).contiguous()
        mask = None if mask is None else mask.to(torch.float32).contiguous()
        loss = C.c_double(0.0)
        grads = np.empty(self.num_params, dtype=np.float32) if want_grads else None
        st = (stream or torch.cuda.current_stream(x.device)).cuda_stream
        rc = _lib.lib().octo_cnn_train_step(
            self._ptr, C.c_void_p(x.data_ptr()), C.c_void_p(target.data_ptr()),
            C.c_void_p(mask.data_ptr()) if mask is not None else None, int(x.shape[0]), float(lr), int(bool(update)),
            C.byref(loss), grads.ctypes.data_as(C.POINTER(C.c_float)) if want_grads else None, C.c_void_p(st))
        if rc != _lib.OCTO_OK:
            raise RuntimeError(f"octo_cnn_train_step failed: {rc}")
        return (loss.value, grads) if want_grads else loss.value


# ------------------------------------------------------------------------------------------------ training data
OUT_SCALE = 100.0  # the network's outputs are (dEx * hx, dEy * hy) of a unit charge times this
EDGE = 2           # nodes within this many of the mesh border are never sampled, so never corrected
KINDS = ("gaussian", "bigaussian", "tilted", "hollow")


def sample_density(kind: str, n: int, aspect: float, gen: torch.Generator, device) -> tuple:
    """A seeded transverse slice density of n macroparticles (x, y) in metres, sigma_y = 10 um and
    sigma_x = aspect * sigma_y: a Gaussian, a two-Gaussian mixture (random offset, sizes and weight), a
    Gaussian tilted by a random angle, or a hollow ring of 20 % radial spread."""
    sy = 1e-5
    sx = aspect * sy

    def u(*shape):
        return torch.rand(*shape, generator=gen, device=device, dtype=torch.float64)

    def g(*shape):
        return torch.randn(*shape, generator=gen, device=device, dtype=torch.float64)

    if kind == "gaussian":
        return sx * g(n), sy * g(n)
    if kind == "bigaussian":
        w2 = float(0.2 + 0.3 * u(1))
        n2 = int(n * w2)
        n1 = n - n2
        ox, oy = float(2 * u(1) - 1) * sx, float(2 * u(1) - 1) * sy
        fx, fy = float(0.3 + 0.7 * u(1)), float(0.3 + 0.7 * u(1))
        x = torch.cat([sx * g(n1), ox + fx * sx * g(n2)])
        y = torch.cat([sy * g(n1), oy + fy * sy * g(n2)])
        return x, y
    if kind == "tilted":
        th = float(0.3 * (2 * u(1) - 1)) / max(1.0, aspect ** 0.5)
        a, b = sx * g(n), sy * g(n)
        c, s = math.cos(th), math.sin(th)
        return c * a - s * b, s * a + c * b
    if kind == "hollow":
        r = 1.0 + 0.2 * g(n)
        phi = 2 * math.pi * u(n)
        return sx * r * torch.cos(phi), sy * r * torch.sin(phi)
    raise ValueError(kind)


COARSE = ("hybrid", "pic")  # the coarse solver the network corrects: the Gaussian-subtracted hybrid or plain PIC


def coarse_solver(kind: str, grid: int, **kw):
    """The coarse solver of a learned form: :slice_pair grids, :integrated Green function without the Green
    cache (every field mesh is its source mesh shifted by whole cells), linear slice interpolation."""
    from .solver import GaussianPICPoissonSolver, PICPoissonSolver
    kw = dict(kw, green_cache="none")
    if kind == "hybrid":
        return GaussianPICPoissonSolver(grid=(grid, grid), **kw)
    if kind == "pic":
        return PICPoissonSolver(grid=(grid, grid), **kw)
    raise ValueError(kind)


def _probe_solvers(grid: int, fine: int, coarse: str = "hybrid"):
    from .solver import LongitudinalSlicing, PICPoissonSolver
    common = dict(slicing=LongitudinalSlicing(nslices=1, method="normal_quantile"), kbb1=1.0, kbb2=1.0,
                  luminosity_scale=1.0)
    return coarse_solver(coarse, grid, **common), PICPoissonSolver(grid=(fine, fine), green_cache="none", **common)


class PairGenerator:
    """Training pairs from the GPU solvers themselves: for a slice density, the coarse hybrid's input (its
    charge grid, through the charge-plane capture) and the correction that brings the coarse hybrid's field to
    the plain fine-grid PIC field, on the coarse source mesh's nodes.  Both fields are read by probe particles
    (one collide of the density with a probe slice, kbb = 1, kicks each probe by twice the field of a unit
    total charge, as in diagnostics.field_error).  Two probes at the density's extreme corners fix the probe
    box, so the meshes of a first collide with only those two hold for the second with the node probes too,
    which sit at the field mesh's nodes inside that box; field node (i, j) is source node (i + sx, j + sy), the
    field mesh being the source mesh shifted by whole cells (no Green cache, the :integrated alignment)."""

    def __init__(self, grid: int = 48, fine: int = 128, device: int = 0, coarse: str = "hybrid"):
        from .api import Context
        self.grid, self.fine, self.device = grid, fine, device
        sh, sf = _probe_solvers(grid, fine, coarse)
        self.ctx_h = Context(sh, device)
        self.ctx_f = Context(sf, device)
        self.dev = torch.device(f"cuda:{device}")

    def close(self):
        self.ctx_h.close()
        self.ctx_f.close()

    def _beam(self, x, y):
        from .beam import Beam, BeamParams
        c = torch.zeros((6, x.numel()), dtype=torch.float64, device=self.dev)
        c[0], c[2] = x, y
        return Beam(c, BeamParams(1.0, 1.0, 1.0, 1.0, 1.0))

    def pair(self, x, y):
        """(input [H, W, 8] float32, target [H, W, 2], mask [H, W], fine field [H, W, 2] in output units, source
        mesh) for the density (x, y)."""
        n = self.grid
        lo_x, hi_x, lo_y, hi_y = (float(v) for v in (x.min(), x.max(), y.min(), y.max()))
        cx = torch.tensor([lo_x, hi_x], dtype=torch.float64, device=self.dev)
        cy = torch.tensor([lo_y, hi_y], dtype=torch.float64, device=self.dev)
        # pass 1: the meshes, with only the two corner probes
        self.ctx_h.capture_charge_plane(1, 1, 1, 0)
        self.ctx_h.collide(self._beam(x, y), self._beam(cx, cy), turn=1, compute_luminosity=False)
        q, mesh, fmesh, _ = self.ctx_h.captured_charge_plane(with_field_mesh=True)
        x0, y0, w, h = mesh
        hx, hy = w / (n - 1), h / (n - 1)
        sx, sy = int(round((fmesh[0] - x0) / hx)), int(round((fmesh[1] - y0) / hy))
        # the field mesh's nodes inside the corner box whose source node is an interior node
        i = torch.arange(n, device=self.dev)
        fxn, fyn = fmesh[0] + i.double() * hx, fmesh[1] + i.double() * hy
        okx = (fxn >= lo_x) & (fxn <= hi_x) & (i + sx >= EDGE) & (i + sx < n - EDGE)
        oky = (fyn >= lo_y) & (fyn <= hi_y) & (i + sy >= EDGE) & (i + sy < n - EDGE)
        ix, iy = i[okx], i[oky]
        gy, gx = torch.meshgrid(iy, ix, indexing="ij")
        gy, gx = gy.reshape(-1), gx.reshape(-1)
        px = torch.cat([fmesh[0] + gx.double() * hx, cx])
        py = torch.cat([fmesh[1] + gy.double() * hy, cy])
        # pass 2: the coarse hybrid's field at those nodes
        probes = self._beam(px, py)
        self.ctx_h.capture_charge_plane(1, 1, 1, 0)
        self.ctx_h.collide(self._beam(x, y), probes, turn=1, compute_luminosity=False)
        _, mesh2, fmesh2, _ = self.ctx_h.captured_charge_plane(with_field_mesh=True)
        tol = 1e-12 * max(abs(x0), abs(y0), w, h)
        if any(abs(a - b) > tol for a, b in zip(mesh2 + fmesh2, mesh + fmesh)):
            raise RuntimeError("the probe slice moved the meshes")
        eh = probes.coords[[1, 3], :-2] / 2.0
        # pass 3: the same probes through the plain fine-grid solver
        probes_f = self._beam(px, py)
        self.ctx_f.collide(self._beam(x, y), probes_f, turn=1, compute_luminosity=False)
        ef = probes_f.coords[[1, 3], :-2] / 2.0
        scale = torch.tensor([hx, hy], dtype=torch.float64, device=self.dev).view(2, 1) * OUT_SCALE
        tgt = torch.zeros((n, n, 2), dtype=torch.float32, device=self.dev)
        fin = torch.zeros((n, n, 2), dtype=torch.float32, device=self.dev)
        mask = torch.zeros((n, n), dtype=torch.float32, device=self.dev)
        rows, cols = gy + sy, gx + sx
        tgt[rows, cols] = ((ef - eh) * scale).T.to(torch.float32)
        fin[rows, cols] = (ef * scale).T.to(torch.float32)
        mask[rows, cols] = 1.0
        qt = torch.from_numpy(q.astype(np.float64)).to(self.dev)
        inp = torch.zeros((n, n, 8), dtype=torch.float32, device=self.dev)
        inp[..., 0] = (qt / qt.sum() * (n * n)).to(torch.float32)
        inp[..., 1] = math.log(hy / hx)
        return inp, tgt, mask, fin, mesh


def make_dataset(n_samples: int, seed: int, grid: int = 48, fine: int = 128, n_src: int = 200_000, device: int = 0,
                 kinds=KINDS, aspects=(1.0, 25.0), coarse: str = "hybrid"):
    """n_samples seeded pairs over the density kinds (round robin), aspect ratios log-uniform in `aspects`
    (one in five with the narrow axis along x).  Returns device tensors X (bf16 [N, H, W, 8]), T, M, F."""
    gen = PairGenerator(grid, fine, device, coarse)
    dev = gen.dev
    tg = torch.Generator(device=dev)
    tg.manual_seed(int(seed))
    X = torch.empty((n_samples, grid, grid, 8), dtype=torch.bfloat16, device=dev)
    T = torch.empty((n_samples, grid, grid, 2), dtype=torch.float32, device=dev)
    M = torch.empty((n_samples, grid, grid), dtype=torch.float32, device=dev)
    F = torch.empty((n_samples, grid, grid, 2), dtype=torch.float32, device=dev)
    la, lb = math.log(aspects[0]), math.log(aspects[1])
    try:
        for k in range(n_samples):
            kind = kinds[k % len(kinds)]
            aspect = math.exp(la + (lb - la) * float(torch.rand(1, generator=tg, device=dev)))
            x, y = sample_density(kind, n_src, aspect, tg, dev)
            if float(torch.rand(1, generator=tg, device=dev)) < 0.2:
                x, y = y, x
            inp, tgt, mask, fin, _ = gen.pair(x, y)
            X[k] = inp.to(torch.bfloat16)
            T[k], M[k], F[k] = tgt, mask, fin
    finally:
        gen.close()
    return X, T, M, F


def train(net: FieldCorrectionNet, X, T, M, steps: int, batch: int = 64, lr: float = 1e-3, seed: int = 0,
          log=None) -> list:
    """Mini-batch Adam on (X, T, M) with a cosine learning-rate decay to 5 % of lr; returns the losses."""
    g = torch.Generator(device=X.device)
    g.manual_seed(int(seed))
    n = X.shape[0]
    losses = []
    perm = torch.randperm(n, generator=g, device=X.device)
    pos = 0
    for step in range(steps):
        if pos + batch > n:
            perm = torch.randperm(n, generator=g, device=X.device)
            pos = 0
        idx = perm[pos:pos + batch]
        pos += batch
        rate = lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * step / max(1, steps))))
        losses.append(net.train_step(X[idx].contiguous(), T[idx].contiguous(), M[idx].contiguous(), lr=rate))
        if log and (step % 200 == 0 or step == steps - 1):
            log(f"step {step} loss {losses[-1]:.4e} lr {rate:.2e}")
    return losses


def evaluate(net: FieldCorrectionNet, X, T, M, F, batch: int = 64) -> dict:
    """RMS field error of the coarse solver alone ("hybrid" key, whichever coarse solver made the pairs) and
    with the correction ("learned"), against the fine plain-PIC field at the corrected nodes, each relative to
    the fine field's RMS (the same units throughout)."""
    num_h = num_c = den = 0.0
    for s in range(0, X.shape[0], batch):
        x = X[s:s + batch].contiguous()
        pred = net.forward(x)
        m = M[s:s + batch, ..., None]
        t = T[s:s + batch]
        num_h += float(((t * m) ** 2).sum())
        num_c += float((((t - pred) * m) ** 2).sum())
        den += float(((F[s:s + batch] * m) ** 2).sum())
    return {"hybrid": math.sqrt(num_h / den), "learned": math.sqrt(num_c / den)}


def default_weights_path(grid: int = 48, coarse: str = "hybrid") -> str:
    import os
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", f"field_correction_{coarse}_{grid}.npz")


def save_weights(net: FieldCorrectionNet, path: str, **meta) -> None:
    import os
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, params=net.get_params().astype(np.float32), height=net.height, width=net.width,
                        out_scale=OUT_SCALE, edge=EDGE, **{k: np.asarray(v) for k, v in meta.items()})


def load_net(path: str = None, max_batch: int = 64, device: int = 0, coarse: str = "hybrid") -> tuple:
    """A network with the saved parameters, and the file's metadata."""
    path = path or default_weights_path(coarse=coarse)
    d = np.load(path)
    net = FieldCorrectionNet(int(d["height"]), int(d["width"]), max_batch=max_batch, device=device)
    net.set_params(d["params"])
    return net, {k: d[k] for k in d.files if k != "params"}


# ------------------------------------------------------------------------------------------------ the learned form
class LearnedForm:
    """The learned form of the collide: a coarse-grid solver (the Gaussian-subtracted hybrid, or plain PIC; see
    coarse_solver) with the network's field correction, falling back to the plain solver for a collide in which
    any plane's error estimate (its largest correction) exceeded the tolerance -- the beams are restored from a
    copy taken before the collide and the plain solver runs instead."""

    def __init__(self, coarse, plain, net: FieldCorrectionNet, tolerance: float, device: int = 0,
                 dtype=torch.float64, out_scale: float = OUT_SCALE, edge: int = EDGE):
        from .api import Context
        self.net = net
        self.ctx = Context(coarse, device, dtype)
        self.fallback = Context(plain, device, dtype)
        rc = _lib.lib().octo_set_field_correction(self.ctx.ptr, net.ptr, float(out_scale), float(tolerance), int(edge))
        if rc != _lib.OCTO_OK:
            raise RuntimeError(_lib.last_error(self.ctx.ptr))
        self.fallbacks = 0
        self.collides = 0

    def close(self):
        if self.ctx is not None:
            _lib.lib().octo_set_field_correction(self.ctx.ptr, None, 1.0, 1.0, 0)
            self.ctx.close()
            self.fallback.close()
            self.ctx = None

    def planes_over_tolerance(self) -> int:
        v = C.c_int32(0)
        _lib.lib().octo_field_correction_report(self.ctx.ptr, C.byref(v))
        return int(v.value)

    def collide(self, beam1, beam2, turn: int = -1, compute_luminosity: bool = True, stream=None) -> float:
        saved = (beam1.coords.clone(), beam2.coords.clone())
        lum = self.ctx.collide(beam1, beam2, turn=turn, compute_luminosity=compute_luminosity, stream=stream)
        self.collides += 1
        if self.planes_over_tolerance() > 0:
            beam1.coords.copy_(saved[0])
            beam2.coords.copy_(saved[1])
            lum = self.fallback.collide(beam1, beam2, turn=turn, compute_luminosity=compute_luminosity, stream=stream)
            self.fallbacks += 1
        return lum


def time_forward(batch: int, grid: int = 48, repeats: int = 50, warmup: int = 5, device: int = 0) -> float:
    """Device microseconds of one network forward pass over `batch` planes (CUDA events on the launching
    stream, after `warmup` passes) -- the cost the learned correction adds to each wavefront."""
    net = FieldCorrectionNet(grid, grid, max_batch=max(64, batch), device=device)
    x = torch.randn(batch, grid, grid, 8, device=f"cuda:{device}").to(torch.bfloat16)
    for _ in range(warmup):
        net.forward(x)
    torch.cuda.synchronize(device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(repeats):
        net.forward(x)
    b.record()
    torch.cuda.synchronize(device)
    net.close()
    return a.elapsed_time(b) / repeats * 1e3


def _main(argv=None):
    """python -m octo_b200.learned --samples N --steps K [--out PATH]: generate pairs, train, evaluate on
    held-out pairs, save the weights.  --time-forward B: only time the network's forward pass over B planes."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--time-forward", type=int, default=0, metavar="B")
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--heldout", type=int, default=512)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--grid", type=int, default=48)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--coarse", default="hybrid", choices=COARSE)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    if a.time_forward:
        print(json.dumps({"batch": a.time_forward, "grid": a.grid, "forward_us": time_forward(a.time_forward, a.grid)}))
        return
    import time
    t0 = time.time()
    X, T, M, F = make_dataset(a.samples, a.seed, grid=a.grid, coarse=a.coarse)
    Xh, Th, Mh, Fh = make_dataset(a.heldout, a.seed + 1, grid=a.grid, coarse=a.coarse)
    t1 = time.time()
    net = FieldCorrectionNet(a.grid, a.grid, max_batch=max(64, a.batch), seed=a.seed)
    before = evaluate(net, Xh, Th, Mh, Fh)
    losses = train(net, X, T, M, a.steps, a.batch, a.lr, a.seed, log=print)
    t2 = time.time()
    after = evaluate(net, Xh, Th, Mh, Fh)
    tmax = float((Th.abs() * Mh[..., None]).amax())
    res = {"coarse": a.coarse, "samples": a.samples, "heldout": a.heldout, "steps": a.steps, "data_s": t1 - t0,
           "train_s": t2 - t1,
           "heldout_rms_err": after, "initial_net_rms_err": before, "final_loss": losses[-1],
           "heldout_max_abs_target": tmax}
    print(json.dumps(res))
    path = a.out or default_weights_path(a.grid, a.coarse)
    save_weights(net, path, coarse=a.coarse, heldout_uncorrected=after["hybrid"], heldout_learned=after["learned"],
                 samples=a.samples, steps=a.steps, seed=a.seed, max_abs_target=tmax)
    print("saved", path)


if __name__ == "__main__":
    _main()
