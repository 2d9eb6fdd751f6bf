#!/usr/bin/env python
"""Benchmark: PIC seconds per turn of the strong-strong collision at the production point.

Workload (one "step" = one turn): 2.56M electron / 1.024M proton seeded 6D Gaussian macroparticles,
flat beams sigma_x = 95 um, sigma_y = 8.5 um, sigma_z = 7 mm / 60 mm, delta_rms 5.5e-4 / 6.6e-4,
N = 1.7e11 / 6.9e10, E = 10 / 275 GeV; 15 :normal_quantile centroid slices, 128x128 :node interaction
grids, CIC, second-order field, linear slice interpolation, luminosity every turn; then the linear
uncoupled 6D one-turn map of each ring (tunes e 0.08/0.06, p 0.228/0.210; synchrotron tunes -0.069 /
-0.01 as in the reference's production example).  FP64 throughout (the plain form).

`python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]` prints one JSON line.
Under torchrun each rank runs an independent replica of the collision (a single collision does not
shard); `value` is the whole-job seconds per turn (max-over-ranks step time / turns done by all ranks).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "octopus.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "PIC s/turn (2.56M e/1.02M p, 15 sl, 128²) plain vs fast form at ≤1% field err"
UNIT = "s/turn"
N_E, N_P = 2_560_000, 1_024_000
SLICES, GRID = 15, 128
COARSE_GRID = 64  # the coarse fast form's grid (RMS field error vs exact Bassetti-Erskine below 1 %)
E_BEAM = dict(beta=(0.55, 0.056, 0.7e-2 / 5.5e-4), sigma=(95e-6, 8.5e-6, 7e-3), rng_id=1)
P_BEAM = dict(beta=(0.8, 0.072, 6e-2 / 6.6e-4), sigma=(95e-6, 8.5e-6, 6e-2), rng_id=2)
E_TUNES, P_TUNES = (0.08, 0.06, -0.069), (0.228, 0.210, -0.01)
SEED = 123456789
CONFIG = {
    "workload": "production EIC-like plain PIC, one turn = collide + one-turn maps",
    "n_electrons": N_E, "n_protons": N_P, "nslices": SLICES, "grid": [GRID, GRID],
    "interaction_grid": "node", "deposit": "CIC", "field_derivative": "second", "slice_interpolation": "linear",
    "luminosity": "every turn", "precision": "fp64 plain form (int64 fixed-point charge grids)",
    "l2": "inputs larger than L2 (172 MB of particle coordinates per turn)",
}
# DRAM bytes (read + write) per field particle of one kick launch, from one `ncu --set full` capture of
# the 15-pair front of this workload (276.9 MB for 3.584M field particles).
KICK_TRAFFIC_BYTES_PER_PARTICLE = 77.3


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    import datetime
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist.get_rank(), dist.get_world_size(), int(os.environ.get("LOCAL_RANK", "0"))


def _solver(ob, grid=GRID):
    return ob.PICPoissonSolver(grid=(grid, grid), interaction_grid="node", deposit_method="CIC",
                               slicing=ob.LongitudinalSlicing(nslices=SLICES, method="normal_quantile",
                                                              center_position="centroid"))


class Clocks:
    """nvidia-smi sampling during the timed region (clocks and throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.first = threading.Event()

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line)
            self.first.set()

    def wait_first(self, timeout: float = 10.0):
        """Returns once the sampler has written its first sample: its start-up (driver and NVML
        initialisation) then lies before the timed region rather than inside it."""
        if self.proc is not None:
            self.first.wait(timeout)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=10)
        except Exception:
            self.proc.kill()
        self.reader.join(timeout=10)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in list(self.lines):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx.append(float(f[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm), "reasons": sorted(reasons)}


def _cpu_baseline(steps_hint: int = 1, start=None):
    """The FP64 CPU oracle (a port of the reference's CPU PIC path) on full turns of the same workload, with
    every host thread; returns (s/turn, threads, sample description, luminosity of the first turn).  start:
    the (e, p) host arrays to begin from (default: the beams built on the host as Beam.jl builds them)."""
    import numpy as np
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    if start is None:
        e = orc.beam_gaussian(N_E, seed=SEED, rng_id=1, beta=E_BEAM["beta"], sigma=E_BEAM["sigma"])
        p = orc.beam_gaussian(N_P, seed=SEED, rng_id=2, beta=P_BEAM["beta"], sigma=P_BEAM["sigma"])
    else:
        e, p = (np.ascontiguousarray(a, dtype=np.float64).copy() for a in start)
    pe = orc.beam_params(-1.0, orc.EMASS_EV, 10e9, 1.7e11)
    pp = orc.beam_params(1.0, orc.PMASS_EV, 275e9, 6.9e10)
    oracle = orc.Oracle(orc.OracleOptions(grid=(GRID, GRID), interaction_grid="node", nslices1=SLICES,
                                          nslices2=SLICES, nthreads=threads))
    me = orc.linear6d_matrix(E_BEAM["beta"], (0, 0, 0), E_TUNES)
    mp = orc.linear6d_matrix(P_BEAM["beta"], (0, 0, 0), P_TUNES)
    times = []
    first_lum = None
    for _ in range(max(1, steps_hint)):
        t0 = time.perf_counter()
        lum = oracle.collide(e, p, pe, pp)
        orc.linear6d(me, e)
        orc.linear6d(mp, p)
        times.append(time.perf_counter() - t0)
        if first_lum is None:
            first_lum = lum
    return (statistics.median(times), threads, f"{len(times)} full turn(s) of the benchmark workload (collide + maps)",
            first_lum)


def run_reference(args, rank):
    """Reference arm: the reference's CPU algorithm (FP64 CPU oracle port; Julia is not available here)."""
    if rank != 0:
        return 0
    budget = 180.0
    t0 = time.perf_counter()
    n_warm = max(1, args.warmup)
    per, threads, _, _ = _cpu_baseline(n_warm)  # the requested warm-up turns (median turn time sizes the sample)
    n_time = max(1, min(args.steps, int(max(1.0, (budget - (time.perf_counter() - t0)) / max(per, 1e-3)))))
    val, threads, sample, _ = _cpu_baseline(n_time)
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": n_time,
        "warmup": n_warm, "ms_per_step": val * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded counter-RNG Gaussian beams)", "config": CONFIG,
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU PIC path restated in C++ (Julia is absent on this machine); all host threads",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    import octo_b200 as ob

    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    solver = _solver(ob)
    e = ob.Beam.gaussian(N_E, seed=SEED, charge=-1.0, mc2=ob.EMASS_EV, E0=10e9, npart=1.7e11, device=dev, **E_BEAM)
    p = ob.Beam.gaussian(N_P, seed=SEED, charge=1.0, mc2=ob.PMASS_EV, E0=275e9, npart=6.9e10, device=dev, **P_BEAM)
    me = ob.Linear6D(E_BEAM["beta"], (0, 0, 0), E_TUNES)
    mp = ob.Linear6D(P_BEAM["beta"], (0, 0, 0), P_TUNES)
    rt = ob.StrongStrongRuntime()
    ctx = rt.context("ip", solver, local_rank)
    stream = torch.cuda.current_stream(dev)
    e0, p0 = e.coords.clone(), p.coords.clone()
    # launch shape picked on copies of the beams, before the warm-up (results do not depend on it)
    shape = ctx.autotune(e, p, rounds=2, stream=stream)

    def turn(t):
        lum = ctx.collide(e, p, turn=t, stream=stream)
        me.track(e, stream=stream)
        mp.track(p, stream=stream)
        return lum

    for t in range(args.warmup):
        turn(t)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    clocks = Clocks(local_rank)
    clocks.start()
    clocks.wait_first()
    time.sleep(0.3)
    # the timed region carries no instrumentation: an event recorded between two kernels of the collide
    # stream costs time and breaks their programmatic launch overlap (~0.3 ms per turn for the kicks'
    # events alone).  The kick's durations (roofline) and the per-phase split come from instrumented passes
    # of the same turns right after it.
    ctx.set_timing(False)
    launches = 0
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # every turn waits on the host for its luminosity, so a host pause is GPU idle time: no Python garbage
    # collection inside the timed loops
    gc.collect()
    gc.disable()
    graph0 = ctx.collide_graph_stats()
    ev0.record(stream)
    for t in range(args.steps):
        lum = turn(args.warmup + t)
        launches += ctx.last_report.kernel_launches + 2
    ev1.record(stream)
    torch.cuda.synchronize()
    gc.enable()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    graph1 = ctx.collide_graph_stats()
    n_kick = max(3, min(args.steps, 20))
    ctx.set_timing(True, phases=["kick"])
    for t in range(n_kick):
        turn(args.warmup + args.steps + t)
    torch.cuda.synchronize()
    kick_report = ctx.timing_report()["kick"]
    n_phase = max(3, min(args.steps, 10))
    ctx.set_timing(True)
    for t in range(n_phase):
        turn(args.warmup + args.steps + n_kick + t)
    torch.cuda.synchronize()
    phases = ctx.timing_report()
    ctx.set_timing(False)

    # end to end through the public API with host-resident beams (pinned), copies inside the region
    he = torch.empty_like(e0, device="cpu").pin_memory()
    hp = torch.empty_like(p0, device="cpu").pin_memory()
    he.copy_(e0); hp.copy_(p0)
    e2e_steps = 0 if args.no_e2e else max(3, min(args.steps, 20))
    torch.cuda.synchronize()
    barrier()
    gc.collect()
    gc.disable()
    w0 = time.perf_counter()
    ev0.record(stream)
    lum_from_start = None
    for t in range(e2e_steps):
        e.coords.copy_(he, non_blocking=True)
        p.coords.copy_(hp, non_blocking=True)
        lum_e2e = turn(10_000 + t)
        if lum_from_start is None:
            lum_from_start = lum_e2e
        he.copy_(e.coords, non_blocking=True)
        hp.copy_(p.coords, non_blocking=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    gc.enable()
    wall = (time.perf_counter() - w0) / max(e2e_steps, 1)
    barrier()
    e2e_ms = ev0.elapsed_time(ev1) / e2e_steps if e2e_steps else float("nan")
    if lum_from_start is None:  # the luminosity of one turn from the workload's initial beams (parity check)
        e.coords.copy_(e0)
        p.coords.copy_(p0)
        lum_from_start = turn(10_000)
        torch.cuda.synchronize()

    # the fast forms on the same workload: float32 beams and the same maps, on the production grid and on a
    # coarse 64^2 :node grid (its RMS field error vs exact Bassetti-Erskine stays below 1 %, reported below)
    solver_coarse = _solver(ob, grid=COARSE_GRID)

    def time_form(sol):
        eX, pX = e.astype(torch.float32), p.astype(torch.float32)
        eX.coords.copy_(e0.to(torch.float32)); pX.coords.copy_(p0.to(torch.float32))
        cX = rt.context("ip", sol, local_rank, torch.float32)
        shapeX = cX.autotune(eX, pX, rounds=2, stream=stream)

        def turnX(t):
            lum = cX.collide(eX, pX, turn=t, stream=stream)
            me.track(eX, stream=stream)
            mp.track(pX, stream=stream)
            return lum

        for t in range(args.warmup):
            turnX(t)
        torch.cuda.synchronize()
        cX.set_timing(False)
        barrier()
        torch.cuda.synchronize()
        gc.collect()
        gc.disable()
        ev0.record(stream)
        for t in range(args.steps):
            lumX = turnX(args.warmup + t)
        ev1.record(stream)
        torch.cuda.synchronize()
        gc.enable()
        barrier()
        msX = ev0.elapsed_time(ev1) / args.steps
        cX.set_timing(True, phases=["kick"])
        for t in range(n_kick):
            turnX(args.warmup + args.steps + t)
        torch.cuda.synchronize()
        kickX = cX.timing_report()["kick"]
        cX.set_timing(True)
        for t in range(n_phase):
            turnX(args.warmup + args.steps + n_kick + t)
        torch.cuda.synchronize()
        phX = cX.timing_report()
        cX.set_timing(False)
        return {"ms": msX, "lum": lumX, "phases": {k: v[0] / n_phase for k, v in phX.items()}, "kick": kickX,
                "shape": shapeX}

    fast = fast_coarse = None
    if not args.no_fast:
        fast = time_form(solver)
        fast_coarse = time_form(solver_coarse)
        shape32, shape32c = fast["shape"], fast_coarse["shape"]
    # the oracle's CPU timings of these passes run once, on a single-GPU run
    cpu_side = world == 1 and not args.no_cpu_baseline
    lines = None if args.no_line else time_lines(ob, e0, p0, args, stream, barrier, cpu_side)
    observer = None if args.no_line else time_observer(ob, e0, p0, args, stream)
    soft = None if args.no_line else time_soft_gaussian(ob, e0, p0, me, mp, rt, local_rank, args, stream, cpu_side)
    learned = None if args.no_fast else time_learned(ob, e0, p0, me, mp, local_rank, args, stream, barrier, ms,
                                                     world)
    clk = clocks.stop()

    # long-term tracking of both forms from the same beams (outside every timed region, one GPU only):
    # the relative emittance growth of each plane after --emittance-turns turns
    emit = None
    if world == 1 and args.emittance_turns > 0:
        from octo_b200.diagnostics import emittances
        emit = {"turns": args.emittance_turns}
        for name, dt, sol in (("plain", torch.float64, solver), ("fast", torch.float32, solver),
                              ("fast_coarse", torch.float32, solver_coarse)):
            if name != "plain" and args.no_fast:
                continue
            ee, pp = e.astype(dt), p.astype(dt)
            ee.coords.copy_(e0.to(dt))
            pp.coords.copy_(p0.to(dt))
            cx = rt.context("ip", sol, local_rank, dt)
            start = (emittances(ee), emittances(pp))
            for t in range(args.emittance_turns):
                cx.collide(ee, pp, turn=20_000 + t, stream=stream)
                me.track(ee, stream=stream)
                mp.track(pp, stream=stream)
            torch.cuda.synchronize()
            end = (emittances(ee), emittances(pp))
            emit[name] = {beam: [end[k][q] / start[k][q] - 1.0 for q in range(3)]
                          for k, beam in enumerate(("electron", "proton"))}

    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms, e2e_ms, fast["ms"] if fast else 0.0, fast_coarse["ms"] if fast_coarse else 0.0],
                          device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms, e2e_ms = float(tt[0]), float(tt[1])
        if fast:
            fast["ms"] = float(tt[2])
        if fast_coarse:
            fast_coarse["ms"] = float(tt[3])

    if rank != 0:
        return 0
    value = ms / 1e3 / world
    kick_ms, kick_launches, kick_bytes = kick_report
    # the luminosity phase runs on the collide's second stream, overlapped with the field solve
    dom = max(((k, v) for k, v in phases.items() if k != "luminosity"), key=lambda kv: kv[1][0])
    roof = None
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    if kick_ms > 0:
        achieved = kick_bytes / (kick_ms / 1e3) / 1e9
        traffic = None
        if KICK_TRAFFIC_BYTES_PER_PARTICLE is not None and kick_launches:
            traffic = KICK_TRAFFIC_BYTES_PER_PARTICLE * (kick_bytes / 88.0) / kick_launches
        roof = {"kernel": "k_kick (gather + 6D synchro-beam kick)", "bound": "hbm", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "traffic_source": "constant: DRAM bytes per field particle from one ncu capture of this kernel "
                                  "(profiles/kick_node_production.md), scaled to the average launch",
                "algorithmic_bytes_per_launch": kick_bytes / max(kick_launches, 1),
                "avg_launch_ms": kick_ms / max(kick_launches, 1),
                "timing": f"CUDA events around every kick launch on the collide stream, in a pass of {n_kick} "
                          "turns right after the (uninstrumented) timed region"}
    fast_line = coarse_line = None
    if fast:
        from octo_b200.diagnostics import field_error
        sy = E_BEAM["sigma"][1]
        errs = {"plain": {}, "fast": {}}
        errs_coarse = {}
        for aspect in (1.0, 5.0, E_BEAM["sigma"][0] / sy, 25.0):
            key = f"{aspect:.3g}"
            errs["plain"][key] = field_error(solver, aspect * sy, sy, torch.float64, local_rank)["rms"]
            errs["fast"][key] = field_error(solver, aspect * sy, sy, torch.float32, local_rank)["rms"]
            errs_coarse[key] = field_error(solver_coarse, aspect * sy, sy, torch.float32, local_rank)["rms"]
        coarse_line = {
            "value": fast_coarse["ms"] / 1e3 / world, "unit": UNIT, "ms_per_step": fast_coarse["ms"],
            "form": f"precision form on a {COARSE_GRID}x{COARSE_GRID} :node grid (other options as the workload)",
            "speedup_vs_plain": ms / fast_coarse["ms"], "luminosity": fast_coarse["lum"],
            "field_rms_err_vs_bassetti_erskine": errs_coarse,
            "max_field_rms_err": max(errs_coarse.values()),
            "phases_ms_per_turn": fast_coarse["phases"],
        }
        k_ms, k_launches, k_bytes = fast["kick"]
        fast_line = {
            "value": fast["ms"] / 1e3 / world, "unit": UNIT, "ms_per_step": fast["ms"],
            "form": "precision form: float32 particles, field planes and FFTs; FP64 Green function, slice "
                    "statistics and luminosity; int64 fixed-point charge grids",
            "speedup_vs_plain": ms / fast["ms"], "luminosity": fast["lum"],
            "field_rms_err_vs_bassetti_erskine": errs,
            "field_err_method": "81x81 probes over +-4 sigma, RMS normalised by max exact field, one collide",
            "kick_achieved_gbs": k_bytes / (k_ms / 1e3) / 1e9 if k_ms > 0 else None,
            "phases_ms_per_turn": fast["phases"],
        }
    cpu = None
    parity = None
    if world == 1 and not args.no_cpu_baseline:
        # one oracle turn from the same initial beams the GPU turns started from (the device-built beams,
        # copied to the host): its luminosity against the GPU's turn from those beams
        v, threads, sample, lum_oracle = _cpu_baseline(1, start=(e0.cpu().numpy(), p0.cpu().numpy()))
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}
        parity = {"luminosity_gpu": lum_from_start, "luminosity_oracle": lum_oracle,
                  "rel_diff": abs(lum_from_start / lum_oracle - 1.0),
                  "tolerance": 1e-10,
                  "what": "luminosity of one turn (collide + maps) from the workload's initial beams, GPU vs the "
                          "FP64 CPU oracle on identical inputs"}
    beam_bytes = (N_E + N_P) * 6 * 8
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded counter-RNG Gaussian beams)",
        "config": CONFIG,
        "parallelism": f"replicas{world}",
        "e2e": {"value": e2e_ms / 1e3 / world, "unit": UNIT, "h2d_bytes_per_step": beam_bytes,
                "d2h_bytes_per_step": beam_bytes + 8, "wall_s_per_step": wall},
        "gpu_launches": launches,
        # timed collides that ran as the captured graph behind its device guard (octo_set_collide_graph)
        "collide_graph": {"replayed_turns": graph1[1] - graph0[1], "declined_turns": graph1[2] - graph0[2],
                          "timed_turns": args.steps, "captures": graph1[0]},
        "launch_shape": {"chosen": list(ctx.AUTOTUNE_SHAPES[shape]),
                         "chosen_fast_form": list(ctx.AUTOTUNE_SHAPES[shape32]) if fast else None,
                         "chosen_fast_form_coarse": list(ctx.AUTOTUNE_SHAPES[shape32c]) if fast else None,
                         "meaning": "(deposit waves of SMs per wavefront, kick resident-slot multiple), picked by "
                                    "octo_pic_autotune on copies of the beams before the warm-up"},
        "roofline": roof,
        "cpu_baseline": cpu,
        "parity": parity,
        "fast_form": fast_line,
        "fast_form_coarse": coarse_line,
        "emittance_growth": emit,
        "line_tracking": lines,
        "moment_observer": observer,
        "soft_gaussian": soft,
        "learned_form": learned,
        "clocks": clk,
        "luminosity": lum,
        "dominant_phase": dom[0],
        "dominant_phase_note": "largest phase on the collide stream (luminosity runs on a second stream, overlapped)",
        "phases_ms_per_turn": {k: v[0] / n_phase for k, v in phases.items()},
        "phases_note": "per-phase CUDA events, from an instrumented pass after the timed region",
    }
    print(json.dumps(line), flush=True)
    rt.close()
    return 0


def time_lines(ob, e0, p0, args, stream, barrier, cpu_side=True):
    """Line tracking between collisions on the same beams: both rings of the strong-strong example's lattice
    (before the collision: inverse crab transport, crab cavity, crab-to-IP transport, Lorentz boost; after
    it: reverse boost, IP-to-crab transport, crab cavity, inverse transport, one-turn map, chromaticity kick
    and, for electrons, lumped radiation), each segment one octo_track_line pass.  Reported per turn (four
    launches) and per segment, each segment against the HBM roofline of its 96 bytes per particle."""
    import torch
    from octo_b200 import line as ln
    beams = {"electron": ob.Beam(e0.clone(), ob.BeamParams(-1.0, ob.EMASS_EV, 10e9, 0.0, 1.7e11)),
             "proton": ob.Beam(p0.clone(), ob.BeamParams(1.0, ob.PMASS_EV, 275e9, 0.0, 6.9e10))}
    segs = {b: ln.eic_like_segments(b) for b in beams}
    K = max(10, min(args.steps, 50))

    def one_turn(t):
        ctx = ob.TrackingContext(turn=t)
        for b, (before, after) in segs.items():
            ob.track(beams[b], before, 1, ctx, stream=stream)
            ob.track(beams[b], after, 1, ctx, stream=stream)

    for t in range(args.warmup):
        one_turn(t)
    torch.cuda.synchronize()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    gc.collect()
    gc.disable()
    ev0.record(stream)
    for t in range(K):
        one_turn(args.warmup + t)
    ev1.record(stream)
    torch.cuda.synchronize()
    gc.enable()
    turn_ms = ev0.elapsed_time(ev1) / K
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    per = {}
    for b, (before, after) in segs.items():
        n = beams[b].n
        for name, seg in (("before", before), ("after", after)):
            ev0.record(stream)
            for t in range(K):
                ob.track(beams[b], seg, 1, ob.TrackingContext(turn=1000 + t), stream=stream)
            ev1.record(stream)
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1) / K
            gbs = n * 96 / (ms / 1e3) / 1e9
            per[f"{b}.{name}"] = {"elements": len(seg), "ms": ms, "achieved_gbs": gbs, "frac_of_hbm": gbs / hbm}
    # the oracle on a bounded sample, all host threads, scaled to the full beams
    cpu_s = None
    sample = 100_000
    if cpu_side:
        from oracle import oracle as orc
        t0 = time.perf_counter()
        for b in beams:
            src = (e0 if b == "electron" else p0)[:, :sample].cpu().numpy()
            elems = [el.to_c() for el in ln.flatten(segs[b])]
            orc.track_line(elems, src, turn=0, turns=1, seed=0, rng_method=1)
        cpu_s = (time.perf_counter() - t0) * (N_E + N_P) / (2 * sample)
    return {"ms_per_turn": turn_ms, "launches_per_turn": 4, "segments": per, "hbm_peak_gbs": hbm,
            "bytes_per_particle_per_launch": 96,
            "cpu_oracle_s_per_turn": cpu_s, "cpu_sample": f"{sample} particles of each beam, scaled",
            "note": "each launch reads and writes the six FP64 coordinates once; a segment of maps alone runs "
                    "at the HBM bound, the radiation's six Philox draws and three Box-Muller transforms per "
                    "particle make the electron's after-collision segment instruction-issue bound"}


def time_learned(ob, e0, p0, me, mp, local_rank, args, stream, barrier, plain_ms, world):
    """The learned forms on the same workload: a 48x48 coarse solver with the tensor-core network's field
    correction (octo_b200.learned, weights trained on the GPU by `python -m octo_b200.learned`), falling back
    to the plain 128x128 :node solver when a plane's correction estimate exceeds twice the largest correction
    seen in training.  "hybrid": the Gaussian-subtracted hybrid (FP64 beams); "pic": plain PIC in the
    precision form (float32 beams).  Each: s/turn (collide + maps), the speed-up over the plain form, RMS
    field error against exact Bassetti-Erskine with and without the correction, fallbacks, and the relative
    emittance growth after --emittance-turns turns."""
    import torch
    from octo_b200 import learned as L
    from octo_b200.diagnostics import emittances, field_error
    out = {}
    slicing = ob.LongitudinalSlicing(nslices=SLICES, method="normal_quantile", center_position="centroid")
    for coarse, dtype in (("hybrid", torch.float64), ("pic", torch.float32)):
        try:
            net, meta = L.load_net(coarse=coarse, max_batch=64, device=local_rank)
        except FileNotFoundError:
            continue
        tol = 2.0 * float(meta.get("max_abs_target", 5.0)) / L.OUT_SCALE
        sol = L.coarse_solver(coarse, 48, slicing=slicing, deposit_method="CIC")
        form = L.LearnedForm(sol, _solver(ob), net, tolerance=tol, device=local_rank, dtype=dtype)
        eX, pX = ob.Beam(e0.to(dtype).clone(), ob.BeamParams(-1.0, ob.EMASS_EV, 10e9, ob.RE, 1.7e11)), \
            ob.Beam(p0.to(dtype).clone(), ob.BeamParams(1.0, ob.PMASS_EV, 275e9, ob.RE * ob.ME0 / ob.PMASS_EV, 6.9e10))

        def turnX(t):
            lum = form.collide(eX, pX, turn=t, stream=stream)
            me.track(eX, stream=stream)
            mp.track(pX, stream=stream)
            return lum

        for t in range(args.warmup):
            turnX(t)
        torch.cuda.synchronize()
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = form.fallbacks
        ev0.record(stream)
        for t in range(args.steps):
            lum = turnX(args.warmup + t)
        ev1.record(stream)
        torch.cuda.synchronize()
        msX = ev0.elapsed_time(ev1) / args.steps
        fb = form.fallbacks - n0
        sy = E_BEAM["sigma"][1]
        errs, errs_raw = {}, {}
        for aspect in (1.0, 5.0, E_BEAM["sigma"][0] / sy, 25.0):
            key = f"{aspect:.3g}"
            errs[key] = field_error(sol, aspect * sy, sy, dtype, local_rank,
                                    correction=(net, L.OUT_SCALE, 1e30, L.EDGE))["rms"]
            errs_raw[key] = field_error(sol, aspect * sy, sy, dtype, local_rank)["rms"]
        grow = None
        if world == 1 and args.emittance_turns > 0:
            eX.coords.copy_(e0.to(dtype))
            pX.coords.copy_(p0.to(dtype))
            start = (emittances(eX), emittances(pX))
            for t in range(args.emittance_turns):
                turnX(30_000 + t)
            torch.cuda.synchronize()
            end = (emittances(eX), emittances(pX))
            grow = {beam: [end[k][q] / start[k][q] - 1.0 for q in range(3)] for k, beam in enumerate(("electron", "proton"))}
        out[coarse] = {
            "value": msX / 1e3 / world, "unit": UNIT, "ms_per_step": msX, "speedup_vs_plain": plain_ms / msX,
            "form": (f"{'Gaussian-subtracted hybrid' if coarse == 'hybrid' else 'plain PIC'} on a 48x48 :slice_pair "
                     f"grid (no Green cache), {'float64' if dtype == torch.float64 else 'float32'} beams, with the "
                     "tensor-core CNN's field correction; plain 128x128 :node fallback"),
            "luminosity": lum, "fallback_collides": fb, "timed_collides": args.steps,
            "error_estimate_tolerance": tol,
            "field_rms_err_vs_bassetti_erskine": errs, "field_rms_err_uncorrected": errs_raw,
            "max_field_rms_err": max(errs.values()),
            "heldout_rms_err_vs_fine_pic": {"uncorrected": float(meta.get("heldout_uncorrected", float("nan"))),
                                            "learned": float(meta.get("heldout_learned", float("nan")))},
            "emittance_growth": grow, "emittance_turns": args.emittance_turns if grow else 0,
            "network": {"params": net.num_params, "trained_samples": int(meta.get("samples", 0)),
                        "train_steps": int(meta.get("steps", 0))},
        }
        form.close()
        net.close()
    return out or None


def time_soft_gaussian(ob, e0, p0, me, mp, rt, local_rank, args, stream, cpu_side=True):
    """The soft-Gaussian solver (GaussianPoissonSolver, 15 slices) on the same beams and maps: s/turn, the
    phase split (moments, kick), the kick's achieved bytes per second (11 FP64 values per field particle per
    pair) and the oracle's time per turn on a 10 % sample."""
    import torch
    solver = ob.GaussianPoissonSolver(slicing=ob.LongitudinalSlicing(nslices=SLICES, method="normal_quantile"))
    e = ob.Beam(e0.clone(), ob.BeamParams(-1.0, ob.EMASS_EV, 10e9, ob.RE, 1.7e11))
    p = ob.Beam(p0.clone(), ob.BeamParams(1.0, ob.PMASS_EV, 275e9, ob.RE * ob.ME0 / ob.PMASS_EV, 6.9e10))
    ctx = rt.context("soft", solver, local_rank)

    def turn(t):
        lum = ctx.collide(e, p, turn=t, stream=stream)
        me.track(e, stream=stream)
        mp.track(p, stream=stream)
        return lum

    for t in range(args.warmup):
        turn(t)
    torch.cuda.synchronize()
    K = max(5, min(args.steps, 30))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    gc.collect()
    gc.disable()
    ev0.record(stream)
    for t in range(K):
        lum = turn(args.warmup + t)
    ev1.record(stream)
    torch.cuda.synchronize()
    gc.enable()
    ms = ev0.elapsed_time(ev1) / K
    ctx.set_timing(True)
    nph = 5
    for t in range(nph):
        turn(args.warmup + K + t)
    torch.cuda.synchronize()
    ph = ctx.timing_report()
    ctx.set_timing(False)
    kick_ms, _, _ = ph["kick"]
    kick_bytes = (N_E + N_P) * SLICES * 11 * 8 * nph
    out = {"value": ms / 1e3, "unit": UNIT, "ms_per_step": ms, "luminosity": lum, "nslices": SLICES,
           "phases_ms_per_turn": {"slicing": ph["slicing"][0] / nph, "moments": ph["bounds"][0] / nph,
                                  "kick": kick_ms / nph, "unsort": ph["unsort"][0] / nph},
           "kick_achieved_gbs": kick_bytes / (kick_ms / 1e3) / 1e9 if kick_ms > 0 else None}
    # the oracle on a 10 % sample of both beams (same slicing), all host threads
    if cpu_side:
        from oracle import oracle as orc
        se, sp = e0[:, : N_E // 10].cpu().numpy().copy(), p0[:, : N_P // 10].cpu().numpy().copy()
        opt = orc.OracleOptions(nslices1=SLICES, nslices2=SLICES)
        t0 = time.perf_counter()
        orc.gaussian_collide(opt, se, sp, orc.beam_params(-1.0, orc.EMASS_EV, 10e9, 1.7e11),
                             orc.beam_params(1.0, orc.PMASS_EV, 275e9, 6.9e10))
        out["cpu_oracle_s_per_turn"] = (time.perf_counter() - t0) * 10
        out["cpu_sample"] = "10 % of each beam, one collide, scaled by 10"
    return out


def time_observer(ob, e0, p0, args, stream):
    """The moment observer on both beams (the default orders 1:2, 27 moments): each observation is two passes
    over the beam (means, then the 21 second-order sums) whose row stays on the device; 96 bytes per
    particle read."""
    import torch
    beams = {"electron": ob.Beam(e0.clone(), ob.BeamParams(-1.0, ob.EMASS_EV, 10e9, 0.0, 1.7e11)),
             "proton": ob.Beam(p0.clone(), ob.BeamParams(1.0, ob.PMASS_EV, 275e9, 0.0, 6.9e10))}
    K = max(10, min(args.steps, 50))
    obs = {b: ob.MomentObserver(b, capacity=K + args.warmup, device=torch.cuda.current_device()) for b in beams}
    for t in range(args.warmup):
        for b in beams:
            obs[b].observe(t, beams[b], stream=stream)
    torch.cuda.synchronize()
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    out = {"moments": len(obs["electron"].moments), "hbm_peak_gbs": hbm}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for b in beams:
        ev0.record(stream)
        for t in range(K):
            obs[b].observe(args.warmup + t, beams[b], stream=stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / K
        gbs = beams[b].n * 96 / (ms / 1e3) / 1e9
        out[b] = {"us_per_row": ms * 1e3, "achieved_gbs": gbs, "frac_of_hbm": gbs / hbm}
    out["note"] = ("rows are written to a device record buffer; the host reads them once per flush, so "
                   "observing a turn adds no host synchronisation")
    return out


def scan_cases(n_cases=64, seed=SEED):
    """Seeded batched-scan cases: N per beam log-uniform in [64k, 2.56M], slices uniform in 5..31, grid in
    {64, 96, 128, 256}^2, sigma_x / sigma_y log-uniform in [1, 25] with sigma_y = 8.5 um."""
    import numpy as np
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(n_cases):
        n1, n2 = (int(np.exp(rng.uniform(np.log(64_000), np.log(2_560_000)))) for _ in range(2))
        s1, s2 = (int(rng.integers(5, 32)) for _ in range(2))
        g = int(rng.choice([64, 96, 128, 256]))
        aspect = float(np.exp(rng.uniform(0.0, np.log(25.0))))
        cases.append(dict(n1=n1, n2=n2, s1=s1, s2=s2, grid=g, aspect=aspect, rng=int(rng.integers(1, 2**31))))
    return cases


def run_scan(args, rank, world, local_rank):
    """The batched scan: independent collisions in the precision form, in batches of --scan-batch collides
    overlapped on their own streams (octo_pic_collide_batch), against the same collides one by one.  Under
    torchrun each rank runs its share of the cases (octo_b200.parallel.partition_collisions, a size-balanced
    greedy partition; no data-path collective); the time is the max over ranks."""
    import torch
    import octo_b200 as ob
    from octo_b200.parallel import collision_cost, max_over_ranks, partition_collisions
    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    cases = scan_cases(args.scan_cases)
    costs = [collision_cost(c["n1"], c["n2"], max(c["s1"], c["s2"]), c["grid"]) for c in cases]
    mine = [cases[k] for k in partition_collisions(costs, world)[rank]]
    turns = args.scan_turns
    sy = 8.5e-6

    def make(case):
        sol = ob.PICPoissonSolver(grid=(case["grid"], case["grid"]),
                                  slicing1=ob.LongitudinalSlicing(nslices=case["s1"], method="normal_quantile"),
                                  slicing2=ob.LongitudinalSlicing(nslices=case["s2"], method="normal_quantile"))
        sx = case["aspect"] * sy
        e = ob.Beam.gaussian(case["n1"], seed=case["rng"], charge=-1.0, mc2=ob.EMASS_EV, E0=10e9, npart=1.7e11,
                             device=dev, dtype=torch.float32, beta=E_BEAM["beta"], sigma=(sx, sy, 7e-3), rng_id=1)
        p = ob.Beam.gaussian(case["n2"], seed=case["rng"], charge=1.0, mc2=ob.PMASS_EV, E0=275e9, npart=6.9e10,
                             device=dev, dtype=torch.float32, beta=P_BEAM["beta"], sigma=(sx, sy, 6e-2), rng_id=2)
        return sol, e, p

    times = {}
    for mode in ("batched", "sequential"):
        total_ms = 0.0
        for g0 in range(0, len(mine), args.scan_batch):
            group = [make(c) for c in mine[g0:g0 + args.scan_batch]]
            ctxs = [ob.Context(sol, local_rank, torch.float32) for sol, _, _ in group]
            streams = [torch.cuda.Stream(device=dev) for _ in group]
            for t in range(2):  # warm-up turns (workspaces, Green caches)
                ob.collide_batch(ctxs, [g[1] for g in group], [g[2] for g in group], turn=t, streams=streams)
            torch.cuda.synchronize()
            main = torch.cuda.current_stream(dev)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(main)
            for st in streams:
                st.wait_event(ev0)
            for t in range(turns):
                if mode == "batched":
                    ob.collide_batch(ctxs, [g[1] for g in group], [g[2] for g in group], turn=2 + t, streams=streams)
                else:
                    for k, (sol, e, p) in enumerate(group):
                        ctxs[k].collide(e, p, turn=2 + t, stream=streams[k])
            for st in streams:  # the end event follows every stream's work
                done = torch.cuda.Event()
                done.record(st)
                main.wait_event(done)
            ev1.record(main)
            torch.cuda.synchronize()
            total_ms += ev0.elapsed_time(ev1)
            for c in ctxs:
                c.close()
            del group
            torch.cuda.empty_cache()
        times[mode] = max_over_ranks(total_ms)
    if rank != 0:
        return 0
    collide_turns = len(cases) * turns
    line = {
        "metric": "batched scan: s per collision-turn", "value": times["batched"] / 1e3 / collide_turns,
        "unit": "s/collision-turn", "n_gpus": world, "higher_is_better": False, "impl": "ours", "scaling": "strong",
        "sequential_value": times["sequential"] / 1e3 / collide_turns,
        "batching_speedup": times["sequential"] / times["batched"],
        "config": {"workload": "independent collisions, precision form (float32 beams), default PICPoissonSolver "
                               "options (:slice_pair grid, slice-pair Green cache, CIC); N log-uniform 64k-2.56M per "
                               "beam, slices 5..31, grids 64/96/128/256, aspect 1-25",
                   "cases": len(cases), "turns": turns, "batch": args.scan_batch,
                   "partition": "size-balanced greedy over ranks (octo_b200.parallel.partition_collisions)",
                   "timing": "CUDA events spanning every collide stream of each group after 2 warm-up turns, "
                             "summed over the rank's groups; max over ranks"},
        "particles": sum(c["n1"] + c["n2"] for c in cases),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_profile_form(args, local_rank):
    """Profiling runs: `args.steps` turns of one form of the workload (plain: FP64 at 128^2; fast: the precision
    form at 128^2; coarse: the precision form at 64^2) with the collide's ordinary launches -- a captured graph's
    kernels are not listed one by one by a kernel profiler -- and no output line."""
    import torch
    import octo_b200 as ob

    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    grid = COARSE_GRID if args.profile_form == "coarse" else GRID
    dtype = torch.float64 if args.profile_form == "plain" else torch.float32
    e = ob.Beam.gaussian(N_E, seed=SEED, charge=-1.0, mc2=ob.EMASS_EV, E0=10e9, npart=1.7e11, device=dev, **E_BEAM)
    p = ob.Beam.gaussian(N_P, seed=SEED, charge=1.0, mc2=ob.PMASS_EV, E0=275e9, npart=6.9e10, device=dev, **P_BEAM)
    if dtype == torch.float32:
        e, p = e.astype(dtype), p.astype(dtype)
    me = ob.Linear6D(E_BEAM["beta"], (0, 0, 0), E_TUNES)
    mp = ob.Linear6D(P_BEAM["beta"], (0, 0, 0), P_TUNES)
    rt = ob.StrongStrongRuntime()
    ctx = rt.context("ip", _solver(ob, grid), local_rank, dtype)
    ctx.set_collide_graph(False)
    stream = torch.cuda.current_stream(dev)
    for t in range(args.steps):
        ctx.collide(e, p, turn=t, stream=stream)
        me.track(e, stream=stream)
        mp.track(p, stream=stream)
    torch.cuda.synchronize()
    rt.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end pass (profiling runs)")
    ap.add_argument("--no-fast", action="store_true", help="skip the precision-form (float32) pass")
    ap.add_argument("--no-line", action="store_true", help="skip the line-tracking (between collisions) pass")
    ap.add_argument("--scan", action="store_true", help="time the batched scan of independent collisions instead")
    ap.add_argument("--scan-cases", type=int, default=64)
    ap.add_argument("--scan-turns", type=int, default=20)
    ap.add_argument("--scan-batch", type=int, default=8)
    ap.add_argument("--profile-form", choices=["plain", "fast", "coarse"], default=None,
                    help="profiling runs: --steps turns of one form with ordinary launches, no output line")
    ap.add_argument("--emittance-turns", type=int, default=1000,
                    help="turns of the emittance-growth comparison of both forms (0 skips it; one GPU only)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local_rank = _dist()
    try:
        if args.impl == "reference":
            return run_reference(args, rank)
        if args.scan:
            return run_scan(args, rank, world, local_rank)
        if args.profile_form:
            return run_profile_form(args, local_rank)
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
