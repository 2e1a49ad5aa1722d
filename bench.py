"""Benchmark of the USL MPM step: particle-steps/s on B200.

Default workload: the 3D granular column collapse (1,331,712 particles,
Drucker-Prager, quadratic B-splines, gravity, slip walls, 257x65x129 nodes,
dt 1e-5), the configuration the headline metric is quoted on.  Synthetic,
seeded particle set (numpy PCG64 seed 0).  The particle state (~154 MB) is
larger than the 126 MB L2, so no flush is needed between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs one independent replica per GPU (the path does not shard at this
size; no collective on the data path), launched by torch.distributed.run.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1xB200: plain vs batched vs fwd+adjoint, <=1e-4 rel err vs FP64"
# algorithmic bytes per particle-step of the whole step (FP32 SoA state read
# and written once; symmetric tensors 6 floats in 3D)
STEP_BYTES = {("3d", "dp"): 224, ("2d", "le"): 96, ("2d", "dp"): 120}


def p2g_kernel_name(kw, variant):
    """The P2G kernel a configuration runs (3D quadratic: the autotuner's pick)."""
    if kw["dim"] == 2:
        return "tile scatter (2D)"
    if kw["shape_function"] == "quadratic":
        return {1: "dual-cell z-sweep", 0: "cell-row scatter"}[variant]
    return "z-sweep (3D %s)" % kw["shape_function"]


def load_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def scene_for(config, scale=1.0):
    from pyroclastmpm_b200 import scenes

    if config == "column":
        return scenes.granular_column(scale=scale)
    if config == "discs":
        return scenes.two_discs()
    if config == "bed":
        return scenes.granular_bed(scale=scale)
    raise ValueError(config)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, value):
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def cpu_reference_ensemble(steps, num):
    """The oracle on the first `num` instances of the ensemble, `steps` each."""
    import oracle
    from pyroclastmpm_b200 import scenes

    insts = scenes.ensemble()[:num]
    refs = [oracle.OracleSim(**scenes.sim_kwargs(sc), positions=sc["positions"],
                             velocities=sc["velocities"]).initialize() for sc in insts]
    t0 = time.perf_counter()
    for r in refs:
        r.solve(steps)
    dt = time.perf_counter() - t0
    n = sum(len(sc["positions"]) for sc in insts)
    return {"value": n * steps / dt, "unit": "particle-steps/s", "cores": 1, "kind": "port",
            "sample": f"first {num} ensemble instances ({n} particles), {steps} steps each, serial C oracle (FP32)",
            "seconds": dt}


def cpu_reference(config, steps, warmup, sample_scale):
    """The oracle (C restatement of the reference step, one thread) on a
    bounded sample of the workload: the same grid, the particle region scaled
    by sample_scale per axis."""
    import oracle
    from pyroclastmpm_b200 import scenes

    if config == "ensemble":
        return cpu_reference_ensemble(max(steps, 1), 16)
    scene = scene_for(config, scale=sample_scale)
    ref = oracle.OracleSim(**scenes.sim_kwargs(scene), positions=scene["positions"],
                           velocities=scene["velocities"]).initialize()
    for _ in range(warmup):
        ref.solve(1)
    t0 = time.perf_counter()
    ref.solve(steps)
    dt = time.perf_counter() - t0
    n = len(scene["positions"])
    return {"value": n * steps / dt, "unit": "particle-steps/s", "cores": 1, "kind": "port",
            "sample": f"{n} particles ({config} particle region scaled {sample_scale:g} per axis, same grid), "
                      f"{steps} steps after {warmup} warm-up, serial C oracle (FP32)",
            "seconds": dt}


def run_reference(args, world, rank, pg):
    line = None
    if rank == 0:
        cb = cpu_reference(args.config, args.steps, args.warmup, args.ref_sample_scale)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "particle-steps/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * cb["seconds"] / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": workload_name(args.config), "sample": cb["sample"]},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    return line


def workload_name(config):
    return {"column": "granular column collapse 3D, Drucker-Prager, quadratic B-spline, 1,331,712 particles, "
                      "257x65x129 nodes, gravity + slip walls, dt 1e-5",
            "discs": "two-disc elastic impact 2D, linear, 2,528 particles, 51x51 nodes, dt 1e-3",
            "bed": "granular bed 3D with a translating, turning half-cylinder scoop (SDF contact, Coulomb 0.3), "
                   "Drucker-Prager, cubic B-spline, 4,915,200 particles, 241x97x129 nodes, dt 8e-6",
            "calibration": "differentiable calibration rollout: 3D Drucker-Prager cube, 262,144 particles "
                           "(64^3 lattice, h 1/128), quadratic, per-particle E and friction angle, 500 steps of "
                           "dt 2e-5, checkpoints every 25, forward + adjoint",
            "ensemble": "batched ensemble of 256 2D instances (column collapses and disc impacts, 2k-64k particles, "
                        "64^2-512^2 grids, LE / NF / DP cycled, per-instance CFL 0.3 dt), quadratic B-spline"
            }[config]


def run_ensemble(args, world, rank, local, pg, emit=True):
    """Batched ensemble: all instances stepped by one launch per phase, timed
    against one simulation handle per instance stepped one after another."""
    import torch

    from pyroclastmpm_b200 import Batch, Simulation, scenes

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    insts = scenes.ensemble()
    n = sum(len(sc["positions"]) for sc in insts)
    b = Batch(insts, device=local, stream=stream.cuda_stream, resort_interval=args.resort_interval).initialize()
    b.solve(args.warmup)
    if b.synchronize() != 0:
        raise RuntimeError("device fault during warm-up")
    barrier(pg)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    l0 = b.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    b.solve(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    clocks = sampler.stop()
    barrier(pg)
    launches = b.launch_count() - l0
    ms = allreduce_max(pg, ev0.elapsed_time(ev1))
    if b.synchronize() != 0:
        raise RuntimeError("device fault in the timed region")
    value = world * n * args.steps / (ms / 1000.0)
    phases = np.zeros(3)
    for _ in range(5):
        p, _nl = b.profile_step()
        phases += np.array(p)
    phases /= 5

    # one handle per instance, launched one after another on one stream
    sims = []
    for sc in insts:
        sim = Simulation(**scenes.sim_kwargs(sc), device=local, stream=stream.cuda_stream,
                         resort_interval=args.resort_interval)
        sim.set_particles(sc["positions"], sc["velocities"]).initialize()
        sims.append(sim)
    for sim in sims:
        sim.solve(args.warmup)
    base_steps = max(3, args.steps // 4)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(base_steps):
        for sim in sims:
            sim.solve(1)
    e1.record(stream)
    e1.synchronize()
    single_value = n * base_steps / (e0.elapsed_time(e1) / 1000.0)
    for sim in sims:
        sim.close()

    # end to end: every instance's positions and velocities up from pinned
    # host memory, one step, back again
    pins = [(torch.empty((len(sc["positions"]), 2), dtype=torch.float32, pin_memory=True),
             torch.empty((len(sc["positions"]), 2), dtype=torch.float32, pin_memory=True)) for sc in insts]
    for i, (px, pv) in enumerate(pins):
        px.copy_(torch.from_numpy(b.get(i, "positions")))
        pv.copy_(torch.from_numpy(b.get(i, "velocities")))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(1, args.e2e_steps // 2)
    for _ in range(e2e_steps):
        for i, (px, pv) in enumerate(pins):
            b.set_ptr(i, "positions", px.data_ptr(), px.numel() * 4)
            b.set_ptr(i, "velocities", pv.data_ptr(), pv.numel() * 4)
        b.solve(1)
        for i, (px, pv) in enumerate(pins):
            b.get_ptr(i, "positions", px.data_ptr(), px.numel() * 4)
            b.get_ptr(i, "velocities", pv.data_ptr(), pv.numel() * 4)
    torch.cuda.synchronize()
    e2e_s = allreduce_max(pg, (time.perf_counter() - t0) / e2e_steps)
    nbytes = n * 2 * 4 * 2

    peak, peak_kind = load_peak()
    st = 4
    algo = {"partition": n * st * 4 + sum(sc_nodes(sc) for sc in insts) * st * 2,
            "p2g": n * st * (2 + 2 + 1 + 1 + 4),
            "g2p_stress": n * st * (2 + 2 + 4 + 4 + 1 + (2 + 2 + 4 + 4 + 1)) + n}
    names = ["partition", "p2g", "g2p_stress"]
    dom = int(np.argmax(phases))
    achieved = algo[names[dom]] / (phases[dom] / 1000.0) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_ensemble(1, 16)
        cpu.pop("seconds", None)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, numpy PCG64 seed 3)",
            "config": {"workload": workload_name("ensemble"), "instances": len(insts), "particles_per_gpu": n,
                       "grid_nodes": int(sum(sc_nodes(sc) for sc in insts)), "resort_interval": args.resort_interval,
                       "l2": "state larger than L2 (no flush)", "parallelism": f"replicas x{world}",
                       "one_sim_per_launch": {"value": single_value, "unit": "particle-steps/s",
                                              "steps": base_steps,
                                              "note": "one pmpm_sim per instance, stepped in turn on one stream"},
                       "batched_over_one_sim_per_launch": value / single_value},
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs", "traffic": None,
                         "algorithmic_bytes_per_launch": algo[names[dom]], "ms_per_launch": float(phases[dom])},
            "phases_ms": dict(zip(names, [float(x) for x in phases])),
            "clocks": clocks, "gpu_launches": int(launches),
            "e2e": {"value": world * n / e2e_s, "unit": "particle-steps/s", "h2d_bytes_per_step": nbytes // 2,
                    "d2h_bytes_per_step": nbytes // 2,
                    "note": "per step: every instance's positions + velocities uploaded from pinned host memory, "
                            "one batched step, read back (host wall clock around synchronised calls)"},
            "cpu_baseline": cpu,
        }
        if emit:
            print(json.dumps(line), flush=True)
    b.close()
    return line if rank == 0 else None


def run_calibration(args, world, rank, local, pg, emit=True):
    """Differentiable calibration rollout: forward with checkpoints plus the
    adjoint, against the plain forward of the same rollout."""
    import torch

    from pyroclastmpm_b200 import Simulation, scenes

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    nsteps, every = args.rollout_steps, 25
    scene, E, phi, (tE, tphi) = scenes.calibration_cube()
    n = len(scene["positions"])
    kw = scenes.sim_kwargs(scene)
    # target rollout with the target parameters (the material's own)
    tgt = Simulation(**kw, device=local, stream=stream.cuda_stream)
    tgt.set_particles(scene["positions"], scene["velocities"]).initialize()
    tgt.solve(nsteps)
    target = tgt.get("positions").astype(np.float64)
    tgt.close()
    sim = Simulation(**kw, device=local, stream=stream.cuda_stream)
    sim.set_particles(scene["positions"], scene["velocities"]).initialize()
    sim.set("youngs_modulus", E)
    sim.set("friction_angle", phi)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    # warm-up: a short rollout and its adjoint
    for _ in range(max(1, args.warmup // 3)):
        sim.rollout_forward(2 * every, every)
        x = sim.get("positions")
        sim.rollout_backward(np.zeros_like(x))
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    # the plain forward of the same rollout (normal stepping, re-sorts on)
    plain = Simulation(**kw, device=local, stream=stream.cuda_stream)
    plain.set_particles(scene["positions"], scene["velocities"]).initialize()
    plain.set("youngs_modulus", E)
    plain.set("friction_angle", phi)
    plain.solve(args.warmup)
    ms_plain, _ = timed(lambda: plain.solve(nsteps))
    plain.close()
    # a full-length rollout and adjoint in each memory mode first (the kept
    # segments are allocated once and reused); each backward leaves `sim` at
    # the initial state
    for budget in (0, -1):
        sim.rollout_set_memory(budget)
        sim.rollout_forward(nsteps, every)
        sim.rollout_backward(np.zeros((n, 3), np.float32))
    l0 = sim.launch_count()
    ms_fwd, _ = timed(lambda: sim.rollout_forward(nsteps, every))
    x = sim.get("positions").astype(np.float64)
    loss = float(((x - target) ** 2).sum() / n)
    grad = (2.0 * (x - target) / n).astype(np.float32)
    ms_bwd, out = timed(lambda: sim.rollout_backward(grad))
    clocks = sampler.stop()
    launches = sim.launch_count() - l0
    if sim.synchronize() != 0:
        raise RuntimeError("device fault in the timed region")
    gE, gphi = out[0], out[1]
    # the same rollout with checkpoints alone (every segment recomputed)
    sim.rollout_set_memory(0)
    sim.rollout_forward(nsteps, every)  # frees the kept segments outside the timing
    sim.rollout_backward(grad)
    ms_fwd0, _ = timed(lambda: sim.rollout_forward(nsteps, every))
    ms_bwd0, _ = timed(lambda: sim.rollout_backward(grad))
    sim.rollout_set_memory(-1)
    ms_total = allreduce_max(pg, ms_fwd + ms_bwd)
    value = world * n * nsteps / (ms_total / 1000.0)
    # G2P-side adjoint traffic per particle-step: state in, adjoints in and out
    peak, peak_kind = load_peak()
    ms_adj_step = ms_bwd / nsteps
    adj_bytes = n * 4 * (28 + 2 * 27 + 2 * 27)
    achieved = adj_bytes / (ms_adj_step / 1000.0) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference("column", 1, 0, 0.3)
        cpu.pop("seconds", None)
        cpu["sample"] += " (forward only: the reference has no adjoint)"
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": nsteps,
            "warmup": args.warmup, "ms_per_step": ms_total / nsteps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (64^3 lattice cube, numpy PCG64 seed 2)",
            "config": {"workload": workload_name("calibration"), "particles_per_gpu": n,
                       "checkpoint_every": every, "parallelism": f"replicas x{world}",
                       "l2": "state larger than L2 (no flush)",
                       "plain_forward_ms_per_step": ms_plain / nsteps,
                       "rollout_forward_ms_per_step": ms_fwd / nsteps,
                       "adjoint_ms_per_step": ms_bwd / nsteps,
                       "fwd_plus_adjoint_over_plain_forward": (ms_fwd + ms_bwd) / ms_plain,
                       "segments": "kept whole from the forward pass where device memory allows (default "
                                   "budget: 60 % of free memory); checkpoints every 25 steps regardless",
                       "checkpoints_only": {"rollout_forward_ms_per_step": ms_fwd0 / nsteps,
                                            "adjoint_ms_per_step": ms_bwd0 / nsteps,
                                            "fwd_plus_adjoint_over_plain_forward": (ms_fwd0 + ms_bwd0) / ms_plain},
                       "loss": loss, "grad_norm_E": float(np.linalg.norm(gE)),
                       "grad_norm_phi": float(np.linalg.norm(gphi))},
            "roofline": {"bound": "hbm", "kernel": "adjoint step (4 kernels + recomputed P2G)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} hbm_gbs", "traffic": None,
                         "algorithmic_bytes_per_launch": adj_bytes, "ms_per_launch": ms_adj_step},
            "clocks": clocks, "gpu_launches": int(launches),
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": int(grad.nbytes // nsteps),
                    "d2h_bytes_per_step": int((gE.nbytes + gphi.nbytes + 4 * 3 * n) // nsteps),
                    "note": "rollout through the C ABI: loss gradient uploaded from host, parameter gradients "
                            "and final positions read back; per-step share of those bytes"},
            "cpu_baseline": cpu,
        }
        if emit:
            print(json.dumps(line), flush=True)
    sim.close()
    return line if rank == 0 else None


def sc_nodes(sc):
    n = 1
    for a in range(sc["dim"]):
        n *= int(np.float32(np.float32(sc["end"][a]) - np.float32(sc["origin"][a])) / np.float32(sc["cell_size"])) + 1
    return n


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="column", choices=["column", "discs", "bed", "ensemble", "calibration"])
    ap.add_argument("--rollout-steps", type=int, default=500)
    ap.add_argument("--resort-interval", type=int, default=32)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--ref-sample-scale", type=float, default=0.45)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--p2g-kernel", default="auto", choices=["auto", "dual", "cells"],
                    help="3D quadratic P2G kernel: autotuned (default) or fixed (fixed for profiling runs, "
                         "whose serialised launches make the autotuner's timings meaningless)")
    ap.add_argument("--no-companions", dest="companions", action="store_false",
                    help="skip the batched-ensemble and calibration legs in the default line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world, rank, local, pg = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return

    if args.config in ("ensemble", "calibration"):
        (run_ensemble if args.config == "ensemble" else run_calibration)(args, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return

    import torch

    from pyroclastmpm_b200 import Simulation, scenes

    torch.cuda.set_device(local)
    scene = scene_for(args.config)
    kw = scenes.sim_kwargs(scene)
    sim = Simulation(**kw, device=local, resort_interval=args.resort_interval)
    sim.set_particles(scene["positions"], scene["velocities"])
    sim.initialize()
    if args.p2g_kernel == "auto":
        p2g_variant = sim.autotune(3)  # the P2G kernel this configuration runs fastest with
    else:
        p2g_variant = {"dual": 1, "cells": 0}[args.p2g_kernel]
        sim.set_p2g_kernel(p2g_variant)
    n = sim.n
    stream = torch.cuda.ExternalStream(sim.stream, device=local)

    for _ in range(args.warmup):
        sim.solve(1)
    status = sim.synchronize()
    if status != 0:
        raise RuntimeError(f"device fault during warm-up: {status}")

    # ---- timed region: K steps, device time on the simulation's stream ----
    barrier(pg)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    launches0 = sim.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    sim.solve(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier(pg)
    launches = sim.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    ms_max = allreduce_max(pg, ms)
    status = sim.synchronize()
    if status != 0:
        raise RuntimeError(f"device fault in the timed region: {status}")
    value = world * n * args.steps / (ms_max / 1000.0)

    # ---- per-phase times (CUDA events inside the library, same stream) ----
    phases = np.zeros(3)
    nprof = 5
    for _ in range(nprof):
        p, _nl = sim.profile_step()
        phases += np.array(p)
    phases /= nprof
    active = sim.active_nodes()
    dim = scene["dim"]
    peak, peak_kind = load_peak()
    step_bytes = STEP_BYTES[("3d", "dp")] if dim == 3 else STEP_BYTES[("2d", "le")]
    grid_bytes = 16 * dim * active
    # algorithmic bytes per launch of each phase
    phase_names = ["partition", "p2g", "g2p_stress"]
    st = 4
    if dim == 3:
        p2g_bytes = n * st * (3 + 3 + 1 + 1 + 6) + active * st * 2 * dim
        g2p_bytes = n * st * (3 + 3 + 9 + 6 + 1 + (3 + 3 + 9 + 6 + 6 + 1)) + n * 1 + active * st * 2 * dim
    else:
        p2g_bytes = n * st * (2 + 2 + 1 + 1 + 4) + active * st * 2 * dim
        g2p_bytes = n * st * (2 + 2 + 4 + 4 + 1 + (2 + 2 + 4 + 4 + 1)) + n * 1 + active * st * 2 * dim
    part_bytes = n * st * (dim + 1 + 1) + sim.num_nodes * st * 2
    algo = {"partition": part_bytes, "p2g": p2g_bytes, "g2p_stress": g2p_bytes}
    dom = int(np.argmax(phases))
    dom_name = phase_names[dom]
    achieved = algo[dom_name] / (phases[dom] / 1000.0) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(args.config, {}).get(dom_name)
        except Exception:
            traffic = None
    step_ms = ms_max / args.steps
    step_achieved = (step_bytes * n + grid_bytes) / (step_ms / 1000.0) / 1e9

    # ---- end to end through the C ABI with host buffers ----
    pin_x = torch.empty((n, dim), dtype=torch.float32, pin_memory=True)
    pin_v = torch.empty((n, dim), dtype=torch.float32, pin_memory=True)
    pin_x.copy_(torch.from_numpy(sim.get("positions")))
    pin_v.copy_(torch.from_numpy(sim.get("velocities")))
    nbytes = n * dim * 4
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    def e2e_step():
        sim.set_ptr("positions", pin_x.data_ptr(), nbytes)
        sim.set_ptr("velocities", pin_v.data_ptr(), nbytes)
        sim.solve(1)
        sim.get_ptr("positions", pin_x.data_ptr(), nbytes)
        sim.get_ptr("velocities", pin_v.data_ptr(), nbytes)

    for _ in range(2):  # untimed: first-use staging buffers and transfers
        e2e_step()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.e2e_steps):
        sim.set_ptr("positions", pin_x.data_ptr(), nbytes)
        sim.set_ptr("velocities", pin_v.data_ptr(), nbytes)
        sim.solve(1)
        sim.get_ptr("positions", pin_x.data_ptr(), nbytes)
        sim.get_ptr("velocities", pin_v.data_ptr(), nbytes)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = allreduce_max(pg, e0.elapsed_time(e1) / args.e2e_steps)
    e2e_value = world * n / (e2e_ms / 1000.0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference(args.config, args.cpu_steps, 0, 1.0)
        cpu.pop("seconds", None)

    # the metric's other two legs, measured by their own configurations
    companions = None
    if args.companions and args.config == "column":
        sim.close()
        sub = argparse.Namespace(**vars(args))
        sub.no_cpu_baseline = True
        sub.steps = 10
        cal = run_calibration(sub, world, rank, local, pg, emit=False)
        ens = run_ensemble(sub, world, rank, local, pg, emit=False)
        if rank == 0:
            companions = {
                "batched": {"value": ens["value"], "unit": "particle-steps/s", "workload": ens["config"]["workload"],
                            "ms_per_step": ens["ms_per_step"],
                            "over_one_sim_per_launch": ens["config"]["batched_over_one_sim_per_launch"]},
                "fwd_adjoint": {"value": cal["value"], "unit": "particle-steps/s",
                                "workload": cal["config"]["workload"], "ms_per_step": cal["ms_per_step"],
                                "plain_forward_ms_per_step": cal["config"]["plain_forward_ms_per_step"],
                                "rollout_forward_ms_per_step": cal["config"]["rollout_forward_ms_per_step"],
                                "adjoint_ms_per_step": cal["config"]["adjoint_ms_per_step"],
                                "over_plain_forward": cal["config"]["fwd_plus_adjoint_over_plain_forward"],
                                "checkpoints_only_over_plain_forward":
                                    cal["config"]["checkpoints_only"]["fwd_plus_adjoint_over_plain_forward"],
                                "clocks": cal.get("clocks")},
            }

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded lattice, numpy PCG64)",
            "config": {"workload": workload_name(args.config), "particles_per_gpu": n, "grid_nodes": sim.num_nodes,
                       "active_nodes": active, "resort_interval": args.resort_interval,
                       "p2g_kernel": p2g_kernel_name(kw, p2g_variant),
                       "l2": "state larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "traffic": traffic, "algorithmic_bytes_per_launch": algo[dom_name],
                         "ms_per_launch": float(phases[dom])},
            "step_roofline": {"achieved": step_achieved, "peak": peak, "unit": "GB/s",
                              "frac": step_achieved / peak,
                              "bytes_per_particle_step": step_bytes, "grid_bytes_per_step": grid_bytes},
            "phases_ms": dict(zip(phase_names, [float(x) for x in phases])),
            "clocks": clocks, "gpu_launches": int(launches),
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": 2 * nbytes,
                    "d2h_bytes_per_step": 2 * nbytes,
                    "note": "per step: positions + velocities uploaded from pinned host memory, one step, "
                            "positions + velocities read back"},
            "cpu_baseline": cpu,
        }
        if companions:
            line["companions"] = companions
        print(json.dumps(line), flush=True)
    sim.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
