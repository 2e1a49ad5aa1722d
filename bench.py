"""Benchmark of the USL MPM step: particle-steps/s on B200.

Default workload: the 3D granular bed dug by a rigid scoop (4,915,200
particles, cubic B-splines, Drucker-Prager, half-cylinder shell contact with
Coulomb friction, gravity, slip walls, 241x97x129 nodes, dt 8e-6), the
largest configuration and the one the plain-step roofline target is stated
on; the granular column (1,331,712 particles, quadratic), the batched
ensemble and the forward + adjoint rollout follow as companion legs.
Synthetic, seeded particle sets (numpy PCG64).  The particle state is larger
than the 126 MB L2, so no flush is needed between timed steps.

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
    """The oracle (C restatement of the reference step, one thread) on the
    workload, or with sample_scale < 1 on a bounded sample of it: the same
    grid, the particle region scaled by sample_scale per axis."""
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
    what = "the full workload" if sample_scale == 1.0 else \
        f"{config} particle region scaled {sample_scale:g} per axis, same grid"
    return {"value": n * steps / dt, "unit": "particle-steps/s", "cores": 1, "kind": "port",
            "sample": f"{n} particles ({what}), {steps} steps after {warmup} warm-up, serial C oracle (FP32)",
            "seconds": dt}


def workload_name(config):
    return {"column": "granular column collapse 3D, Drucker-Prager, quadratic B-spline, 1,331,712 particles, "
                      "257x65x129 nodes, gravity + slip walls, dt 1e-5",
            "discs": "two-disc elastic impact 2D, linear, 2,528 particles, 51x51 nodes, dt 1e-3",
            "bed": "granular bed 3D dug by a translating, turning half-cylinder scoop (R 0.15, t 0.01, L 0.4; "
                   "SDF contact, Coulomb 0.3), Drucker-Prager, cubic B-spline, 4,915,200 particles, "
                   "241x97x129 nodes, gravity + slip walls, dt 8e-6",
            "calibration": "differentiable calibration rollout: 3D Drucker-Prager cube, 262,144 particles "
                           "(64^3 lattice, h 1/128), quadratic, per-particle E and friction angle, 500 steps of "
                           "dt 2e-5, checkpoints every 25, forward + adjoint",
            "ensemble": "batched ensemble of 256 2D instances (column collapses and disc impacts, 2k-64k particles, "
                        "64^2-512^2 grids, LE / NF / DP cycled, per-instance CFL 0.3 dt), quadratic B-spline"
            }[config]


def static_config(config, world):
    """The workload's description: the same for both arms (nothing measured)."""
    from pyroclastmpm_b200 import scenes

    if config in ("ensemble", "calibration"):
        return {"workload": workload_name(config), "parallelism": f"replicas x{world}"}
    scene = scene_for(config)
    return {"workload": workload_name(config), "particles_per_gpu": int(len(scene["positions"])),
            "grid_nodes": int(sc_nodes(scene)), "l2": "state larger than L2 (no flush)",
            "parallelism": f"replicas x{world}"}


def run_reference(args, world, rank, pg):
    """The reference arm: the reference step (the oracle's C restatement, one
    thread as the reference's CPU build) on the same workload and particle
    count as the B200 arm, for a few steps (about 50 s per step of the bed)."""
    line = None
    if rank == 0:
        steps, warmup = max(1, min(args.steps, args.ref_steps)), max(0, min(args.warmup, args.ref_warmup))
        cb = cpu_reference(args.config, steps, warmup, 1.0)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "particle-steps/s",
                "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
                "ms_per_step": 1000.0 * cb["seconds"] / steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": static_config(args.config, world),
                "cpu_baseline": {k: v for k, v in cb.items() if k != "seconds"},
                "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "note": f"timed {steps} steps after {warmup} warm-up (the --steps/--warmup asked for, capped at "
                        f"--ref-steps {args.ref_steps} / --ref-warmup {args.ref_warmup}: one serial step of this "
                        "workload takes tens of seconds)"}
        print(json.dumps(line), flush=True)
    return line


def rel_err_fields(gpu_get, ref, names):
    out = {}
    for name in names:
        a = np.asarray(gpu_get(name), np.float64)
        b = np.asarray(ref[name], np.float64)
        out[name] = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
    return out


def summarise_err(err, floor):
    """value: the largest error over the fields the reference's own FP32
    arithmetic resolves to 1e-4 of FP64 (the FP32 oracle's distance); fields
    it does not (FP32 rounding noise in a quantity near zero, such as the
    Tait pressure of a fluid at rest) are listed apart, each with the ratio
    of the GPU's error to the FP32 oracle's."""
    good = [k for k in err if floor[k] <= 1e-4]
    ill = {k: {"gpu": err[k], "fp32_oracle": floor[k], "ratio": err[k] / max(floor[k], 1e-30)}
           for k in err if floor[k] > 1e-4}
    return {"value": max([err[k] for k in good], default=None), "per_field": err, "fp32_oracle_vs_fp64": floor,
            "ill_conditioned": ill}


def plain_rel_err(config, local, steps=5, scale=None):
    """Error of the GPU step against the FP64 oracle on a bounded sample of
    the workload (same grid and physics, the particle region scaled), after
    `steps` steps: max |a - b| / max |b| per field; the FP32 oracle's own
    distance from FP64 beside it (what the reference's FP32 arithmetic
    reaches).  Outside any timed region."""
    import oracle
    from pyroclastmpm_b200 import Simulation, scenes

    scale = scale if scale is not None else {"bed": 0.35, "column": 0.5, "discs": 1.0}[config]
    scene = scene_for(config, scale=scale)
    kw = scenes.sim_kwargs(scene)
    sim = Simulation(**kw, device=local)
    sim.set_particles(scene["positions"], scene["velocities"]).initialize()
    sim.solve(steps)
    if sim.synchronize() != 0:
        raise RuntimeError("device fault in the error check")
    names = ("positions", "velocities", "stresses")
    refs = {p: oracle.OracleSim(**kw, positions=scene["positions"], velocities=scene["velocities"],
                                precision=p).initialize() for p in ("f64", "f32")}
    for r in refs.values():
        r.solve(steps)
    err = rel_err_fields(sim.get, refs["f64"], names)
    floor = rel_err_fields(lambda nm: refs["f32"][nm], refs["f64"], names)
    sim.close()
    return {**summarise_err(err, floor), "steps": steps,
            "sample": f"{len(scene['positions'])} particles ({config} particle region scaled {scale:g} per axis, "
                      f"same grid), {steps} steps, FP64 C oracle",
            "measure": "max |gpu - fp64| / max |fp64| per field (positions, velocities, stresses)"}


# FP32 flops per particle-step, counted from the algorithm (not the
# instruction stream): per (particle, node) pair of P2G the weight and its
# gradient (D - 1 + D (D - 1) products), mass and momentum (2 + 2D), the
# stress force -V sigma grad N (2 D^2 + D); per pair of G2P the weight and
# gradient again, the FLIP increment (3D), the PIC velocity (2D) and the
# velocity gradient (2 D^2); per particle the spline pieces of both maps
# (2 D WIN evaluations of N and dN), and the particle-local update (FLIP/PIC
# blend, position, F = (I + L dt) F, det F, the return mapping) as a lump.
SPLINE_FLOPS = {"linear": 3, "quadratic": 6, "cubic": 11}
WIN = {"linear": 2, "quadratic": 3, "cubic": 4}
LOCAL_FLOPS = {2: 100, 3: 330}
NODE_FLOPS = 18  # per active node: p_nt = p + f dt, v = p / m, v_nt, conditions


def flops_per_particle(dim, sf):
    nsn = WIN[sf] ** dim
    p2g_pair = (dim - 1) + dim * (dim - 1) + 2 + 2 * dim + 2 * dim * dim + dim
    g2p_pair = (dim - 1) + dim * (dim - 1) + 3 * dim + 2 * dim + 2 * dim * dim
    weights = dim * WIN[sf] * SPLINE_FLOPS[sf]
    return {"p2g": nsn * p2g_pair + weights, "g2p_stress": nsn * g2p_pair + weights + LOCAL_FLOPS[dim],
            "step": nsn * (p2g_pair + g2p_pair) + 2 * weights + LOCAL_FLOPS[dim]}


def fp32_peak_tflops(sm_mhz):
    """148 SMs x 128 FP32 lanes x 2 flops (FMA) per clock."""
    return 148 * 128 * 2 * sm_mhz * 1e6 / 1e12


def ensemble_rel_err(local, picks=(0, 1, 2, 3, 4, 5), steps=20):
    """Error of batched instances against the FP64 oracle: one instance of
    each scene and material kind stepped in a batch of their own (the same
    kernels) for `steps` steps; max over instances and fields, the FP32
    oracle's own distance beside it."""
    import oracle
    from pyroclastmpm_b200 import Batch, scenes

    insts = scenes.ensemble()
    sel = [insts[i] for i in picks]
    b = Batch(sel, device=local).initialize()
    b.solve(steps)
    if b.synchronize() != 0:
        raise RuntimeError("device fault in the error check")
    names = ("positions", "velocities", "stresses")
    err, floor = {}, {}
    for k, sc in enumerate(sel):
        kw = scenes.sim_kwargs(sc)
        refs = {p: oracle.OracleSim(**kw, positions=sc["positions"], velocities=sc["velocities"],
                                    precision=p).initialize() for p in ("f64", "f32")}
        for r in refs.values():
            r.solve(steps)
        e = rel_err_fields(lambda nm: b.get(k, nm), refs["f64"], names)
        f = rel_err_fields(lambda nm: refs["f32"][nm], refs["f64"], names)
        for nm in names:
            key = f"{nm}[{picks[k]}]"
            err[key], floor[key] = e[nm], f[nm]
    b.close()
    return {**summarise_err(err, floor), "steps": steps,
            "sample": f"ensemble instances {list(picks)} (LE / NF / DP, columns and discs) in one batch, "
                      f"{steps} steps, FP64 C oracle per instance",
            "measure": "max |gpu - fp64| / max |fp64| per field and instance (field[instance])"}


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
    err = ensemble_rel_err(local) if rank == 0 and args.error_check else None
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
            "rel_err_vs_fp64": err,
            "cpu_baseline": cpu,
        }
        if emit:
            print(json.dumps(line), flush=True)
    b.close()
    return line if rank == 0 else None


def calibration_rel_err(local, steps=50, every=10, eps=1e-4):
    """Errors of the differentiable rollout on the 4,096-particle copy of the
    calibration cube (16^3 lattice): final positions of the forward rollout
    against the FP64 oracle, and the adjoint's directional derivatives of
    the loss w . x_final (fixed random w) along random perturbations of the
    per-particle E and friction angle against FP64 central differences."""
    import oracle
    from pyroclastmpm_b200 import Simulation, scenes

    scene, E, phi, _ = scenes.calibration_cube(n_side=16, cell_size=1.0 / 32, domain=0.5, dt=1e-4)
    n = len(scene["positions"])
    kw = scenes.sim_kwargs(scene)
    sim = Simulation(**kw, device=local)
    sim.set_particles(scene["positions"], scene["velocities"]).initialize()
    sim.set("youngs_modulus", E)
    sim.set("friction_angle", phi)
    sim.rollout_forward(steps, every)
    x_gpu = sim.get("positions")
    w = np.random.default_rng(7).normal(0, 1, (n, 3))
    gE, gphi, _gx, _gv = sim.rollout_backward(w)
    if sim.synchronize() != 0:
        raise RuntimeError("device fault in the error check")
    sim.close()

    def final(Ep, phip, precision="f64"):
        o = oracle.OracleSim(**kw, positions=scene["positions"], velocities=scene["velocities"],
                             youngs_modulus=Ep, friction_angle=phip, precision=precision).initialize()
        o.solve(steps)
        return np.array(o["positions"], np.float64)

    x64 = final(E, phi)
    x32 = final(E, phi, "f32")
    fwd = float(np.abs(x_gpu - x64).max() / np.abs(x64).max())
    fwd_floor = float(np.abs(x32 - x64).max() / np.abs(x64).max())
    rng = np.random.default_rng(0)
    dE = E * rng.normal(0, 1, n)
    dphi = rng.normal(0, 1, n)
    grads = {}
    for name, adj, run in (("E", float(np.dot(gE.astype(np.float64), dE)),
                            lambda e: final(E + e * dE, phi)),
                           ("friction_angle", float(np.dot(gphi.astype(np.float64), dphi)),
                            lambda e: final(E, phi + e * dphi))):
        fd = (float((w * run(eps)).sum()) - float((w * run(-eps)).sum())) / (2 * eps)
        grads[name] = abs(adj - fd) / max(abs(fd), 1e-30)
    return {"value": max([fwd] + list(grads.values())), "forward_positions": fwd,
            "fp32_oracle_forward_positions": fwd_floor, "gradient_directional": grads,
            "sample": f"4,096-particle copy of the cube (16^3 lattice, h 1/32, dt 1e-4), {steps} steps, "
                      f"checkpoints every {every}; FP64 C oracle, central differences with step {eps:g}",
            "measure": "forward: max |gpu - fp64| / max |fp64| of final positions; gradients: |adjoint - FD| / "
                       "|FD| of directional derivatives"}


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
        cpu = cpu_reference("column", 3, 1, 0.3)
        cpu.pop("seconds", None)
        cpu["sample"] += " (forward only: the reference has no adjoint)"
    err = calibration_rel_err(local) if rank == 0 and args.error_check else None
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
            "rel_err_vs_fp64": err,
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


def run_plain(args, config, world, rank, local, pg, steps, with_cpu, with_err=True):
    """One simulation per GPU: K device-timed steps, phase split, rooflines,
    end to end through the C ABI, error against FP64, CPU baseline."""
    import torch

    from pyroclastmpm_b200 import Simulation, scenes

    torch.cuda.set_device(local)
    scene = scene_for(config, scale=args.scale)
    kw = scenes.sim_kwargs(scene)
    sim = Simulation(**kw, device=local, resort_interval=args.resort_interval)
    sim.set_particles(scene["positions"], scene["velocities"])
    sim.initialize()
    if args.p2g_kernel == "auto" and args.staging == "auto":
        # P2G kernel, staging and re-sort interval this configuration runs fastest with
        p2g_variant = sim.autotune(3)
    else:
        # fixed choices (profiling runs, whose serialised launches make the
        # autotuner's timings meaningless)
        if args.p2g_kernel != "auto":
            sim.set_p2g_kernel({"dual": 1, "cells": 0}[args.p2g_kernel])
        if args.staging != "auto":
            sim.set_p2g_staging({"bulk": 1, "gather": 0}[args.staging])
    tuning = sim.tuning()
    p2g_variant = tuning["p2g_kernel"]
    n = sim.n
    dim = scene["dim"]
    sf = scene["shape_function"]
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
    sim.solve(steps)
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
    value = world * n * steps / (ms_max / 1000.0)

    # ---- per-phase times (CUDA events inside the library, same stream) ----
    phases = np.zeros(3)
    nprof = 5
    for _ in range(nprof):
        p, _nl = sim.profile_step()
        phases += np.array(p)
    phases /= nprof
    active = sim.active_nodes()
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
            traffic = json.load(open(tpath)).get(config, {}).get(dom_name)
        except Exception:
            traffic = None
    step_ms = ms_max / steps
    step_achieved = (step_bytes * n + grid_bytes) / (step_ms / 1000.0) / 1e9
    # FP32 flops against the SIMT peak at the sampled clock
    fl = flops_per_particle(dim, sf)
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    fpeak = fp32_peak_tflops(sm_mhz)
    dom_flops = n * fl.get(dom_name, 0) + (active * NODE_FLOPS if dom_name == "p2g" else 0)
    dom_tflops = dom_flops / (phases[dom] / 1000.0) / 1e12
    step_tflops = (n * fl["step"] + active * NODE_FLOPS) / (step_ms / 1000.0) / 1e12

    # ---- end to end through the C ABI with host buffers (host wall clock) ----
    pin_x = torch.empty((n, dim), dtype=torch.float32, pin_memory=True)
    pin_v = torch.empty((n, dim), dtype=torch.float32, pin_memory=True)
    pin_x.copy_(torch.from_numpy(sim.get("positions")))
    pin_v.copy_(torch.from_numpy(sim.get("velocities")))
    nbytes = n * dim * 4

    def e2e_step():
        sim.set_ptr("positions", pin_x.data_ptr(), nbytes)
        sim.set_ptr("velocities", pin_v.data_ptr(), nbytes)
        sim.solve(1)
        sim.get_ptr("positions", pin_x.data_ptr(), nbytes)   # returns after the copy: synchronous
        sim.get_ptr("velocities", pin_v.data_ptr(), nbytes)

    for _ in range(2):  # untimed: first-use staging buffers and transfers
        e2e_step()
    torch.cuda.synchronize()
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = allreduce_max(pg, 1000.0 * (time.perf_counter() - t0) / args.e2e_steps)
    e2e_value = world * n / (e2e_ms / 1000.0)
    sim.close()

    err = None
    if with_err and rank == 0:
        err = plain_rel_err(config, local)
    cpu = None
    if with_cpu and rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference(config, args.cpu_steps, 1, args.cpu_sample_scale.get(config, 1.0))
        cpu.pop("seconds", None)

    if rank != 0:
        return None
    return {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded lattice, numpy PCG64)",
        "config": static_config(config, world),
        "tuned": {"p2g_kernel": p2g_kernel_name(kw, p2g_variant),
                  "p2g_staging": {1: "bulk copies of sorted records (cp.async.bulk + mbarrier)",
                                  0: "gather through the sorted order", -1: None}[tuning["staging"]],
                  "resort_interval": tuning["resort_interval"],
                  "by": "pmpm_autotune" if args.p2g_kernel == "auto" and args.staging == "auto" else "fixed"},
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                     "traffic": traffic, "algorithmic_bytes_per_launch": algo[dom_name],
                     "ms_per_launch": float(phases[dom])},
        "flop_roofline": {"bound": "fp32", "kernel": dom_name, "achieved": dom_tflops, "peak": fpeak,
                          "unit": "TFLOP/s", "frac": dom_tflops / fpeak, "flops_per_launch": dom_flops,
                          "peak_source": f"148 SMs x 128 FP32 lanes x 2 flops x sampled SM clock {sm_mhz:g} MHz"},
        "step_roofline": {"achieved": step_achieved, "peak": peak, "unit": "GB/s",
                          "frac": step_achieved / peak, "bytes_per_particle_step": step_bytes,
                          "grid_bytes_per_step": grid_bytes, "active_nodes": active,
                          "fp32_tflops": step_tflops, "fp32_frac": step_tflops / fpeak,
                          "flops_per_particle_step": fl["step"]},
        "phases_ms": dict(zip(phase_names, [float(x) for x in phases])),
        "clocks": clocks, "gpu_launches": int(launches),
        "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": 2 * nbytes,
                "d2h_bytes_per_step": 2 * nbytes,
                "note": "per step: positions + velocities uploaded from pinned host memory through "
                        "pmpm_set_field, one step, both read back through pmpm_get_field; host wall clock"},
        "rel_err_vs_fp64": err,
        "cpu_baseline": cpu,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="bed", choices=["column", "discs", "bed", "ensemble", "calibration"])
    ap.add_argument("--rollout-steps", type=int, default=500)
    ap.add_argument("--resort-interval", type=int, default=32)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--ref-steps", type=int, default=2,
                    help="most steps the reference arm times (one serial step of the bed takes ~50 s)")
    ap.add_argument("--ref-warmup", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="profiling runs only: the particle region scaled per axis (same grid); the line's config "
                         "still names the full workload")
    ap.add_argument("--no-error-check", dest="error_check", action="store_false",
                    help="skip the FP64 error checks (profiling runs)")
    ap.add_argument("--staging", default="auto", choices=["auto", "bulk", "gather"],
                    help="3D sweep P2G staging: autotuned (default) or fixed")
    ap.add_argument("--p2g-kernel", default="auto", choices=["auto", "dual", "cells"],
                    help="3D quadratic P2G kernel: autotuned (default) or fixed (fixed for profiling runs, "
                         "whose serialised launches make the autotuner's timings meaningless)")
    ap.add_argument("--no-companions", dest="companions", action="store_false",
                    help="skip the column, batched-ensemble and calibration legs in the default line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    # cpu_baseline samples: the same grid, the particle region scaled per axis
    # so that one warm-up step and --cpu-steps steps take about half a minute
    args.cpu_sample_scale = {"bed": 0.5, "column": 0.75, "discs": 1.0}

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

    line = run_plain(args, args.config, world, rank, local, pg, args.steps, with_cpu=True,
                     with_err=args.error_check)
    # the metric's other legs, measured by their own configurations
    if args.companions and args.config == "bed":
        sub = argparse.Namespace(**vars(args))
        sub.no_cpu_baseline = True
        col = run_plain(sub, "column", world, rank, local, pg, args.steps, with_cpu=False,
                        with_err=args.error_check)
        sub.steps = 10
        cal = run_calibration(sub, world, rank, local, pg, emit=False)
        ens = run_ensemble(sub, world, rank, local, pg, emit=False)
        if rank == 0:
            line["companions"] = {
                "column": {"value": col["value"], "unit": "particle-steps/s", "workload": col["config"]["workload"],
                           "ms_per_step": col["ms_per_step"], "phases_ms": col["phases_ms"],
                           "roofline": col["roofline"], "flop_roofline": col["flop_roofline"],
                           "step_roofline": col["step_roofline"], "e2e": col["e2e"],
                           "rel_err_vs_fp64": col["rel_err_vs_fp64"], "tuned": col["tuned"]},
                "batched": {"value": ens["value"], "unit": "particle-steps/s", "workload": ens["config"]["workload"],
                            "ms_per_step": ens["ms_per_step"],
                            "over_one_sim_per_launch": ens["config"]["batched_over_one_sim_per_launch"],
                            "rel_err_vs_fp64": ens.get("rel_err_vs_fp64")},
                "fwd_adjoint": {"value": cal["value"], "unit": "particle-steps/s",
                                "workload": cal["config"]["workload"], "ms_per_step": cal["ms_per_step"],
                                "plain_forward_ms_per_step": cal["config"]["plain_forward_ms_per_step"],
                                "rollout_forward_ms_per_step": cal["config"]["rollout_forward_ms_per_step"],
                                "adjoint_ms_per_step": cal["config"]["adjoint_ms_per_step"],
                                "over_plain_forward": cal["config"]["fwd_plus_adjoint_over_plain_forward"],
                                "checkpoints_only_over_plain_forward":
                                    cal["config"]["checkpoints_only"]["fwd_plus_adjoint_over_plain_forward"],
                                "rel_err_vs_fp64": cal.get("rel_err_vs_fp64"),
                                "clocks": cal.get("clocks")},
            }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
