"""Batched ensembles (pmpm_batch): every instance must give what a single
simulation of the same scene gives, and agree with the oracle.

With the deterministic flag both paths sum P2G contributions in the same
fixed order, so the batch must match the single simulations bit for bit.
"""
import numpy as np
import pytest

import oracle
from pyroclastmpm_b200 import scenes
from pyroclastmpm_b200._capi import Batch, Simulation

pytestmark = pytest.mark.gpu

FIELDS = ("positions", "velocities", "stresses", "F", "volumes", "masses")


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def small_ensemble(num=8, seed=4, shape_function="quadratic"):
    return scenes.ensemble(num=num, seed=seed, shape_function=shape_function, np_range=(400, 3000),
                           grid_range=(24, 80))


def single(sc, flags, steps):
    sim = Simulation(**scenes.sim_kwargs(sc), flags=flags)
    sim.set_particles(sc["positions"], sc["velocities"], sc.get("colors")).initialize()
    sim.solve(steps)
    assert sim.synchronize() == 0
    return sim


@pytest.mark.parametrize("shape_function", ["linear", "quadratic", "cubic"])
def test_batch_bitwise_equals_single_simulations(shape_function):
    insts = small_ensemble(shape_function=shape_function)
    b = Batch(insts, flags=2, resort_interval=3).initialize()
    b.solve(7)
    assert b.synchronize() == 0
    for i, sc in enumerate(insts):
        sim = single(sc, 2, 7)  # resort_interval 32: storage order does not change the sums
        for name in FIELDS:
            np.testing.assert_array_equal(b.get(i, name), sim.get(name), err_msg=f"instance {i} {name}")
        np.testing.assert_array_equal(b.get(i, "node_masses"), sim.get("node_masses"))
        np.testing.assert_array_equal(b.get(i, "node_moments_nt"), sim.get("node_moments_nt"))


def test_batch_matches_oracle_per_instance():
    insts = small_ensemble(num=6, seed=9)
    b = Batch(insts).initialize()
    b.solve(3)
    assert b.synchronize() == 0
    for i, sc in enumerate(insts):
        refs = [oracle.OracleSim(**scenes.sim_kwargs(sc), positions=sc["positions"], velocities=sc["velocities"],
                                 precision=p).initialize() for p in ("f32", "f64")]
        for r in refs:
            r.solve(3)
        for name in ("positions", "velocities", "stresses"):
            tol = max(1e-5, 3.0 * rel(refs[0][name], refs[1][name]))
            err = rel(b.get(i, name), refs[0][name])
            assert err <= tol, f"instance {i} {name}: {err:.2e} > {tol:.1e}"


def test_batch_dynamic_bcs_and_set_field():
    """Instances with a gravity ramp and a moving rigid body (per-step view
    updates), stresses set before initialisation, against single handles."""
    insts = small_ensemble(num=4, seed=12)
    insts[0]["bcs"] = [{"type": "Gravity", "gravity": [0.0, -9.81], "is_ramp": True, "ramp_step": 4,
                        "gravity_end": [0.0, -9.81]}] + insts[0]["bcs"]
    insts[3]["bcs"] = insts[3]["bcs"] + [{"type": "RigidBodyLevelSet", "shape": "sphere", "center": [0.41, 0.23],
                                          "velocity": [0.0, 0.3], "dims": [0.1311, 0, 0], "friction": 0.2}]
    rng = np.random.default_rng(1)
    stress = rng.normal(0, 10.0, (len(insts[1]["positions"]), 3, 3))
    stress = 0.5 * (stress + stress.transpose(0, 2, 1))
    stress[:, 2, :2] = stress[:, :2, 2] = 0
    b = Batch(insts, flags=2)
    b.set(1, "stresses", stress)
    b.initialize()
    b.solve(6)
    assert b.synchronize() == 0
    for i, sc in enumerate(insts):
        sim = Simulation(**scenes.sim_kwargs(sc), flags=2)
        sim.set_particles(sc["positions"], sc["velocities"])
        if i == 1:
            sim.set("stresses", stress)
        sim.initialize()
        sim.solve(6)
        for name in FIELDS:
            np.testing.assert_array_equal(b.get(i, name), sim.get(name), err_msg=f"instance {i} {name}")


def test_batch_out_of_domain_is_reported_and_contained():
    insts = small_ensemble(num=3, seed=5)
    v = insts[1]["velocities"].copy()
    v[0] = [-1e6, 0.0]  # leaves the grid on the first step
    insts[1]["velocities"] = v
    b = Batch(insts, flags=2).initialize()
    b.solve(2)
    assert b.synchronize() == 16  # PMPM_ERR_OUT_OF_DOMAIN
    for i in (0, 2):
        sim = single(insts[i], 2, 2)
        for name in FIELDS:
            np.testing.assert_array_equal(b.get(i, name), sim.get(name), err_msg=f"instance {i} {name}")
