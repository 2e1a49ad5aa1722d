"""Modified Cam Clay and Drucker-Prager cap on the sm_100a path against the
CPU oracle.

Two levels, as the reference's constitutive analyses and its USL solver use
the material: repeated stress updates of material points under fixed
velocity gradients (the history of elastic strain, alpha and pc builds up
over the updates), and full USL steps of a prestressed block under gravity
in 2D and 3D.  Tolerance per field: 1e-5 relative, or three times the FP32
oracle's distance from the FP64 oracle where that is larger (the reference's
FP32 Newton iteration stops on its growing bound, within FP32 noise of the
root the FP64 iteration finds).
"""
import numpy as np
import pytest

import oracle
from pyroclastmpm_b200 import Simulation

from test_dpc_oracle import DPC
from test_mcc_oracle import MCC, assert_strain_close

MATERIALS = {"mcc": MCC, "dpc": DPC}

pytestmark = pytest.mark.gpu

BASE = 1e-5


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def block(dim, shape_function, seed=3, R=1.0, n=None, material="mcc"):
    rng = np.random.default_rng(seed)
    n = n or (4000 if dim == 3 else 2000)
    h = 0.1
    V = h ** dim / (2 ** dim)
    g = [0.0] * dim
    g[-1] = -9.81
    return dict(dim=dim, origin=[0.0] * dim, end=[1.0] * dim, cell_size=h, shape_function=shape_function,
                dt=1e-4, particles_per_cell=2 ** dim, alpha=0.99,
                materials=[dict(MATERIALS[material], Vs=V / 1.8, R=R)],
                bcs=[{"type": "Gravity", "gravity": g},
                     {"type": "NodeDomain", "face0_mode": [1] * dim, "face1_mode": [1] * dim}],
                positions=rng.uniform(0.15, 0.85, (n, dim)), velocities=rng.normal(0, 0.2, (n, dim)),
                stresses=np.broadcast_to(-5e3 * np.eye(3), (n, 3, 3)).copy())


def sim_kw(scene):
    return {k: scene[k] for k in ("dim", "origin", "end", "cell_size", "shape_function", "dt",
                                  "particles_per_cell", "alpha", "materials", "bcs")}


def make_gpu(scene):
    sim = Simulation(**sim_kw(scene))
    sim.set_particles(scene["positions"], scene["velocities"])
    sim.set("stresses", scene["stresses"])
    return sim.initialize()


def make_oracle(scene, precision):
    return oracle.OracleSim(**sim_kw(scene), positions=scene["positions"], velocities=scene["velocities"],
                            stresses=scene["stresses"], precision=precision).initialize()


def point_loads(n, dim, seed):
    """Velocity gradients (1/s): shear with some compression.  Sustained
    extension drives the pressure to zero, where the ellipse (no tensile
    strength, Pt = 0) degenerates and the reference's iteration stops
    converging; those states are left out."""
    rng = np.random.default_rng(seed)
    L = rng.normal(0, 0.3, (n, dim, dim))
    L -= (np.trace(L, axis1=1, axis2=2) / dim)[:, None, None] * np.eye(dim)
    L -= rng.uniform(0.02, 0.3, n)[:, None, None] * np.eye(dim)
    L[: n // 3] -= 0.5 * np.eye(dim)  # compression: on to the cap
    L[n // 3: n // 2] *= 0.05         # nearly elastic
    return L


def run_points(obj, L, updates, on_gpu):
    for _ in range(updates):
        if on_gpu:
            obj.set("velocity_gradient", L)
            obj.stress_update()
        else:
            obj["velocity_gradient"][:] = L
            obj.call("or_stress_update")


HISTORY = ("stresses", "pc", "alpha")


def oracle_fields(o):
    return {"stresses": o["stresses"], "pc": o["pc"], "alpha": o["acc_eps_p"], "eps_e": o["eps_e"],
            "positions": o["positions"], "velocities": o["velocities"], "F": o["F"], "volumes": o["volumes"]}


@pytest.mark.parametrize("material", ["mcc", "dpc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_material_point_updates_match_oracle(dim, material):
    scene = block(dim, "linear", seed=5 + dim, R=1.1, material=material)
    n = len(scene["positions"])
    L = point_loads(n, dim, seed=dim)
    sim = make_gpu(scene)
    np.testing.assert_allclose(sim.get("pc"), 5.5e3, rtol=1e-6)
    np.testing.assert_array_equal(sim.get("stress_ref"), scene["stresses"].astype(np.float32))
    refs = {p: make_oracle(scene, p) for p in ("f32", "f64")}
    for o in refs.values():
        run_points(o, L, 30, False)
    run_points(sim, L, 30, True)
    f32, f64 = oracle_fields(refs["f32"]), oracle_fields(refs["f64"])
    got = {"stresses": sim.get("stresses"), "pc": sim.get("pc"), "alpha": sim.get("alpha")}
    assert (f64["alpha"] > 0).sum() > n // 4
    assert (f64["alpha"] == 0).sum() > n // 20
    for name in HISTORY:
        tol = max(BASE, 3.0 * rel(f32[name], f64[name]))
        assert rel(got[name], f64[name]) <= tol, (name, rel(got[name], f64[name]), tol)
    assert_strain_close(sim.get("eps_e"), f64["eps_e"], max(1e-4, 3.0 * rel(f32["eps_e"], f64["eps_e"])))


@pytest.mark.parametrize("material", ["mcc", "dpc"])
@pytest.mark.parametrize("dim,shape_function", [(2, "linear"), (2, "quadratic"), (3, "quadratic"), (3, "linear")])
def test_usl_steps_match_oracle(dim, shape_function, material):
    scene = block(dim, shape_function, material=material)
    steps = 4
    sim = make_gpu(scene)
    refs = {p: make_oracle(scene, p) for p in ("f32", "f64")}
    for o in refs.values():
        o.solve(steps)
    sim.solve(steps)
    assert sim.synchronize() == 0
    f32, f64 = oracle_fields(refs["f32"]), oracle_fields(refs["f64"])
    assert (f64["alpha"] > 0).sum() > 100
    for name in ("positions", "velocities", "stresses", "F", "volumes", "pc", "alpha"):
        tol = max(BASE, 3.0 * rel(f32[name], f64[name]))
        err = rel(sim.get(name), f32[name])
        assert err <= tol, (name, err, tol)
    assert_strain_close(sim.get("eps_e"), f64["eps_e"], max(1e-4, 3.0 * rel(f32["eps_e"], f64["eps_e"])))


@pytest.mark.parametrize("material", ["mcc", "dpc"])
def test_rejected_where_unsupported(material):
    """Differentiable rollouts take neither material."""
    from pyroclastmpm_b200._capi import PmpmError

    scene = block(3, "quadratic", n=500, material=material)
    sim = make_gpu(scene)
    with pytest.raises(PmpmError):
        sim.rollout_forward(4, 2)
