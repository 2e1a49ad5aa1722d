"""The CUDA adjoint of a rollout (pmpm_rollout_forward / _backward) against
torch.autograd through a small plain-PyTorch MPM of the same step
(oracle/torch_mpm.py, FP64): 512 particles, quadratic B-splines,
Drucker-Prager with per-particle Young's modulus and friction angle,
gravity and slip walls.  The loss is w . x_final with fixed random weights;
its gradients with respect to E, the friction angle (per degree), the
initial positions and velocities must agree within 1e-4 (relative, in the
2-norm over particles).  The return mapping differentiated is
update_dp_rheo (src/materials/dp_rheo_inline.h:50-96, 123-246).
"""
import numpy as np
import pytest
import torch

from oracle.torch_mpm import TorchMPM
from pyroclastmpm_b200 import Simulation, scenes

pytestmark = pytest.mark.gpu


def small_cube():
    return scenes.calibration_cube(n_side=8, cell_size=1.0 / 32, domain=0.5, dt=1e-4)


def flight():
    """Cohesive cube in free flight with a random velocity field: elastic,
    away from the walls (the map is smooth)."""
    scene, E, phi, _ = small_cube()
    scene["positions"] = scene["positions"] + np.array([0.0, 0.0, 0.15])
    scene["materials"][0]["cohesion"] = 2e4
    rng = np.random.default_rng(3)
    scene["velocities"] = np.array([0.7, 0.0, -2.0]) + rng.normal(0, 0.05, scene["positions"].shape)
    return scene, E, phi


def impact():
    """The cube thrown at the floor and sideways: compressed against the
    wall within a few steps, it yields (cone and apex returns)."""
    scene, E, phi, _ = small_cube()
    v = np.zeros_like(scene["positions"])
    v[:, 0] = 0.7
    v[:, 2] = -2.0
    scene["velocities"] = v
    scene["materials"][0]["cohesion"] = 200.0
    return scene, E, phi


def gpu_gradients(scene, E, phi, steps, every, w):
    sim = Simulation(**scenes.sim_kwargs(scene))
    sim.set_particles(scene["positions"], scene["velocities"]).initialize()
    sim.set("youngs_modulus", E)
    sim.set("friction_angle", phi)
    sim.rollout_forward(steps, every)
    x_final = sim.get("positions").astype(np.float64)
    gE, gphi, gx0, gv0 = sim.rollout_backward(w.astype(np.float32))
    assert sim.synchronize() == 0
    sim.close()
    return x_final, {"E": gE, "phi": gphi, "x0": gx0, "v0": gv0}


def torch_gradients(scene, E, phi, steps, w):
    mpm = TorchMPM(scene)
    f64 = lambda a: torch.tensor(np.asarray(a, np.float32).astype(np.float64), requires_grad=True)
    x0, v0, Et, pt = f64(scene["positions"]), f64(scene["velocities"]), f64(E), f64(phi)
    st = mpm.rollout(x0, v0, Et, pt, steps)
    loss = (torch.tensor(w) * st["x"]).sum()
    loss.backward()
    return st["x"].detach().numpy(), {"E": Et.grad.numpy(), "phi": pt.grad.numpy(), "x0": x0.grad.numpy(),
                                      "v0": v0.grad.numpy()}


def rel2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("case,names,steps,every", [
    ("flight", ("E", "x0", "v0"), 10, 4),
    ("impact", ("E", "phi", "x0"), 10, 4),
])
def test_adjoint_matches_torch_autograd(case, names, steps, every):
    scene, E, phi = {"flight": flight, "impact": impact}[case]()
    w = np.random.default_rng(7).normal(0, 1, scene["positions"].shape)
    x_gpu, g_gpu = gpu_gradients(scene, E, phi, steps, every, w)
    x_t, g_t = torch_gradients(scene, E, phi, steps, w)
    # the forward passes agree (FP32 against FP64)
    assert np.abs(x_gpu - x_t).max() <= 1e-5 * np.abs(x_t).max()
    if case == "impact":
        assert np.linalg.norm(g_t["phi"]) > 0  # the friction angle matters: particles yielded
    for name in names:
        err = rel2(g_gpu[name], g_t[name])
        assert err <= 1e-4, f"{case} d/d{name}: {err:.3e}"
