"""Differentiable rollouts: per-particle Drucker-Prager parameters in the
forward step, and the checkpointed adjoint against finite differences of
the FP64 oracle (directional derivatives, central differences).

The loss is the mean squared distance of the final positions from a target
rollout made with other parameters, as in the calibration configuration.
"""
import numpy as np
import pytest

import oracle
from pyroclastmpm_b200 import Simulation, scenes

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def small_cube(steps_dt=1e-4):
    scene, E, phi, target = scenes.calibration_cube(n_side=16, cell_size=1.0 / 32, domain=0.5, dt=steps_dt)
    return scene, E, phi, target


def oracle_final(scene, E, phi, steps, precision="f64", x0=None, v0=None):
    o = oracle.OracleSim(**scenes.sim_kwargs(scene), positions=scene["positions"] if x0 is None else x0,
                         velocities=scene["velocities"] if v0 is None else v0, youngs_modulus=E,
                         friction_angle=phi, precision=precision).initialize()
    o.solve(steps)
    return np.array(o["positions"], np.float64)


def make_sim(scene, E, phi, flags=0):
    sim = Simulation(**scenes.sim_kwargs(scene), flags=flags)
    sim.set_particles(scene["positions"], scene["velocities"]).initialize()
    sim.set("youngs_modulus", E)
    sim.set("friction_angle", phi)
    return sim


def test_per_particle_parameters_forward_matches_oracle():
    scene, E, phi, _ = small_cube()
    sim = make_sim(scene, E, phi)
    np.testing.assert_array_equal(sim.get("youngs_modulus"), E)
    sim.solve(10)
    assert sim.synchronize() == 0
    ref = [oracle.OracleSim(**scenes.sim_kwargs(scene), positions=scene["positions"],
                            velocities=scene["velocities"], youngs_modulus=E, friction_angle=phi,
                            precision=p).initialize() for p in ("f32", "f64")]
    for r in ref:
        r.solve(10)
    for name in ("positions", "velocities", "stresses"):
        tol = max(1e-5, 3 * rel(ref[0][name], ref[1][name]))
        assert rel(sim.get(name), ref[0][name]) <= tol, name
    # the material's own values reproduce the material path
    sim2 = Simulation(**scenes.sim_kwargs(scene))
    sim2.set_particles(scene["positions"], scene["velocities"]).initialize()
    filled = sim2.get("youngs_modulus")
    np.testing.assert_allclose(filled, 1e7, rtol=1e-6)
    np.testing.assert_allclose(sim2.get("friction_angle"), 30.0, rtol=1e-5)


def impact_cube():
    """The small cube thrown at the floor and sideways (2 m/s): within a few
    steps it is compressed against the wall and yields, so the parameters
    shape the final positions well above FP32 resolution."""
    scene, E, phi, target = small_cube()
    v = np.zeros_like(scene["positions"])
    v[:, 0] = 0.7
    v[:, 2] = -2.0
    scene["velocities"] = v
    return scene, E, phi, target


def flight_cube():
    """A cohesive cube in free flight with a random velocity field: it stays
    elastic and away from the walls, so the rollout is a smooth map and
    central differences converge in every direction."""
    scene, E, phi, target = small_cube()
    scene["positions"] = scene["positions"] + np.array([0.0, 0.0, 0.15])
    scene["materials"][0]["cohesion"] = 2e4
    rng = np.random.default_rng(3)
    scene["velocities"] = np.array([0.7, 0.0, -2.0]) + rng.normal(0, 0.05, scene["positions"].shape)
    return scene, E, phi, target


def directional_checks(scene, E, phi, steps, every, names, tol, eps=1e-4):
    """Loss w . x_final with fixed random weights w (its gradient is O(1) in
    every direction, so FP32 roundoff of the positions does not mask it):
    the adjoint's directional derivatives against FP64 central differences."""
    n = len(scene["positions"])
    w = np.random.default_rng(7).normal(0, 1, (n, 3))
    sim = make_sim(scene, E, phi)
    sim.rollout_forward(steps, every)
    gE, gphi, gx0, gv0 = sim.rollout_backward(w)
    # the backward leaves the simulation at the initial state
    np.testing.assert_array_equal(sim.get("positions"), scene["positions"].astype(np.float32))
    rng = np.random.default_rng(0)
    dE = E * rng.normal(0, 1, n)
    dphi = rng.normal(0, 1, n)
    dx = rng.normal(0, 1e-3 * scene["cell_size"], (n, 3))
    dv = rng.normal(0, 1e-2, (n, 3))
    cases = {
        "E": (np.dot(gE.astype(np.float64), dE), lambda e: oracle_final(scene, E + e * dE, phi, steps)),
        "phi": (np.dot(gphi.astype(np.float64), dphi), lambda e: oracle_final(scene, E, phi + e * dphi, steps)),
        "x0": ((gx0.astype(np.float64) * dx).sum(),
               lambda e: oracle_final(scene, E, phi, steps, x0=scene["positions"] + e * dx)),
        "v0": ((gv0.astype(np.float64) * dv).sum(),
               lambda e: oracle_final(scene, E, phi, steps, v0=scene["velocities"] + e * dv)),
    }
    for name in names:
        adj, run = cases[name]
        fd = (float((w * run(eps)).sum()) - float((w * run(-eps)).sum())) / (2 * eps)
        assert fd != 0.0
        assert abs(adj - fd) <= tol * abs(fd), f"{name}: adjoint {adj:.6e} vs FD {fd:.6e}"


def test_adjoint_smooth_rollout_matches_fp64_finite_differences():
    scene, E, phi, _ = flight_cube()
    directional_checks(scene, E, phi, 16, 5, ("E", "x0", "v0"), 1e-4)


@pytest.mark.parametrize("steps,every", [(4, 1), (16, 5)])
def test_adjoint_plastic_impact_matches_fp64_finite_differences(steps, every):
    """Yielding against the floor.  The slip-wall clamps and the yield
    surface put kinks in the map; along the velocity direction central
    differences do not converge there, so v0 is checked in the smooth case."""
    scene, E, phi, _ = impact_cube()
    directional_checks(scene, E, phi, steps, every, ("E", "phi", "x0"), 2e-2)


def test_autograd_function_matches_direct_backward():
    torch = pytest.importorskip("torch")
    from pyroclastmpm_b200.autograd import rollout

    scene, E, phi, _ = small_cube()
    n = len(scene["positions"])
    sim = make_sim(scene, E, phi)
    target = torch.tensor(scene["positions"], dtype=torch.float32, device="cuda") + 0.001
    Et = torch.tensor(E, device="cuda", requires_grad=True)
    pt = torch.tensor(phi, device="cuda", requires_grad=True)
    for _ in range(2):  # a second evaluation starts from the same state
        x = rollout(sim, Et, pt, 6, 3)
        loss = ((x - target) ** 2).sum() / n
        Et.grad = None
        pt.grad = None
        loss.backward()
    sim2 = make_sim(scene, E, phi)
    sim2.rollout_forward(6, 3)
    x2 = sim2.get("positions")
    np.testing.assert_allclose(x.detach().cpu().numpy(), x2, rtol=0, atol=1e-6)
    gE, gphi, _, _ = sim2.rollout_backward(2.0 * (x2 - target.cpu().numpy()) / n)
    np.testing.assert_allclose(Et.grad.cpu().numpy(), gE, rtol=1e-3, atol=1e-3 * np.abs(gE).max())
    np.testing.assert_allclose(pt.grad.cpu().numpy(), gphi, rtol=1e-3, atol=1e-3 * np.abs(gphi).max())


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("cohesion", [0.0, 2e3])
def test_return_mapping_vjp_reverse_equals_dual_numbers(dim, cohesion):
    """The reverse-mode VJP of the Drucker-Prager update (used by the rollout
    adjoint) against forward-mode dual numbers, over states in the elastic,
    cone and apex branches."""
    from pyroclastmpm_b200._capi import material_point_vjp

    rng = np.random.default_rng(11 + dim)
    n = 6000
    mat = {"type": "DruckerPrager", "density": 1500.0, "E": 1e7, "pois": 0.3, "friction_angle": 30.0,
           "dilatancy_angle": 5.0, "cohesion": cohesion}
    L = rng.normal(0, 40.0, (n, dim, dim))
    L[: n // 3] *= 0.02                                   # mostly elastic
    L[n // 3: n // 2] += 60.0 * np.eye(dim)               # tension: apex
    eps = rng.normal(0, 2e-4, (n, dim, dim))
    eps = 0.5 * (eps + eps.transpose(0, 2, 1))
    sref = rng.normal(0, 2e3, (n, 3, 3))
    sref = 0.5 * (sref + sref.transpose(0, 2, 1)) - 1e4 * np.eye(3)
    if dim == 2:
        sref[:, 2, :2] = sref[:, :2, 2] = 0
    E = rng.uniform(2e6, 2e7, n)
    phi = rng.uniform(20.0, 40.0, n)
    gS = rng.normal(0, 1, (n, 3, 3))
    gEo = rng.normal(0, 1e4, (n, dim, dim))
    out = [material_point_vjp(mat, dim, 1e-4, L, eps, sref, gS, gEo, E, phi, method=m) for m in (0, 1)]
    for k, name in enumerate(("L", "eps_e", "E", "phi")):
        a, b = out[0][k].astype(np.float64), out[1][k].astype(np.float64)
        scale = np.abs(b).max()
        assert scale > 0
        err = np.abs(a - b).max() / scale
        assert err < 2e-4, f"{name}: {err:.2e}"


def test_kept_segments_and_checkpoints_give_the_same_gradients():
    """Backward from segments kept whole, from checkpoints alone (recomputed
    segments) and from a mix: the same gradients up to FP32 summation order.
    Deterministic P2G, so a recomputed segment repeats the forward bit for
    bit (otherwise summation order can move a particle across the yield
    surface and change its local Jacobian)."""
    scene, E, phi, _ = impact_cube()
    n = len(scene["positions"])
    w = np.random.default_rng(2).normal(0, 1, (n, 3))
    grads = []
    for budget in (-1, 0, None):
        sim = make_sim(scene, E, phi, flags=2)
        if budget is None:  # room for one segment of 5 steps
            nodes = sim.num_nodes
            per_step = 4 * (sim.n + 63) // 64 * 64 * 28 + 4 * nodes * (1 + 6 + 8) + 4 * 1024
            budget = 5 * per_step * 3 // 2
        sim.rollout_set_memory(budget)
        sim.rollout_forward(12, 5)
        grads.append(sim.rollout_backward(w))
    for g in grads[1:]:
        for a, b in zip(grads[0], g):
            np.testing.assert_allclose(a, b, rtol=1e-3, atol=1e-4 * np.abs(b).max())


def test_kept_and_recomputed_segments_agree_with_dual_cell_binning():
    """Default (non-deterministic) mode, where each step's G2P already bins
    the next partition: the node snapshots kept by the forward pass must
    carry the tiles of their own step's P2G.  Kept segments and segments
    recomputed from checkpoints give the same gradients up to FP32
    summation order (the elastic flight keeps the map smooth)."""
    scene, E, phi, _ = flight_cube()
    n = len(scene["positions"])
    w = np.random.default_rng(5).normal(0, 1, (n, 3))
    grads = []
    for budget in (-1, 0):
        sim = make_sim(scene, E, phi)
        sim.rollout_set_memory(budget)
        sim.rollout_forward(12, 5)
        grads.append(sim.rollout_backward(w))
    for a, b in zip(*grads):
        assert np.isfinite(a).all()
        np.testing.assert_allclose(a, b, rtol=1e-3, atol=1e-4 * np.abs(b).max())
