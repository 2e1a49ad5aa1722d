"""The reference's Python workflows, run through MPM2D / MPM3D on the GPU."""
import json
import os

import numpy as np
import pytest

import oracle
from pyroclastmpm_b200 import scenes

pytestmark = pytest.mark.gpu
G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_unit_vectors.json")))


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def test_two_disc_example_through_module():
    """examples/two_disc_impact/run.py, shortened, vs the FP32 oracle."""
    import pyroclastmpm_b200.MPM2D as pm

    sc = scenes.two_discs()
    rng = np.random.default_rng(5)
    sc["velocities"] = sc["velocities"] * (1.0 + 0.01 * rng.uniform(-1, 1, sc["velocities"].shape))
    pm.set_globals(sc["dt"], sc["particles_per_cell"], "linear", "output")
    pm.set_global_step(0)
    nodes = pm.NodesContainer([0.0, 0.0], [1.0, 1.0], sc["cell_size"])
    particles = pm.ParticlesContainer(sc["positions"], sc["velocities"])
    mpm = pm.USL(particles, nodes, [pm.LinearElastic(1000.0, 1000.0, 0.3)], alpha=0.99)
    mpm.run(9, 100)  # 10 solves
    assert mpm.current_step == 10
    ref = oracle.OracleSim(**scenes.sim_kwargs(sc), positions=sc["positions"], velocities=sc["velocities"])
    ref.initialize()
    ref.run(9)
    assert rel(mpm.particles.positions, ref["positions"]) < 1e-5
    assert rel(mpm.particles.velocities, ref["velocities"]) < 1e-5
    assert rel(mpm.particles.stresses, ref["stresses"]) < 2e-4
    assert mpm.particles.positions.shape == (len(sc["positions"]), 2)


@pytest.mark.parametrize("dim", [2, 3])
def test_usl_stepwise_through_module(dim):
    """tests/unit/test_usl.h:32-176 written against the module API."""
    import importlib

    pm = importlib.import_module(f"pyroclastmpm_b200.MPM{dim}D")
    v = G["usl_stepwise"]
    k = str(dim)
    pm.set_globals(v["dt"], 1, "linear", "output")
    pm.set_global_step(0)
    pos = np.array(v["positions"][k])
    particles = pm.ParticlesContainer(pos, np.ones_like(pos))
    nodes = pm.NodesContainer([0.0] * dim, [1.0] * dim, 1.0)
    usl = pm.USL(particles, nodes)
    stresses = np.zeros((2, 3, 3))
    stresses[0] = 1.0
    usl.particles.masses = v["masses"]
    usl.particles.volumes = v["volumes"]
    usl.particles.volumes_original = v["volumes"]
    usl.particles.stresses = stresses
    usl.partition()
    usl.P2G()
    tol = v["tol"]
    np.testing.assert_allclose(usl.nodes.masses[:2], v["node_masses"][k], atol=tol)
    np.testing.assert_allclose(usl.nodes.moments[:2], v["node_moments"][k], atol=tol)
    usl.G2P()
    np.testing.assert_allclose(usl.particles.volumes[0], v["particle0_volume"][k], atol=tol)
    np.testing.assert_allclose(usl.particles.positions[0], v["particle0_position"][k], atol=tol)
    np.testing.assert_allclose(np.diag(usl.particles.F[0]), v["particle0_F_diag"][k], atol=tol)


def test_granular_column_through_module():
    import pyroclastmpm_b200.MPM3D as pm

    sc = scenes.granular_column(cell_size=1.0 / 64)
    pm.set_globals(sc["dt"], sc["particles_per_cell"], "quadratic", "output")
    pm.set_global_step(0)
    nodes = pm.NodesContainer(sc["origin"], sc["end"], sc["cell_size"])
    particles = pm.ParticlesContainer(sc["positions"], sc["velocities"])
    mat = pm.DruckerPrager(1500.0, 1.0e7, 0.3, 30.0, 0.0, 0.0)
    bcs = [pm.Gravity([0.0, 0.0, -9.81]), pm.NodeDomain([1, 1, 1], [1, 1, 1])]
    mpm = pm.USL(particles, nodes, [mat], bcs)
    mpm.solve_nsteps(5)
    ref = oracle.OracleSim(**scenes.sim_kwargs(sc), positions=sc["positions"], velocities=sc["velocities"])
    ref.initialize()
    ref.solve(5)
    for name in ("positions", "velocities", "stresses", "F"):
        assert rel(getattr(mpm.particles, name), ref[name]) < 1e-5, name


def test_scoop_through_module_matches_capi():
    """RigidBodyLevelSet with an analytic half-cylinder shell, set up through
    the module API, gives the C ABI Simulation's result for the same scene."""
    import pyroclastmpm_b200.MPM3D as pm
    from pyroclastmpm_b200 import Simulation

    sc = scenes.granular_bed(cell_size=1.0 / 40, scale=0.25, shape_function="cubic", dt=1e-5)
    body = sc["bcs"][1]
    pm.set_globals(sc["dt"], sc["particles_per_cell"], "cubic", "output")
    pm.set_global_step(0)
    nodes = pm.NodesContainer(sc["origin"], sc["end"], sc["cell_size"])
    particles = pm.ParticlesContainer(sc["positions"], sc["velocities"])
    mat = pm.DruckerPrager(1500.0, 1.0e7, 0.3, 30.0, 0.0, 0.0)
    rb = pm.RigidBodyLevelSet()
    rb.set_shape_half_cylinder_shell(body["center"], body["axis"], *body["dims"], body["angle"])
    rb.set_motion(body["velocity"], body["angular_velocity"])
    rb.friction = body["friction"]
    mpm = pm.USL(particles, nodes, [mat], [pm.Gravity([0.0, 0.0, -9.81]), rb, pm.NodeDomain([1, 1, 1], [1, 1, 1])])
    mpm.solve_nsteps(5)
    sim = Simulation(**scenes.sim_kwargs(sc))
    sim.set_particles(sc["positions"], sc["velocities"]).initialize()
    sim.solve(5)
    for name in ("positions", "velocities", "stresses"):
        assert rel(getattr(mpm.particles, name), sim.get(name)) < 1e-6, name


def test_musl_through_module_matches_capi():
    """The MUSL class (declared by the reference, built here) against a C ABI
    handle with the MUSL flag, deterministic reduction: bit for bit."""
    import pyroclastmpm_b200.MPM2D as pm
    from pyroclastmpm_b200 import Simulation

    sc = scenes.two_discs()
    rng = np.random.default_rng(5)
    sc["velocities"] = sc["velocities"] * (1.0 + 0.01 * rng.uniform(-1, 1, sc["velocities"].shape))
    pm.set_globals(sc["dt"], sc["particles_per_cell"], "linear", "output")
    pm.set_global_step(0)
    nodes = pm.NodesContainer([0.0, 0.0], [1.0, 1.0], sc["cell_size"])
    particles = pm.ParticlesContainer(sc["positions"], sc["velocities"])
    mpm = pm.MUSL(particles, nodes, [pm.LinearElastic(1000.0, 1000.0, 0.3)], alpha=0.99, flags=2)
    mpm.solve_nsteps(5)
    sim = Simulation(**scenes.sim_kwargs(sc), flags=2 | 4)
    sim.set_particles(sc["positions"], sc["velocities"]).initialize()
    sim.solve(5)
    for name in ("positions", "velocities", "stresses"):
        np.testing.assert_array_equal(getattr(mpm.particles, name), sim.get(name))


def test_output_writers_and_run_schedule(tmp_path):
    """Solver.run(total, frequency) writes particles<step>.vtp/.csv/.obj at
    step 0 and every `frequency` steps, nodes at steps 0 and 1 only (the
    reference's rule); the files hold the state the getters return."""
    import xml.etree.ElementTree as ET

    import pyroclastmpm_b200.MPM2D as pm

    sc = scenes.two_discs()
    pm.set_globals(sc["dt"], sc["particles_per_cell"], "linear", str(tmp_path))
    pm.set_global_step(0)
    nodes = pm.NodesContainer([0.0, 0.0], [1.0, 1.0], sc["cell_size"])
    nodes.set_output_formats(["vtk"])
    particles = pm.ParticlesContainer(sc["positions"], sc["velocities"])
    particles.set_output_formats(["vtk", "csv", "obj"])
    mpm = pm.USL(particles, nodes, [pm.LinearElastic(1000.0, 1000.0, 0.3)])
    mpm.run(10, 5)
    names = sorted(f.name for f in tmp_path.iterdir())
    for step in (0, 5, 10):
        for ext in ("vtp", "csv", "obj"):
            assert f"particles{step}.{ext}" in names
    assert "nodes0.vtp" in names and "nodes5.vtp" not in names
    root = ET.parse(tmp_path / "particles10.vtp").getroot()
    arrays = {a.get("Name"): a for a in root.iter("DataArray")}
    for key in ("Positions", "Velocity", "Stress", "Pressure", "q", "dev strain", "vol strain"):
        assert key in arrays, key
    pos10 = np.array(arrays["Positions"].text.split(), np.float64).reshape(-1, 2)
    assert float(arrays["Time"].text) == pytest.approx(10 * sc["dt"], rel=1e-6)
    # run(10) made 11 solves; the last file was written after the 11th solve
    np.testing.assert_allclose(pos10, mpm.particles.positions, rtol=0, atol=1e-6)
    header = (tmp_path / "particles0.csv").read_text().splitlines()[0]
    assert header.startswith('"isRigid","Positions:0","Positions:1","Velocity:0"')


def test_particles_pickle_restart():
    """A bound container pickled after some steps restarts a new solver with
    the same state (stress, F, masses, volumes)."""
    import pickle

    import pyroclastmpm_b200.MPM2D as pm

    sc = scenes.two_discs()
    pm.set_globals(sc["dt"], sc["particles_per_cell"], "linear", "output")
    pm.set_global_step(0)
    nodes = pm.NodesContainer([0.0, 0.0], [1.0, 1.0], sc["cell_size"])
    particles = pm.ParticlesContainer(sc["positions"], sc["velocities"])
    mpm = pm.USL(particles, nodes, [pm.LinearElastic(1000.0, 1000.0, 0.3)])
    mpm.solve_nsteps(20)
    saved = pickle.dumps(mpm.particles)
    restored = pickle.loads(saved)
    mpm2 = pm.USL(restored, pm.NodesContainer([0.0, 0.0], [1.0, 1.0], sc["cell_size"]),
                  [pm.LinearElastic(1000.0, 1000.0, 0.3)])
    for name in ("positions", "velocities", "stresses", "F", "masses", "volumes"):
        np.testing.assert_array_equal(getattr(mpm2.particles, name), getattr(mpm.particles, name), err_msg=name)


def test_modified_cam_clay_through_module_matches_capi():
    """The reference's Modified Cam Clay workflow: prestressed particles,
    material.initialize(particles, 0), then a USL solver; the same steps as
    the C ABI run of the same scene."""
    import pyroclastmpm_b200.MPM3D as pm
    from pyroclastmpm_b200 import Simulation

    rng = np.random.default_rng(9)
    n, h = 2000, 0.1
    x = rng.uniform(0.15, 0.85, (n, 3))
    v = rng.normal(0, 0.2, (n, 3))
    S = np.broadcast_to(-5e3 * np.eye(3), (n, 3, 3)).copy()
    Vs = h ** 3 / 8 / 1.8
    args = (1000.0, 1e6, 0.2, 1.05, 0.13, 0.033, Vs, 1.0, 0.0, 1.0)
    pm.set_globals(1e-4, 8, "quadratic", "output")
    pm.set_global_step(0)
    particles = pm.ParticlesContainer(x, v)
    particles.stresses = S
    mat = pm.ModifiedCamClay(*args)
    particles, _ = mat.initialize(particles, 0)
    nodes = pm.NodesContainer([0.0] * 3, [1.0] * 3, h)
    usl = pm.USL(particles, nodes, [mat], [pm.Gravity([0.0, 0.0, -9.81])], alpha=0.99)
    usl.solve_nsteps(3)
    m = dict(zip(("density", "E", "pois", "M", "lam", "kap", "Vs", "R", "Pt", "beta"), args))
    sim = Simulation(3, [0.0] * 3, [1.0] * 3, h, shape_function="quadratic", dt=1e-4, particles_per_cell=8,
                     alpha=0.99, materials=[dict(m, type="ModifiedCamClay")],
                     bcs=[{"type": "Gravity", "gravity": [0.0, 0.0, -9.81]}])
    sim.set_particles(x, v)
    sim.set("stresses", S)
    sim.initialize()
    sim.solve(3)
    for name in ("positions", "stresses"):
        assert rel(getattr(usl.particles, name), sim.get(name)) < 1e-5, name
    assert mat.calculate_timestep(h, 0.3, mat.bulk_modulus, mat.shear_modulus, 1000.0) > 0
