"""The MPM2D / MPM3D modules expose the reference's Python API (CPU checks)."""
import numpy as np
import pytest

NAMES = ["set_globals", "set_global_shapefunction", "set_global_timestep", "set_global_step",
         "set_global_output_directory", "NodesContainer", "ParticlesContainer", "Solver", "USL",
         "Material", "LinearElastic", "NewtonFluid", "DruckerPrager", "BoundaryCondition", "Gravity",
         "NodeDomain", "BodyForce", "PlanarDomain", "RigidBodyLevelSet", "calculate_timestep", "MUSL",
         "VonMises", "ModifiedCamClay", "DruckerPragerCap", "global_dimension"]


@pytest.mark.parametrize("dim", [2, 3])
def test_module_names(dim):
    import importlib

    pm = importlib.import_module(f"pyroclastmpm_b200.MPM{dim}D")
    for n in NAMES:
        assert hasattr(pm, n), n
    assert pm.global_dimension == dim


def test_nodes_container_grid_and_coords():
    import oracle
    import pyroclastmpm_b200.MPM3D as pm

    nodes = pm.NodesContainer([0.0, 0.0, 0.0], [1.0, 0.25, 0.5], 1.0 / 64)
    assert nodes.num_cells == oracle.grid_dims(3, [0, 0, 0], [1.0, 0.25, 0.5], 1.0 / 64)
    xyz = nodes.give_coords()
    assert xyz.shape == (nodes.num_cells_total, 3)
    np.testing.assert_allclose(xyz[1], [1.0 / 64, 0.0, 0.0], rtol=1e-6)
    np.testing.assert_allclose(xyz[nodes.num_cells[0]], [0.0, 1.0 / 64, 0.0], rtol=1e-6)


def test_material_constants_and_unknown_shape_function():
    import pyroclastmpm_b200.MPM2D as pm

    le = pm.LinearElastic(1000.0, 1000.0, 0.3)
    E, nu = np.float32(1000.0), np.float32(0.3)
    assert le.shear_modulus == pytest.approx(float(E / (np.float32(2) * (np.float32(1) + nu))))
    with pytest.raises(ValueError):
        pm.set_global_shapefunction("quartic")  # the reference calls exit(1) here


def test_solver_without_gpu_raises():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import pyroclastmpm_b200.MPM2D as pm

    pm.set_globals(1e-3, 4, "linear", "./output/")
    p = pm.ParticlesContainer(np.array([[0.5, 0.5]]))
    n = pm.NodesContainer([0.0, 0.0], [1.0, 1.0], 0.1)
    with pytest.raises(RuntimeError):
        pm.USL(p, n, [pm.LinearElastic(1000.0, 1000.0, 0.3)])


def test_calculate_timestep_and_rigid_body_api():
    import pyroclastmpm_b200.MPM3D as pm
    from pyroclastmpm_b200 import _capi

    le = pm.LinearElastic(1500.0, 1e7, 0.3)
    dt = le.calculate_timestep(1.0 / 160, 0.3)
    assert dt == _capi.calculate_timestep(1.0 / 160, 0.3, le.bulk_modulus, le.shear_modulus, 1500.0)
    assert pm.calculate_timestep(1.0 / 160, 0.3, le.bulk_modulus, le.shear_modulus, 1500.0) == dt
    dp = pm.DruckerPrager(1500.0, 1e7, 0.3, 30.0, 0.0, 0.0)
    assert dp.calculate_timestep(1.0 / 160, 0.3) == dt
    rb = pm.RigidBodyLevelSet()
    rb.set_mode_loop_rotate([0.0, 0.0, 1.0], [0.5, 0.5, 0.5])
    scoop = pm.RigidBodyLevelSet()
    scoop.set_shape_half_cylinder_shell([0.15, 0.25, 0.3], 1, 0.15, 0.01, 0.4)
    scoop.set_motion([0.5, 0.0, 0.0], 1.0)
    scoop.friction = 0.3
    assert scoop.friction == pytest.approx(0.3)


def test_particles_pickle_round_trip_unbound():
    """pickle_save_particles / pickle_load_particles layout (13 entries) for a
    container not yet bound to a solver (no GPU needed)."""
    import pickle

    import pyroclastmpm_b200.MPM2D as pm

    rng = np.random.default_rng(0)
    x = rng.uniform(0.2, 0.8, (20, 2))
    v = rng.normal(0, 1, (20, 2))
    rx = rng.uniform(0.2, 0.8, (5, 2))
    p = pm.ParticlesContainer(x, v, colors=np.arange(20) % 2, rigid_positions=rx, rigid_colors=[3] * 5)
    p.set_output_formats(["vtk", "csv"])
    t = p.__getstate__()
    assert len(t) == 13
    np.testing.assert_allclose(t[0], np.concatenate([x, rx]).astype(np.float32))
    assert list(t[3]) == [0] * 20 + [1] * 5
    assert list(t[2]) == list(np.arange(20) % 2) + [3] * 5
    q = pickle.loads(pickle.dumps(p))
    assert q.num_particles == 25
    assert q.output_formats == ["vtk", "csv"]
    t2 = q.__getstate__()
    for a, b in zip(t, t2):
        if isinstance(a, np.ndarray):
            np.testing.assert_array_equal(a, b)
        else:
            assert list(a) == list(b)
