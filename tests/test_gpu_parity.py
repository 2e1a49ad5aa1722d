"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Tolerances: binning is bit-exact.  One FP32 step must agree with the FP32
oracle within 1e-5 relative (max |a - b| / max |b| per field), or, where the
reference's own FP32 arithmetic is worse conditioned than that, within three
times the FP32 oracle's distance from the FP64 oracle (the Tait pressure of a
Newtonian fluid loses digits to the cancellation (rho/rho0)^gamma - 1).
Multi-step drift against the FP64 oracle: 1e-4, with the same conditioning
allowance.
"""
import json
import os

import numpy as np
import pytest

import oracle
from pyroclastmpm_b200 import Simulation, scenes

pytestmark = pytest.mark.gpu

G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_unit_vectors.json")))
STEP_TOL = 1e-5


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def particle_kwargs(scene):
    """Particle arrays of a scene (rigid particles follow the others)."""
    return dict(positions=scene["positions"], velocities=scene["velocities"], colors=scene.get("colors"),
                rigid_positions=scene.get("rigid_positions"), rigid_velocities=scene.get("rigid_velocities"),
                rigid_colors=scene.get("rigid_colors"))


def cond_tol(scene, steps, names, base):
    """Per-field tolerance: base, or 3x the FP32-vs-FP64 oracle distance."""
    kw = scenes.sim_kwargs(scene)
    o = [oracle.OracleSim(**kw, **particle_kwargs(scene), precision=p).initialize() for p in ("f32", "f64")]
    for x in o:
        x.solve(steps)
    return {n: max(base, 3.0 * rel(o[0][n], o[1][n])) for n in names}


def perturbed(scene, amount=0.01, seed=5):
    rng = np.random.default_rng(seed)
    v = scene["velocities"]
    scene["velocities"] = v + amount * np.abs(v).max() * rng.uniform(-1, 1, size=v.shape)
    return scene


def make_pair(scene, precision="f32", **extra):
    kw = scenes.sim_kwargs(scene)
    sim = Simulation(**kw, **extra)
    sim.set_particles(**particle_kwargs(scene))
    ref = oracle.OracleSim(**kw, **particle_kwargs(scene), precision=precision)
    return sim, ref


def random_scene(dim, n, shape_function, seed, margin=0.0, lo=0.0, hi=1.0, cell=0.1, mats=None, bcs=None):
    rng = np.random.default_rng(seed)
    x = rng.uniform(lo + margin, hi - margin, size=(n, dim))
    v = rng.normal(0.0, 0.1, size=(n, dim))
    return dict(dim=dim, origin=[0.0] * dim, end=[1.0] * dim, cell_size=cell, shape_function=shape_function,
                dt=1e-3, particles_per_cell=4 if dim == 2 else 8, alpha=0.99,
                materials=mats or [{"type": "LinearElastic", "density": 1000.0, "E": 1e4, "pois": 0.3}],
                bcs=bcs or [], positions=x, velocities=v)


# ----------------------------------------------------------------------------
# known-answer vectors of the reference's unit tests, through the GPU path
# ----------------------------------------------------------------------------

@pytest.mark.parametrize("dim", [2, 3])
def test_reference_vectors_spatialpartition(dim):
    v = G["spatialpartition"]
    sim = Simulation(dim, [0.0] * dim, [1.0] * dim, v["cell_size"])
    sim.set_particles(np.array(v["positions"][str(dim)]))
    sim.partition()
    assert sim.num_cells == v["num_cells"][str(dim)]
    assert sim.get("bins").tolist() == v["bins"][str(dim)]
    assert sim.get("hash_unsorted").tolist() == v["hash_unsorted"]
    assert sim.get("hash_sorted").tolist() == v["hash_sorted"]
    assert sim.get("sorted_index").tolist() == v["sorted_index"]
    cs, ce = sim.get("cell_start"), sim.get("cell_end")
    for c in range(sim.num_nodes):
        assert [cs[c], ce[c]] == v["cell_ranges"].get(str(c), [0, 0])


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("sf", ["linear", "cubic"])
def test_reference_vectors_shapefunctions(dim, sf):
    v = G["shapefunctions"]
    sim = Simulation(dim, [0.0] * dim, [1.0] * dim, v["cell_size"], shape_function=sf)
    sim.set_particles(np.array([v["position"][str(dim)]]))
    sim.partition()
    psi, dpsi = sim.shape_functions()
    exp = v[sf][str(dim)]
    np.testing.assert_allclose(psi[0, : len(exp["psi"])], exp["psi"], atol=v["tol"])
    np.testing.assert_allclose(dpsi[0, : len(exp["dpsi"])], exp["dpsi"], atol=v["tol"])
    assert abs(psi.sum() - 1.0) < v["tol"]


@pytest.mark.parametrize("dim", [2, 3])
def test_reference_vectors_usl_stepwise(dim):
    v = G["usl_stepwise"]
    k = str(dim)
    pos = np.array(v["positions"][k])
    sim = Simulation(dim, [0.0] * dim, [1.0] * dim, 1.0, shape_function="linear", dt=v["dt"],
                     particles_per_cell=1)
    sim.set_particles(pos, np.ones_like(pos))
    sim.initialize()
    stresses = np.zeros((2, 3, 3))
    stresses[0] = 1.0
    sim.set("masses", v["masses"])
    sim.set("volumes", v["volumes"])
    sim.set("volumes_original", v["volumes"])
    sim.set("stresses", stresses)
    sim.partition()
    sim.p2g()
    tol = v["tol"]
    np.testing.assert_allclose(sim.get("node_masses")[:2], v["node_masses"][k], atol=tol)
    np.testing.assert_allclose(sim.get("node_moments")[:2], v["node_moments"][k], atol=tol)
    sim.g2p()
    np.testing.assert_allclose(sim.get("volumes")[0], v["particle0_volume"][k], atol=tol)
    np.testing.assert_allclose(sim.get("positions")[0], v["particle0_position"][k], atol=tol)
    np.testing.assert_allclose(sim.get("velocities")[0], v["particle0_velocity"][k], atol=tol)
    np.testing.assert_allclose(np.diag(sim.get("F")[0]), v["particle0_F_diag"][k], atol=tol)


@pytest.mark.parametrize("dim", [2, 3])
def test_reference_vectors_particles(dim):
    v = G["particles"]
    sim = Simulation(dim, [0.0] * dim, [1.0] * dim, v["cell_size"], particles_per_cell=v["ppc"],
                     materials=[{"type": "Material", "density": v["density"]}])
    sim.set_particles(np.array(v["positions"][str(dim)]))
    sim.initialize()
    np.testing.assert_allclose(sim.get("volumes"), v["volume"][str(dim)], atol=v["tol"])
    np.testing.assert_allclose(sim.get("masses"), v["mass"][str(dim)], atol=v["tol"])


# ----------------------------------------------------------------------------
# binning: bit-exact against the oracle (reference semantics)
# ----------------------------------------------------------------------------

@pytest.mark.parametrize("dim,sf", [(2, "linear"), (3, "linear"), (3, "quadratic")])
@pytest.mark.parametrize("seed", [0, 1])
def test_binning_bit_exact(dim, sf, seed):
    """The reference partition views are bit-exact; with the 3D quadratic
    fast path the step bins by dual cell and the views come from the stored
    reference hashes."""
    rng = np.random.default_rng(seed)
    n = 20000 if dim == 3 else 5000
    x = rng.uniform(0.0, 1.0, size=(n, dim))
    # edge cases: exact node lines, the far boundary, slightly outside (aliasing
    # rows and hashes past the grid), duplicates, dense clusters
    x[:50] = np.round(x[:50] * 10) / 10
    x[50:60] = 1.0
    x[60:70, 0] = 1.05
    x[70:80, 0] = -0.05
    x[80:90] = 5.0
    x[90:200] = x[90]
    x[200:1000] = rng.uniform(0.3, 0.31, size=(800, dim))
    sim = Simulation(dim, [0.0] * dim, [1.0] * dim, 0.05, shape_function=sf)
    sim.set_particles(x)
    sim.partition()
    ref = oracle.OracleSim(dim, [0.0] * dim, [1.0] * dim, 0.05, x, shape_function=sf)
    ref.call("or_partition")
    for name in ("bins", "hash_unsorted", "hash_sorted", "sorted_index", "cell_start", "cell_end"):
        np.testing.assert_array_equal(sim.get(name), ref[name], err_msg=name)
    assert sim.synchronize() == 16  # particles past the grid are reported


def test_binning_big_cells_and_resort():
    """More than 32 particles in a cell (bitonic path), and physical re-sorts
    keep the reference permutation."""
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(0.5, 0.52, size=(1500, 2)), rng.uniform(0, 1, size=(3000, 2))])
    sc = random_scene(2, 10, "linear", 0)
    sc["positions"], sc["velocities"] = x, np.zeros_like(x)
    sim, ref = make_pair(sc, resort_interval=1)
    sim.initialize()
    ref.initialize()
    for name in ("hash_sorted", "sorted_index", "cell_start", "cell_end"):
        np.testing.assert_array_equal(sim.get(name), ref[name], err_msg=name)
    sim.solve(2)
    ref.solve(2)
    np.testing.assert_array_equal(sim.get("sorted_index"), ref["sorted_index"])
    assert rel(sim.get("positions"), ref["positions"]) < STEP_TOL


# ----------------------------------------------------------------------------
# shape functions against the oracle
# ----------------------------------------------------------------------------

@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("sf", ["linear", "quadratic", "cubic"])
def test_shape_functions_match_oracle(dim, sf):
    rng = np.random.default_rng(7)
    x = rng.uniform(0.0, 1.0, size=(2000, dim))
    x[:10] = 0.0
    x[10:20] = 1.0
    sim = Simulation(dim, [0.0] * dim, [1.0] * dim, 0.1, shape_function=sf)
    sim.set_particles(x)
    sim.partition()
    psi, dpsi = sim.shape_functions()
    ref = oracle.OracleSim(dim, [0.0] * dim, [1.0] * dim, 0.1, x, shape_function=sf)
    ref.call("or_partition")
    ref.call("or_shape_functions")
    np.testing.assert_allclose(psi.ravel(), ref["psi"], atol=2e-6)
    np.testing.assert_allclose(dpsi.ravel(), ref["dpsi"], atol=2e-5 * 10)
    # cubic: in the first cell the out-of-grid slot aliases onto the previous
    # row's boundary node (reference flat-index check), and the reference never
    # assigns the type-4 node next to the upper boundary, so the weights sum to
    # one only for cells 1 .. N-4
    lo, hi = (0.1, 0.8) if sf == "cubic" else (0.0, 0.9)
    inside = np.all((x > lo) & (x < hi), axis=1)
    np.testing.assert_allclose(psi[inside].sum(axis=1), 1.0, atol=1e-5)   # partition of unity
    np.testing.assert_allclose(dpsi[inside].sum(axis=1), 0.0, atol=1e-3)  # sum of gradients


# ----------------------------------------------------------------------------
# one step and several steps against the oracle
# ----------------------------------------------------------------------------

STEP_CASES = {
    "discs_2d_linear_le": lambda: perturbed(scenes.two_discs()),
    "water_2d_quadratic_nf": lambda: scenes.water_column(),
    "random_2d_cubic_le": lambda: random_scene(2, 3000, "cubic", 1, margin=0.05),
    "random_2d_quadratic_nf": lambda: random_scene(
        2, 3000, "quadratic", 2, margin=0.0,
        mats=[{"type": "NewtonFluid", "density": 1000.0, "viscosity": 1e-3, "bulk_modulus": 2e6, "gamma": 7.0}],
        bcs=[{"type": "Gravity", "gravity": [0.0, -9.81]},
             {"type": "NodeDomain", "face0_mode": [1, 1], "face1_mode": [1, 1]}]),
    "random_2d_linear_dp_mixed": lambda: dict(
        random_scene(2, 3000, "linear", 3, margin=0.02,
                     mats=[{"type": "DruckerPrager", "density": 1500.0, "E": 1e6, "pois": 0.3, "friction_angle": 30.0,
                            "cohesion": 10.0},
                           {"type": "LinearElastic", "density": 1000.0, "E": 1e5, "pois": 0.2}],
                     bcs=[{"type": "NodeDomain", "face0_mode": [0, 1], "face1_mode": [1, 0]}]),
        colors=np.random.default_rng(3).integers(0, 2, 3000)),
    "column_3d_quadratic_dp": lambda: scenes.granular_column(cell_size=1.0 / 64),
    # 64 x 32 x 32 nodes, particles up to the upper x and y faces: a tile
    # whose last node column is the grid's last has 27 dual pairs per axis
    # (the clamped offsets fold onto the last node), more work items than
    # the dual sweep's 640 threads, so this grid runs the cell scatter
    "column_3d_quadratic_dp_face_tiles": lambda: scenes.granular_column(
        domain=(63 / 64, 31 / 64, 31 / 64), cell_size=1.0 / 64, column=(63 / 64, 31 / 64, 0.2)),
    "random_3d_cubic_le_gravity": lambda: random_scene(
        3, 4000, "cubic", 4, margin=0.05, cell=0.1,
        bcs=[{"type": "Gravity", "gravity": [0.0, 0.0, -9.81]},
             {"type": "NodeDomain", "face0_mode": [1, 1, 1], "face1_mode": [1, 1, 1]}]),
    "random_3d_quadratic_le_walls": lambda: random_scene(
        3, 4000, "quadratic", 6, margin=0.0, cell=0.1,
        bcs=[{"type": "Gravity", "gravity": [0.0, -9.81, 0.0]},
             {"type": "NodeDomain", "face0_mode": [1, 0, 1], "face1_mode": [1, 1, 0]}]),
    "random_3d_linear_nf_planar": lambda: random_scene(
        3, 4000, "linear", 5, margin=0.0, cell=0.1,
        mats=[{"type": "NewtonFluid", "density": 1000.0, "viscosity": 1e-2, "bulk_modulus": 1e4, "gamma": 7.0}],
        bcs=[{"type": "PlanarDomain", "face0_friction": [10.0, 0.0, 5.0], "face1_friction": [0.0, 20.0, 0.0]}]),
}

def rigid_block_scene(dim, mode="static", rate=None, corrected=False, seed=7):
    """A linear-elastic block driven into a block of rigid particles
    (RigidBodyLevelSet in the reference's nearest-rigid-particle mode)."""
    rng = np.random.default_rng(seed)
    h = 0.05
    sp = h / 2
    lo, hi = np.full(dim, 0.3), np.full(dim, 0.5)
    soft = scenes._lattice(lo, hi, sp)
    soft = soft + rng.uniform(-0.2 * sp, 0.2 * sp, soft.shape)
    rlo = lo.copy()
    rlo[0] = 0.5
    rhi = hi.copy()
    rhi[0] = 0.6
    rigid = scenes._lattice(rlo, rhi, sp)
    v = np.zeros_like(soft)
    v[:, 0] = 0.5
    v += rng.normal(0, 0.02, v.shape)
    com = list(0.5 * (rlo + rhi))
    bc = {"type": "RigidBodyLevelSet", "mode": mode, "COM": com, "corrected_rotation": corrected,
          "euler_angles_per_second": rate or [0.0] * dim}
    return dict(dim=dim, origin=[0.0] * dim, end=[1.0] * dim, cell_size=h, shape_function="linear", dt=1e-3,
                particles_per_cell=2 ** dim, alpha=0.99,
                materials=[{"type": "LinearElastic", "density": 1000.0, "E": 1e4, "pois": 0.3},
                           {"type": "Material", "density": 2000.0}],
                bcs=[{"type": "Gravity", "gravity": [0.0, -9.81] + [0.0] * (dim - 2)}, bc,
                     {"type": "NodeDomain", "face0_mode": [1] * dim, "face1_mode": [1] * dim}],
                positions=soft, velocities=v, rigid_positions=rigid, rigid_colors=np.ones(len(rigid), np.uint8))


def scoop_scene(dim, shape_function, shape="half_cylinder_shell", friction=0.3, seed=8, n_side=None):
    """A Drucker-Prager bed with an analytic rigid body cutting into it,
    translating and turning (RigidBodyLevelSet with a signed distance)."""
    rng = np.random.default_rng(seed)
    h = 0.05 if dim == 2 else 0.1
    sp = h / 2
    lo = np.zeros(dim)
    hi = np.full(dim, 0.6)
    hi[0] = 0.9
    pts = scenes._lattice(lo, hi, sp) + 0.05
    pts = pts + rng.uniform(-0.2 * sp, 0.2 * sp, pts.shape)
    up = dim - 1
    # geometry off the node lattice, so no node sits on the body's surface
    c = [0.3137, 0.4871, 0.5][:dim]
    c[up] = 0.6071
    dims = [0.2513, 0.0617, 0.5129] if shape == "half_cylinder_shell" else [0.2213, 0.0, 0.0]
    body = {"type": "RigidBodyLevelSet", "shape": shape, "axis": 1, "center": c,
            "velocity": [0.5, 0.0, 0.0][:dim], "angular_velocity": 1.0, "angle": -0.3, "dims": dims,
            "friction": friction, "contact_distance": 0.0}
    g = [0.0] * dim
    g[up] = -9.81
    return dict(dim=dim, origin=[0.0] * dim, end=[1.0] * dim, cell_size=h, shape_function=shape_function,
                dt=1e-4, particles_per_cell=2 ** dim, alpha=0.99,
                materials=[{"type": "DruckerPrager", "density": 1500.0, "E": 1e6, "pois": 0.3,
                            "friction_angle": 30.0, "cohesion": 100.0}],
                bcs=[{"type": "Gravity", "gravity": g}, body,
                     {"type": "NodeDomain", "face0_mode": [1] * dim, "face1_mode": [1] * dim}],
                positions=pts, velocities=rng.normal(0, 0.05, pts.shape))


STEP_CASES.update({
    "random_3d_quadratic_vm": lambda: random_scene(
        3, 4000, "quadratic", 13, margin=0.0, cell=0.1,
        mats=[{"type": "VonMises", "density": 1000.0, "E": 1e5, "pois": 0.3, "yield_stress": 200.0, "H": 1e3},
              {"type": "VonMises", "density": 2000.0, "E": 3e5, "pois": 0.25, "yield_stress": 50.0, "H": 0.0}],
        bcs=[{"type": "Gravity", "gravity": [0.0, 0.0, -9.81]},
             {"type": "NodeDomain", "face0_mode": [1, 1, 1], "face1_mode": [1, 1, 1]}]) | {
        "colors": np.random.default_rng(13).integers(0, 2, 4000)},
    "rigid_nn_2d_static": lambda: rigid_block_scene(2),
    "rigid_nn_2d_rotate": lambda: rigid_block_scene(2, "loop_rotate", [2.0, 0.0]),
    "rigid_nn_3d_static": lambda: rigid_block_scene(3),
    "rigid_nn_3d_rotate_reference": lambda: rigid_block_scene(3, "loop_rotate", [1e-4, 2e-4, 3e-4]),
    "rigid_nn_3d_rotate_corrected": lambda: rigid_block_scene(3, "loop_rotate", [1.0, 2.0, 3.0], True),
    "sdf_2d_quadratic_shell": lambda: scoop_scene(2, "quadratic"),
    "sdf_2d_linear_sphere_frictionless": lambda: scoop_scene(2, "linear", "sphere", 0.0),
    "sdf_3d_quadratic_shell": lambda: scoop_scene(3, "quadratic"),
    "sdf_3d_cubic_sphere": lambda: scoop_scene(3, "cubic", "sphere", 0.5),
    "sdf_3d_cubic_shell": lambda: scoop_scene(3, "cubic"),
    "sdf_3d_linear_shell_stick": lambda: scoop_scene(3, "linear", friction=100.0),
})

FIELDS = ("positions", "velocities", "stresses", "F", "volumes")


@pytest.mark.parametrize("case", sorted(STEP_CASES))
def test_one_step_matches_oracle(case):
    scene = STEP_CASES[case]()
    sim, ref = make_pair(scene, flags=1)
    sim.initialize()
    ref.initialize()
    sim.solve(1)
    ref.solve(1)
    names = FIELDS + ("velocity_gradient", "node_masses", "node_moments", "node_moments_nt")
    tol = cond_tol(scene, 1, names, STEP_TOL)
    for name in names:
        err = rel(sim.get(name), ref[name])
        assert err <= tol[name], f"{case} {name}: {err:.3e} > {tol[name]:.1e}"


@pytest.mark.parametrize("case", ["discs_2d_linear_le", "column_3d_quadratic_dp", "water_2d_quadratic_nf",
                                  "sdf_3d_quadratic_shell", "sdf_2d_quadratic_shell", "rigid_nn_2d_rotate",
                                  "random_3d_quadratic_vm", "random_3d_cubic_le_gravity", "sdf_3d_cubic_shell"])
def test_multi_step_drift_vs_fp64(case):
    """20 steps: FP32 GPU against the FP64 oracle (drift bound 1e-4)."""
    scene = STEP_CASES[case]()
    sim, ref = make_pair(scene, precision="f64")
    sim.initialize()
    ref.initialize()
    sim.solve(20)
    ref.solve(20)
    assert sim.synchronize() == 0
    names = ("positions", "velocities", "stresses")
    tol = cond_tol(scene, 20, names, 1e-4)
    for name in names:
        err = rel(sim.get(name), ref[name])
        assert err <= tol[name], f"{case} {name}: {err:.3e} > {tol[name]:.1e}"


@pytest.mark.parametrize("case", ["discs_2d_linear_le", "column_3d_quadratic_dp", "random_3d_cubic_le_gravity",
                                  "rigid_nn_3d_static", "sdf_3d_quadratic_shell"])
def test_deterministic_path_matches_oracle(case):
    """The deterministic (gather) P2G against the FP32 oracle, one step."""
    scene = STEP_CASES[case]()
    sim, ref = make_pair(scene, flags=2)
    sim.initialize()
    ref.initialize()
    sim.solve(1)
    ref.solve(1)
    names = FIELDS + ("node_masses", "node_moments", "node_moments_nt")
    tol = cond_tol(scene, 1, names, STEP_TOL)
    for name in names:
        err = rel(sim.get(name), ref[name])
        assert err <= tol[name], f"{case} {name}: {err:.3e} > {tol[name]:.1e}"


def test_tile_and_gather_paths_agree():
    scene = scenes.granular_column(cell_size=1.0 / 64)
    out = []
    for flags in (0, 2):
        sim, _ = make_pair(scene, flags=flags)
        sim.initialize()
        sim.solve(5)
        out.append([sim.get(n) for n in FIELDS])
    for a, b in zip(*out):
        assert rel(a, b) < 1e-5


def test_deterministic_bitwise():
    scene = scenes.granular_column(cell_size=1.0 / 64)
    outs = []
    for _ in range(2):
        sim, _ref = make_pair(scene, resort_interval=4, flags=2)
        sim.initialize()
        sim.solve(10)
        outs.append([sim.get(n) for n in FIELDS])
        sim.close()
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def test_drucker_prager_points_match_reference_dp_rheo():
    """Per-point cone / apex return (reference DP_rheo parameters) on random
    strain histories, against the oracle's restatement of update_dp_rheo."""
    from pyroclastmpm_b200 import material_point_update

    rng = np.random.default_rng(11)
    for dim in (2, 3):
        n = 4000
        mat = {"type": "DP_rheo", "density": 1500.0, "E": 1e7, "pois": 0.3, "M": 1.2, "Pt": 20.0,
               "dilatancy_angle": 6.0}
        L = rng.normal(0, 0.5, size=(n, dim, dim))
        sref = rng.normal(0, 1e4, size=(n, 3, 3))
        sref = 0.5 * (sref + sref.transpose(0, 2, 1))
        sref[:, np.arange(3), np.arange(3)] -= 3e4
        eps = rng.normal(0, 1e-4, size=(n, dim, dim))
        eps = 0.5 * (eps + eps.transpose(0, 2, 1))
        S0 = np.zeros((n, 3, 3))
        S, E = material_point_update(mat, dim, L, S0, eps_e=eps, stress_ref=sref, dt=1e-3)
        for i in range(0, n, 97):
            s_ref, e_ref = oracle.dp_point(dim, L[i], S0[i], eps[i], sref[i], 1e-3, mat)
            assert rel(S[i], s_ref) < 2e-5
            assert rel(E[i], e_ref) < 2e-5


def test_two_disc_kinetic_energy():
    """tests/examples/two_disc_impact/test_two_disks.py: KE(0) ~ 2.51 (+-10 %)
    and |KE(end) - KE(0)| / KE(0) < 0.2 over 3600 steps."""
    v = G["two_disc_impact"]
    scene = scenes.two_discs(cell_size=1.0 / 20, centers=((0.2, 0.2), (0.8, 0.8)), ppc_1d=2)
    scene["materials"] = scene["materials"] * 2
    n = len(scene["positions"])
    scene["colors"] = (np.arange(n) >= n // 2).astype(np.uint8)
    sim, _ = make_pair(scene)
    sim.initialize()

    def ke():
        m = sim.get("masses")
        vel = sim.get("velocities")
        return 0.5 * float((m[:, None] * vel ** 2).sum())

    ke0 = ke()
    assert abs(ke0 - v["ke0"]) / v["ke0"] < v["ke0_rel_tol"]
    sim.solve(v["steps"])
    assert sim.synchronize() == 0
    assert abs(ke() - ke0) / ke0 < v["ke_drift_max"]


def test_out_of_domain_is_reported_not_fatal():
    sc = random_scene(2, 500, "linear", 9, margin=0.1)
    sc["positions"][0] = [3.0, 3.0]
    sim, _ = make_pair(sc)
    sim.initialize()
    sim.solve(2)
    assert sim.synchronize() == 16
    sim.solve(1)
    assert sim.synchronize() == 16
    assert np.isfinite(sim.get("positions")[1:]).all()


# ----------------------------------------------------------------------------
# MUSL (second momentum mapping)
# ----------------------------------------------------------------------------

MUSL_CASES = ["discs_2d_linear_le", "column_3d_quadratic_dp", "random_2d_quadratic_nf", "random_3d_cubic_le_gravity",
              "sdf_3d_quadratic_shell"]


def musl_pair(scene, precision, flags):
    kw = scenes.sim_kwargs(scene)
    sim = Simulation(**kw, flags=flags | 4)
    sim.set_particles(**particle_kwargs(scene))
    ref = oracle.OracleSim(**kw, **particle_kwargs(scene), precision=precision, musl=True)
    return sim, ref


@pytest.mark.parametrize("case", MUSL_CASES)
@pytest.mark.parametrize("flags", [1, 3])
def test_musl_one_step_matches_oracle(case, flags):
    scene = STEP_CASES[case]()
    sim, ref = musl_pair(scene, "f32", flags)
    sim.initialize()
    ref.initialize()
    sim.solve(1)
    ref.solve(1)
    names = FIELDS + ("velocity_gradient",)
    refs = [oracle.OracleSim(**scenes.sim_kwargs(scene), **particle_kwargs(scene), precision=p,
                             musl=True).initialize() for p in ("f32", "f64")]
    for r in refs:
        r.solve(1)
    for name in names:
        tol = max(STEP_TOL, 3.0 * rel(refs[0][name], refs[1][name]))
        err = rel(sim.get(name), ref[name])
        assert err <= tol, f"{case} {name}: {err:.3e} > {tol:.1e}"


@pytest.mark.parametrize("case", ["discs_2d_linear_le", "column_3d_quadratic_dp"])
def test_musl_drift_vs_fp64(case):
    scene = STEP_CASES[case]()
    sim, ref = musl_pair(scene, "f64", 0)
    sim.initialize()
    ref.initialize()
    sim.solve(20)
    ref.solve(20)
    assert sim.synchronize() == 0
    for name in ("positions", "velocities", "stresses"):
        err = rel(sim.get(name), ref[name])
        assert err <= 1e-4, f"{case} {name}: {err:.3e}"


def test_musl_stages_equal_solve():
    """partition, P2G, the three MUSL stages and the step counter by hand give
    what one solve gives (deterministic reduction, so bit for bit)."""
    scene = STEP_CASES["column_3d_quadratic_dp"]()
    a, _ = musl_pair(scene, "f32", 3)
    b, _ = musl_pair(scene, "f32", 3)
    a.initialize()
    b.initialize()
    a.solve(1)
    from pyroclastmpm_b200._capi import check, lib
    b.partition()
    b.p2g(apply_bcs=True)
    for stage in (1, 2, 3):
        check(lib().pmpm_musl_stage(b.handle, stage), "musl stage")
    for name in ("positions", "velocities", "stresses", "F"):
        np.testing.assert_array_equal(a.get(name), b.get(name))


def test_von_mises_history_matches_oracle():
    """The VonMises history (elastic strain, accumulated plastic strain)
    against the oracle after 5 steps; some particles must have yielded."""
    scene = STEP_CASES["random_3d_quadratic_vm"]()
    sim, ref = make_pair(scene)
    sim.initialize()
    ref.initialize()
    sim.solve(5)
    ref.solve(5)
    acc = sim.get("acc_eps_p")
    assert (ref["acc_eps_p"] > 0).sum() > 100
    tol = cond_tol(scene, 5, ("eps_e", "acc_eps_p"), 1e-4)
    assert rel(sim.get("eps_e"), ref["eps_e"]) <= tol["eps_e"]
    assert rel(acc, ref["acc_eps_p"]) <= tol["acc_eps_p"]


def test_autotune_keeps_state_and_both_variants_match_oracle():
    """The autotuner times both 3D quadratic P2G kernels from the same state
    and puts the state back; the simulation then matches the oracle."""
    from pyroclastmpm_b200._capi import check, lib
    scene = STEP_CASES["column_3d_quadratic_dp"]()
    sim, ref = make_pair(scene)
    sim.initialize()
    before = {n: sim.get(n) for n in ("positions", "velocities", "stresses", "F")}
    v = sim.autotune(3)
    assert v in (0, 1)
    t = sim.tuning()
    assert t["p2g_kernel"] == v and t["staging"] in (0, 1) and t["resort_interval"] in (8, 16, 32, 64, 128)
    for n, a in before.items():
        np.testing.assert_array_equal(sim.get(n), a)
    assert sim.step == 0
    ref.initialize()
    ref.solve(2)
    sim.solve(2)
    tol = cond_tol(scene, 2, FIELDS, STEP_TOL)
    for name in FIELDS:
        assert rel(sim.get(name), ref[name]) <= tol[name], name


def test_binning_ahead_keeps_reference_views_and_survives_edits():
    """3D quadratic steps bin the next partition inside their G2P: after a
    step the reference partition views still describe that step's own
    partition, and positions edited between steps are binned afresh."""
    scene = STEP_CASES["column_3d_quadratic_dp"]()
    sim, ref = make_pair(scene)
    sim.initialize()
    ref.initialize()
    sim.solve(2)
    ref.solve(2)
    for name in ("hash_unsorted", "hash_sorted", "sorted_index", "cell_start", "cell_end"):
        np.testing.assert_array_equal(sim.get(name), ref[name], err_msg=name)
    rng = np.random.default_rng(8)
    x = ref["positions"].astype(np.float64)
    x = (x + rng.uniform(-0.3, 0.3, x.shape) * scene["cell_size"]).astype(np.float32)
    lo = np.array(scene["origin"]) + 1.5 * scene["cell_size"]
    hi = np.array(scene["end"]) - 1.5 * scene["cell_size"]
    x = np.clip(x, lo, hi).astype(np.float32)
    sim.set("positions", x)
    ref["positions"][:] = x
    sim.solve(1)
    ref.solve(1)
    assert sim.synchronize() == 0
    np.testing.assert_array_equal(sim.get("hash_unsorted"), ref["hash_unsorted"])
    for name in ("positions", "velocities"):
        assert rel(sim.get(name), ref[name]) <= 1e-4, name


@pytest.mark.parametrize("variant", [0, 1])
def test_each_3d_quadratic_p2g_kernel_matches_oracle(variant):
    """Both 3D quadratic P2G kernels (cell-row scatter 0, dual sweep 1),
    selected directly, against the oracle over two steps."""
    scene = STEP_CASES["column_3d_quadratic_dp"]()
    sim, ref = make_pair(scene)
    sim.set_p2g_kernel(variant)
    sim.initialize()
    ref.initialize()
    sim.solve(2)
    ref.solve(2)
    tol = cond_tol(scene, 2, FIELDS, STEP_TOL)
    for name in FIELDS:
        assert rel(sim.get(name), ref[name]) <= tol[name], name


@pytest.mark.parametrize("staging", [0, 1])
@pytest.mark.parametrize("case", ["column_3d_quadratic_dp", "random_3d_cubic_le_gravity", "sdf_3d_cubic_shell",
                                  "random_3d_linear_nf_planar", "sdf_3d_linear_shell_stick"])
def test_each_p2g_staging_matches_oracle(case, staging):
    """The 3D sweeps' two stagings (bulk copies of sorted records 1, gather
    through the sorted order 0), selected directly, against the oracle over
    two steps, across re-sorts (interval 1) and with a PlanarDomain."""
    scene = STEP_CASES[case]()
    sim, ref = make_pair(scene, resort_interval=1)
    sim.set_p2g_staging(staging)
    sim.initialize()
    ref.initialize()
    sim.solve(2)
    ref.solve(2)
    assert sim.synchronize() == 0
    tol = cond_tol(scene, 2, FIELDS, STEP_TOL)
    for name in FIELDS:
        assert rel(sim.get(name), ref[name]) <= tol[name], name


def test_autotune_picks_staging_and_resort_interval_on_cubic():
    """On a cubic sweep the autotuner chooses the staging and the re-sort
    interval and leaves the state as it was."""
    scene = STEP_CASES["random_3d_cubic_le_gravity"]()
    sim, ref = make_pair(scene)
    sim.initialize()
    sim.solve(1)
    ref.initialize()
    ref.solve(1)
    before = {n: sim.get(n) for n in ("positions", "velocities", "stresses", "F")}
    sim.autotune(2)
    t = sim.tuning()
    assert t["staging"] in (0, 1) and t["resort_interval"] in (8, 16, 32, 64, 128)
    for n, a in before.items():
        np.testing.assert_array_equal(sim.get(n), a)
    assert sim.step == 1
    sim.solve(2)
    ref.solve(2)
    tol = cond_tol(scene, 3, FIELDS, STEP_TOL)
    for name in FIELDS:
        assert rel(sim.get(name), ref[name]) <= tol[name], name


def test_dual_sweep_refused_where_face_tiles_exceed_its_threads():
    """On a grid with a node count divisible by 8 along x (64 x 32 x 32
    nodes) the tiles at the upper face have 27 dual pairs along that axis and
    more work items than the dual sweep's CTA: the handle runs the cell
    scatter, refuses the sweep, and the autotuner keeps to the scatter; on
    the 65 x 17 x 33 column the sweep stays the default."""
    from pyroclastmpm_b200._capi import PmpmError

    face = STEP_CASES["column_3d_quadratic_dp_face_tiles"]()
    sim, _ref = make_pair(face)
    sim.initialize()
    assert sim.tuning()["p2g_kernel"] == 0
    with pytest.raises(PmpmError):
        sim.set_p2g_kernel(1)
    sim.set_p2g_kernel(0)
    sim.autotune(1)
    assert sim.tuning()["p2g_kernel"] == 0
    sim.close()
    col = STEP_CASES["column_3d_quadratic_dp"]()
    sim, _ref = make_pair(col)
    sim.initialize()
    assert sim.tuning()["p2g_kernel"] == 1
    sim.close()
