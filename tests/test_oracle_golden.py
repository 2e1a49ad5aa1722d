"""Pin the CPU oracle against the reference's own known-answer unit tests.

The vectors in tests/golden/reference_unit_vectors.json are transcribed from
PyroclastMPM's tests/unit/*.h (cited per group).  These tests exercise only the
oracle (test infrastructure) on the CPU.
"""
import json
import os

import numpy as np
import pytest

import oracle

G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_unit_vectors.json")))


@pytest.mark.parametrize("dim", [2, 3])
def test_spatialpartition_vectors(dim):
    v = G["spatialpartition"]
    pos = np.array(v["positions"][str(dim)])
    s = oracle.OracleSim(dim, [0.0] * dim, [1.0] * dim, v["cell_size"], pos)
    assert list(s.grid.num_cells) == v["num_cells"][str(dim)]
    assert s.grid.num_cells_total == v["num_cells_total"][str(dim)]
    s.call("or_partition")
    assert s["bins"].tolist() == v["bins"][str(dim)]
    assert s["hash_unsorted"].tolist() == v["hash_unsorted"]
    assert s["hash_sorted"].tolist() == v["hash_sorted"]
    assert s["sorted_index"].tolist() == v["sorted_index"]
    for c in range(s.grid.num_cells_total):
        exp = v["cell_ranges"].get(str(c), [v["empty_cell_value"]] * 2)
        assert [s["cell_start"][c], s["cell_end"][c]] == exp


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("sf", ["linear", "cubic"])
def test_shapefunction_vectors(dim, sf):
    v = G["shapefunctions"]
    pos = np.array([v["position"][str(dim)]])
    s = oracle.OracleSim(dim, [0.0] * dim, [1.0] * dim, v["cell_size"], pos, shape_function=sf)
    s.call("or_partition")
    s.call("or_shape_functions")
    exp = v[sf][str(dim)]
    psi = s["psi"]
    dpsi = s["dpsi"].reshape(-1, dim)
    np.testing.assert_allclose(psi[: len(exp["psi"])], exp["psi"], atol=v["tol"])
    np.testing.assert_allclose(dpsi[: len(exp["dpsi"])], exp["dpsi"], atol=v["tol"])
    assert abs(psi.sum() - v["sum_psi"]) < v["tol"]


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_usl_stepwise_vectors(dim, precision):
    v = G["usl_stepwise"]
    k = str(dim)
    pos = np.array(v["positions"][k])
    vel = np.ones_like(pos) * v["velocity"]
    stresses = np.zeros((2, 3, 3))
    stresses[0] = 1.0
    s = oracle.OracleSim(dim, [0.0] * dim, [1.0] * dim, 1.0, pos, vel, shape_function="linear",
                         dt=v["dt"], particles_per_cell=1, precision=precision,
                         stresses=stresses, volumes=v["volumes"], masses=v["masses"],
                         volumes_original=v["volumes"])
    s.call("or_partition")
    s.call("or_shape_functions")
    s.call("or_p2g")
    tol = v["tol"]
    np.testing.assert_allclose(s["node_masses"][:2], v["node_masses"][k], atol=tol)
    np.testing.assert_allclose(s["node_moments"][:2], v["node_moments"][k], atol=tol)
    s.call("or_g2p")
    np.testing.assert_allclose(s["volumes"][0], v["particle0_volume"][k], atol=tol)
    np.testing.assert_allclose(s["positions"][0], v["particle0_position"][k], atol=tol)
    np.testing.assert_allclose(s["velocities"][0], v["particle0_velocity"][k], atol=tol)
    np.testing.assert_allclose(np.diag(s["F"][0]), v["particle0_F_diag"][k], atol=tol)


@pytest.mark.parametrize("dim", [2, 3])
def test_particle_volume_mass_vectors(dim):
    v = G["particles"]
    pos = np.array(v["positions"][str(dim)])
    s = oracle.OracleSim(dim, [0.0] * dim, [1.0] * dim, v["cell_size"], pos,
                         particles_per_cell=v["ppc"],
                         materials=[{"type": "Material", "density": v["density"]}])
    s.call("or_partition")
    s.call("or_initial_volumes")
    s.lib.or_initial_masses(__import__("ctypes").byref(s.s), 0, s._creal(v["density"]))
    np.testing.assert_allclose(s["volumes"], v["volume"][str(dim)], atol=v["tol"])
    np.testing.assert_allclose(s["masses"], v["mass"][str(dim)], atol=v["tol"])
    s["volumes"][:] = v["preset_volume_kept"]
    s.call("or_initial_volumes")
    np.testing.assert_allclose(s["volumes"], v["preset_volume_kept"])


def test_node_id_vectors():
    v = G["nodes"]
    s = oracle.OracleSim(3, [0.0] * 3, [1.0] * 3, v["cell_size"], np.zeros((1, 3)))
    assert s.num_nodes == v["num_cells_total"]["3"]
    assert s["node_ids"][:18].tolist() == v["node_ids_3d_first18"]
