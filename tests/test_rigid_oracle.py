"""CPU checks of the rigid-body boundary conditions in the oracle and of the
time-step helper of the native library (no GPU).

RigidBodyLevelSet has two forms: the reference's nearest-rigid-particle stick
contact (src/boundaryconditions/rigidbodylevelset_inline.h:65-199) and the
analytic signed-distance body with Coulomb friction (no reference; its
parity is against the FP64 oracle only).  The signed distance is restated
here in numpy, independently of the C oracle, and the contact law is checked
node by node on the oracle's result.
"""
import math

import numpy as np
import pytest

import oracle
from pyroclastmpm_b200 import scenes


def shell_sdf(dim, bc, t, x):
    """Signed distance and outward normal of the RigidBodyLevelSet body (numpy)."""
    A = bc.get("axis", 1) if dim == 3 else 2
    P, Q = ((A + 1) % 3, (A + 2) % 3) if dim == 3 else (0, 1)
    c = np.array(bc["center"], float) + np.array(bc.get("velocity", [0.0] * dim), float) * t
    d = np.zeros(3)
    d[:dim] = x[:dim] - c
    if bc["shape"] == "sphere":
        r = np.linalg.norm(d)
        n = d / r
        return r - bc["dims"][0], n[:dim]
    ang = bc.get("angle", 0.0) + bc.get("angular_velocity", 0.0) * t
    cs, sn = math.cos(ang), math.sin(ang)
    lp, lq = cs * d[P] + sn * d[Q], cs * d[Q] - sn * d[P]
    R, ht, L = bc["dims"][0], 0.5 * bc["dims"][1], bc["dims"][2]
    if lq <= 0:
        rho = math.hypot(lp, lq)
        phi2 = abs(rho - R) - ht
        g = np.sign(rho - R or 1.0) * np.array([lp, lq]) / rho
    else:
        w = np.array([lp - (R if lp >= 0 else -R), lq])
        phi2 = np.linalg.norm(w) - ht
        g = w / np.linalg.norm(w)
    ga = 0.0
    phi = phi2
    if dim == 3:
        hA = abs(d[A]) - 0.5 * L
        sa = 1.0 if d[A] >= 0 else -1.0
        if phi2 > 0 and hA > 0:
            phi = math.hypot(phi2, hA)
            g, ga = g * phi2 / phi, hA * sa / phi
        elif hA > phi2:
            phi, g, ga = hA, np.zeros(2), sa
    n = np.zeros(3)
    n[P] = cs * g[0] - sn * g[1]
    n[Q] = sn * g[0] + cs * g[1]
    n[A] = ga if dim == 3 else 0.0
    return phi, n[:dim]


def body_velocity(dim, bc, t, x):
    A = bc.get("axis", 1) if dim == 3 else 2
    P, Q = ((A + 1) % 3, (A + 2) % 3) if dim == 3 else (0, 1)
    c = np.array(bc["center"], float) + np.array(bc.get("velocity", [0.0] * dim), float) * t
    v = np.zeros(3)
    v[:dim] = bc.get("velocity", [0.0] * dim)
    w = bc.get("angular_velocity", 0.0)
    v[P] -= w * (x[Q] - c[Q])
    v[Q] += w * (x[P] - c[P])
    return v[:dim]


def bed_with_body(dim, shape, friction, wall_free=True):
    rng = np.random.default_rng(11)
    h = 0.05 if dim == 2 else 0.1
    sp = h / 2
    hi = np.full(dim, 0.55)
    pts = scenes._lattice(np.zeros(dim), hi, sp) + 0.2
    pts = pts + rng.uniform(-0.2 * sp, 0.2 * sp, pts.shape)
    c = [0.4123, 0.5077, 0.4871][:dim]
    body = {"type": "RigidBodyLevelSet", "shape": shape, "axis": 1, "center": c,
            "velocity": [0.3, -0.2, 0.1][:dim], "angular_velocity": 2.0, "angle": 0.4,
            "dims": [0.2213, 0.0813, 0.3917] if shape == "half_cylinder_shell" else [0.1913, 0, 0],
            "friction": friction, "contact_distance": 0.0}
    return dict(dim=dim, origin=[0.0] * dim, end=[1.0] * dim, cell_size=h, shape_function="quadratic",
                dt=1e-4, particles_per_cell=2 ** dim, alpha=0.99,
                materials=[{"type": "LinearElastic", "density": 1000.0, "E": 1e5, "pois": 0.3}],
                bcs=[{"type": "Gravity", "gravity": [0.0] * (dim - 1) + [-9.81]}, body],
                positions=pts, velocities=rng.normal(0, 0.3, pts.shape)), body


def run_one(scene, with_body, global_step=3):
    sc = dict(scene)
    if not with_body:
        sc["bcs"] = [b for b in scene["bcs"] if b["type"] != "RigidBodyLevelSet"]
    o = oracle.OracleSim(**scenes.sim_kwargs(sc), positions=sc["positions"], velocities=sc["velocities"],
                         precision="f64", global_step=global_step).initialize()
    o.solve(1)
    return o


@pytest.mark.parametrize("dim,shape,friction", [(2, "half_cylinder_shell", 0.3), (3, "half_cylinder_shell", 0.0),
                                                (3, "sphere", 0.5), (2, "sphere", 1e3)])
def test_sdf_contact_law_node_by_node(dim, shape, friction):
    scene, body = bed_with_body(dim, shape, friction)
    free = run_one(scene, False)
    hit = run_one(scene, True)
    t = 3 * scene["dt"]
    h = scene["cell_size"]
    m = hit["node_masses"]
    ids = hit["node_ids"][:, :dim]
    n_contact = n_changed = 0
    for k in np.nonzero(m > 1e-9)[0]:
        x = ids[k] * h
        phi, n = shell_sdf(dim, body, t, x)
        v0 = free["node_moments_nt"][k] / m[k]
        v1 = hit["node_moments_nt"][k] / m[k]
        if not phi < 0:
            np.testing.assert_allclose(v1, v0, rtol=0, atol=1e-12)
            continue
        n_contact += 1
        vb = body_velocity(dim, body, t, x)
        r0, r1 = v0 - vb, v1 - vb
        vn0 = r0 @ n
        if vn0 >= 0:
            np.testing.assert_allclose(v1, v0, rtol=0, atol=1e-12)
            continue
        n_changed += 1
        assert abs(r1 @ n) < 1e-9                        # no normal relative velocity left
        vt0 = r0 - vn0 * n
        vt1 = r1 - (r1 @ n) * n
        if np.linalg.norm(vt0) <= -friction * vn0:
            assert np.linalg.norm(vt1) < 1e-9             # stick
        else:                                              # slip: |vt| reduced by mu |vn|, same direction
            assert np.linalg.norm(vt1) == pytest.approx(np.linalg.norm(vt0) + friction * vn0, rel=1e-9, abs=1e-12)
            assert vt1 @ vt0 >= 0
    assert n_contact > 0 and n_changed > 0


def test_static_rigid_block_stays_and_leaves_distant_material_alone():
    """Reference nearest-rigid-particle mode, STATIC: nodes around an isolated
    rigid block have no normal (no non-rigid particles), so they stick to
    the body's zero velocity; the block does not move under gravity, and a
    deformable block far away evolves as without the condition."""
    h = 0.05
    sp = h / 2
    soft = scenes._lattice(np.array([0.1, 0.1]), np.array([0.3, 0.3]), sp)
    rigid = scenes._lattice(np.array([0.6, 0.6]), np.array([0.8, 0.8]), sp)
    base = dict(dim=2, origin=[0.0, 0.0], end=[1.0, 1.0], cell_size=h, shape_function="linear", dt=1e-3,
                particles_per_cell=4, alpha=0.99,
                materials=[{"type": "LinearElastic", "density": 1000.0, "E": 1e4, "pois": 0.3},
                           {"type": "Material", "density": 2000.0}])
    grav = {"type": "Gravity", "gravity": [0.0, -9.81]}
    rb = {"type": "RigidBodyLevelSet", "mode": "static"}
    v = np.tile([0.2, 0.1], (len(soft), 1))
    runs = []
    for bcs in ([grav, rb], [grav]):
        o = oracle.OracleSim(**base, bcs=bcs, positions=soft, velocities=v, rigid_positions=rigid,
                             rigid_colors=np.ones(len(rigid), np.uint8), precision="f64").initialize()
        o.solve(20)
        runs.append(o)
    n = len(soft)
    np.testing.assert_array_equal(runs[0]["positions"][n:], rigid)
    assert np.abs(runs[1]["positions"][n:] - rigid).max() > 1e-4   # without it the block falls
    np.testing.assert_allclose(runs[0]["positions"][:n], runs[1]["positions"][:n], rtol=0, atol=1e-12)


def test_rigid_rotation_matrices():
    """LOOP_ROTATE: 2D rotates by -rate*dt per step (delta = previous - new);
    the reference's 3D product is zero because Rz is never assigned, so rigid
    particles get v = -(x - COM)/dt; the corrected form is a rotation."""
    h = 0.1
    rigid = np.array([[0.55, 0.45, 0.5], [0.45, 0.55, 0.52]])
    com = [0.5, 0.5, 0.5]
    for corrected in (False, True):
        o = oracle.OracleSim(dim=3, origin=[0.0] * 3, end=[1.0] * 3, cell_size=h, shape_function="linear",
                             dt=1e-3, particles_per_cell=8, materials=[{"type": "Material", "density": 1.0}],
                             bcs=[{"type": "RigidBodyLevelSet", "mode": "loop_rotate", "COM": com,
                                   "euler_angles_per_second": [0.5, 1.0, 1.5], "corrected_rotation": corrected}],
                             positions=np.zeros((0, 3)), rigid_positions=rigid, precision="f64").initialize()
        o.call("or_reset")
        o.call("or_partition")
        o.call("or_shape_functions")
        o.call("or_p2g")
        o.call("or_apply_on_nodes_moments")
        r = rigid - np.array(com)
        v = o["velocities"]
        if not corrected:
            np.testing.assert_allclose(v, -r / 1e-3, rtol=1e-12)
        else:
            d = -np.array([0.5, 1.0, 1.5]) * 1e-3
            cx, sx, cy, sy, cz, sz = np.cos(d[0]), np.sin(d[0]), np.cos(d[1]), np.sin(d[1]), np.cos(d[2]), np.sin(d[2])
            Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
            Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
            Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
            R = Rz @ Ry @ Rx
            np.testing.assert_allclose(v, (r @ R.T - r) / 1e-3, rtol=1e-9, atol=1e-12)
            np.testing.assert_allclose(np.linalg.norm(r + v * 1e-3, axis=1), np.linalg.norm(r, axis=1), rtol=1e-12)


def test_calculate_timestep_matches_reference_formula():
    """tools::calculate_timestep: dt = factor h / sqrt((K + 4G/3)/rho), the
    square root taken in double and rounded, then factor * (h / c) in FP32."""
    from pyroclastmpm_b200 import _capi

    E, nu, rho, h, fac = 1e7, 0.3, 1500.0, 1.0 / 160, 0.3
    K = np.float32(E) / (np.float32(3) * (np.float32(1) - np.float32(2) * np.float32(nu)))
    G = np.float32(E) / (np.float32(2) * (np.float32(1) + np.float32(nu)))
    c = np.float32(math.sqrt((float(K) + 4.0 * float(G) / 3.0) / rho))
    want = np.float32(fac) * (np.float32(h) / c)
    assert _capi.calculate_timestep(h, fac, float(K), float(G), rho) == float(want)
    mat = {"type": "LinearElastic", "density": rho, "E": E, "pois": nu}
    assert _capi.material_timestep(mat, h, fac) == float(want)
    dp = dict(mat, type="DruckerPrager", friction_angle=30.0)
    assert _capi.material_timestep(dp, h, fac) == float(want)
    nf = {"type": "NewtonFluid", "density": 1000.0, "viscosity": 1e-3, "bulk_modulus": 2e6, "gamma": 7.0}
    want_nf = np.float32(0.3) * (np.float32(0.02) / np.float32(math.sqrt(2e6 / 1000.0)))
    assert _capi.material_timestep(nf, 0.02, 0.3) == float(want_nf)
