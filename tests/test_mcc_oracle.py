"""CPU checks of the Modified Cam Clay restatement in the oracle (no GPU).

The reference has no unit test for this material, so the restatement is
checked against what the model itself implies: isotropic compression of a
normally consolidated point follows the virgin consolidation line (p = pc,
d ln p / d eps_v = v / lam), yielded points end on the yield surface with pc
hardened by v / (lam - kap) times their plastic volumetric strain, elastic
points stay inside it, and the FP32 restatement (the reference's mixed
FP32 / FP64 arithmetic, whose Newton iteration stops on the growing bound)
lands within FP32 noise of the FP64 one.
"""
import numpy as np
import pytest

import oracle

MCC = {"type": "ModifiedCamClay", "density": 1000.0, "E": 1e6, "pois": 0.2, "M": 1.05, "lam": 0.13,
       "kap": 0.033, "Vs": 1.0 / 1.8, "R": 1.0, "Pt": 0.0, "beta": 1.0}


def pq(S):
    S = np.asarray(S, np.float64)
    p = -np.trace(S, axis1=-2, axis2=-1) / 3.0
    s = S + p[..., None, None] * np.eye(3)
    q = np.sqrt(1.5 * (s * s).sum((-2, -1)))
    return p, q


def yield_value(p, q, pc, M, Pt=0.0):
    ps = 0.5 * (pc + Pt)
    return (ps - p - Pt) ** 2 + (q / M) ** 2 - ps ** 2


def test_isotropic_compression_follows_the_virgin_consolidation_line():
    dim = 3
    p0, V, dt, rate = 5e3, 1.0, 1e-3, 0.05
    S = -p0 * np.eye(3)
    eps = np.zeros((dim, dim))
    alpha, pc = 0.0, p0  # normally consolidated: R = 1
    L = -rate * np.eye(dim)
    v = V / MCC["Vs"]
    ev = 0.0
    for _ in range(200):
        S, eps, alpha, pc = oracle.mcc_point(dim, L, S, eps, -p0 * np.eye(3), alpha, pc, V, dt, MCC, "f64")
        ev += dim * rate * dt
        p, q = pq(S)
        assert q < 1e-6 * p
        assert abs(p - pc) <= 1e-6 * pc  # stays on the cap tip p = pc
    assert alpha > 0
    # d ln p = v / lam d eps_v along the consolidation line (first order in
    # the increment: 200 steps of 1e-4 volumetric strain)
    np.testing.assert_allclose(np.log(p / p0), v / MCC["lam"] * ev, rtol=2e-2)
    # plastic part: alpha = (lam - kap) / lam of the total volumetric strain
    np.testing.assert_allclose(alpha, (MCC["lam"] - MCC["kap"]) / MCC["lam"] * ev, rtol=2e-2)


def column(dim, precision, R=1.0, steps=4):
    rng = np.random.default_rng(21 + dim)
    n = 3000 if dim == 3 else 1500
    x = rng.uniform(0.15, 0.85, (n, dim))
    v = rng.normal(0, 0.2, (n, dim))
    h = 0.1
    V = h ** dim / (2 ** dim)
    mat = dict(MCC, Vs=V / 1.8, R=R)
    p0 = 5e3
    S = np.broadcast_to(-p0 * np.eye(3), (n, 3, 3)).copy()
    g = [0.0] * dim
    g[-1] = -9.81
    o = oracle.OracleSim(dim=dim, origin=[0.0] * dim, end=[1.0] * dim, cell_size=h, positions=x, velocities=v,
                         shape_function="quadratic", dt=1e-4, particles_per_cell=2 ** dim, materials=[mat],
                         bcs=[{"type": "Gravity", "gravity": g},
                              {"type": "NodeDomain", "face0_mode": [1] * dim, "face1_mode": [1] * dim}],
                         stresses=S, precision=precision).initialize()
    np.testing.assert_allclose(o["pc"], R * p0, rtol=1e-6)
    o.solve(steps)
    return o, mat


def test_return_mapping_ends_on_the_yield_surface():
    """3D: there the trial deviator is traceless, so p and q of the final
    stress are the iteration's own (in 2D the reference zeroes the zz
    deviatoric strain, which leaves a trace in its 'deviator')."""
    o, mat = column(3, "f64", steps=3)
    alpha_before = o["acc_eps_p"].copy()
    o.solve(1)
    p, q = pq(o["stresses"])
    pc, alpha = o["pc"], o["acc_eps_p"]
    f = yield_value(p, q, pc, mat["M"])
    yielded = alpha != alpha_before  # plastic in the last step
    assert yielded.sum() > 100 and (~yielded).sum() > 0
    # the Newton iteration stops at |residual| <= 1e-2 (Pa^2 scale ~ pc^2)
    assert np.abs(f[yielded]).max() <= 1e-6 * pc[yielded].max() ** 2
    assert f[~yielded].max() <= 1e-6 * pc.max() ** 2
    # elastic strain keeps its trace history; the reference stress is the prestress
    np.testing.assert_array_equal(o["stress_ref"], np.broadcast_to(-5e3 * np.eye(3), o["stress_ref"].shape))


def test_hardening_law_of_first_yield():
    """One step from the initial state: pc = pc0 (1 + v / (lam - kap) alpha)."""
    o, mat = column(3, "f64", steps=1)
    alpha, pc = o["acc_eps_p"], o["pc"]
    y = alpha != 0
    assert y.sum() > 50
    v = o["volumes"][y] / mat["Vs"]
    expect = 5e3 * (1.0 + v / (mat["lam"] - mat["kap"]) * alpha[y])
    np.testing.assert_allclose(pc[y], expect, rtol=1e-5)


def split_strain(eps):
    """Deviatoric part and trace of D x D strains."""
    eps = np.asarray(eps, np.float64)
    d = eps.shape[-1]
    tr = np.trace(eps, axis1=-2, axis2=-1)
    return eps - tr[..., None, None] / d * np.eye(d), tr


def assert_strain_close(a, b, tol, boundary_share=0.01):
    """Elastic strains: the deviatoric parts everywhere; the traces on all
    but a small share of particles.  The reference's plastic branch
    subtracts the previous elastic volumetric strain where the elastic branch
    adds it (it mixes the sign conventions), so a particle within round-off
    of the yield surface flips its trace with the branch it takes."""
    (da, ta), (db, tb) = split_strain(a), split_strain(b)
    scale = np.abs(np.asarray(b, np.float64)).max()
    assert np.abs(da - db).max() <= tol * scale
    off = np.abs(ta - tb) > tol * scale
    assert off.mean() <= boundary_share, off.sum()


@pytest.mark.parametrize("dim", [2, 3])
def test_fp32_restatement_agrees_with_fp64(dim):
    a, _ = column(dim, "f32")
    b, _ = column(dim, "f64")
    for name in ("stresses", "pc", "acc_eps_p", "positions"):
        x, y = np.asarray(a[name], np.float64), np.asarray(b[name], np.float64)
        scale = np.abs(y).max()
        assert scale > 0, name
        assert np.abs(x - y).max() / scale < 2e-3, name
    assert_strain_close(a["eps_e"], b["eps_e"], 2e-3)
