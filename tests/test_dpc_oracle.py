"""CPU checks of the Drucker-Prager cap restatement in the oracle (no GPU).

The reference has no unit test for this material either; the checks follow
from the model: isotropic compression of a normally consolidated point rides
the cap's tip with pc = pc0 exp(v0 / (lam - kap) alpha); shear at a pressure
well inside the cap returns to the cone in closed form (sqrt(J2) + eta p = 0,
alpha reduced by the dilatancy); yielded points of a prestressed block end on
one of the two surfaces; the FP32 restatement stays within FP32 noise of the
FP64 one.
"""
import numpy as np
import pytest

import oracle
from test_mcc_oracle import assert_strain_close

DPC = {"type": "DruckerPragerCap", "density": 1000.0, "E": 1e6, "pois": 0.2, "M": 1.05, "lam": 0.13,
       "kap": 0.033, "Vs": 1.0 / 1.8, "R": 1.0, "Pt": 0.0, "beta": 1.0, "dilatancy_angle": 5.0}


def p_sqrtJ2(S):
    S = np.asarray(S, np.float64)
    p = np.trace(S, axis1=-2, axis2=-1) / 3.0
    s = S - p[..., None, None] * np.eye(3)
    return p, np.sqrt(0.5 * (s * s).sum((-2, -1)))


def cone(p, sJ2, mat):
    return sJ2 + mat["M"] / np.sqrt(3.0) * (p - mat["Pt"])


def cap(p, sJ2, pc, mat):
    a = (pc + mat["Pt"]) / (1.0 + mat["beta"])
    b = np.where(p < mat["Pt"] - a, mat["beta"], 1.0)
    q = np.sqrt(3.0) * sJ2
    return (p - mat["Pt"] + a) ** 2 / b ** 2 + (q / mat["M"]) ** 2 - a ** 2


def test_isotropic_compression_rides_the_cap_tip():
    p0, V0, dt, rate = 5e3, 1.0, 1e-3, 0.05
    S = -p0 * np.eye(3)
    eps = np.zeros((3, 3))
    alpha, pc = 0.0, p0
    L = -rate * np.eye(3)
    C = V0 / DPC["Vs"] / (DPC["lam"] - DPC["kap"])
    for _ in range(100):
        S, eps, alpha, pc = oracle.mcc_point(3, L, S, eps, -p0 * np.eye(3), alpha, pc, V0, dt, DPC, "f64")
        p, sJ2 = p_sqrtJ2(S)
        assert sJ2 < 1e-6 * pc
        assert abs(p + pc) <= 1e-4 * pc  # the cap's compressive tip: p = Pt - (1 + beta) a = -pc
    assert alpha > 0
    np.testing.assert_allclose(pc, p0 * np.exp(C * alpha), rtol=1e-9)


def test_shear_inside_the_cap_returns_to_the_cone():
    rng = np.random.default_rng(1)
    mat = dict(DPC, R=20.0)
    C_eta = mat["M"] / np.sqrt(3.0)
    psi = np.radians(mat["dilatancy_angle"])
    eta_bar = 6 * np.sin(psi) / (np.sqrt(3) * (3 + np.sin(psi)))
    hits = 0
    for k in range(40):
        L = rng.normal(0, 5.0, (3, 3))
        L -= np.trace(L) / 3 * np.eye(3)
        S0 = -5e3 * np.eye(3)
        S, eps, alpha, pc = oracle.mcc_point(3, L, S0, np.zeros((3, 3)), S0, 0.0, 20 * 5e3, 1.0, 1e-3, mat, "f64")
        p, sJ2 = p_sqrtJ2(S)
        if alpha == 0.0:
            assert cone(p, sJ2, mat) <= 1e-9 * 5e3
            continue
        hits += 1
        assert abs(sJ2 + C_eta * p) <= 1e-9 * 5e3      # on the cone
        assert alpha < 0                                # dilatant: alpha -= eta_bar dgamma
        assert eta_bar > 0
        np.testing.assert_allclose(pc, 20 * 5e3 * np.exp(1.8 / (mat["lam"] - mat["kap"]) * alpha), rtol=1e-9)
    assert hits > 10


def block(dim, precision, R=1.0, steps=4, seed=31):
    rng = np.random.default_rng(seed + dim)
    n = 3000 if dim == 3 else 1500
    h = 0.1
    V = h ** dim / (2 ** dim)
    mat = dict(DPC, Vs=V / 1.8, R=R)
    g = [0.0] * dim
    g[-1] = -9.81
    o = oracle.OracleSim(dim=dim, origin=[0.0] * dim, end=[1.0] * dim, cell_size=h,
                         positions=rng.uniform(0.15, 0.85, (n, dim)), velocities=rng.normal(0, 0.2, (n, dim)),
                         shape_function="quadratic", dt=1e-4, particles_per_cell=2 ** dim, materials=[mat],
                         bcs=[{"type": "Gravity", "gravity": g},
                              {"type": "NodeDomain", "face0_mode": [1] * dim, "face1_mode": [1] * dim}],
                         stresses=np.broadcast_to(-5e3 * np.eye(3), (n, 3, 3)).copy(),
                         precision=precision).initialize()
    o.solve(steps)
    return o, mat


def test_yielded_points_end_on_a_surface():
    o, mat = block(3, "f64", steps=3)
    a0 = o["acc_eps_p"].copy()
    o.solve(1)
    p, sJ2 = p_sqrtJ2(o["stresses"])
    pc = o["pc"]
    y = o["acc_eps_p"] != a0
    assert y.sum() > 100
    f_cone, f_cap = cone(p, sJ2, mat), cap(p, sJ2, pc, mat)
    # the cap iteration stops at |R| <= 0.1 (Pa^2); the cone return is exact
    on = (np.abs(f_cap) <= 1e-6 * pc ** 2) | (np.abs(f_cone) <= 1e-6 * pc)
    assert on[y].all()
    assert (f_cone[~y] <= 1e-6 * pc[~y]).all() and (f_cap[~y] <= 1e-6 * pc[~y] ** 2).all()


@pytest.mark.parametrize("dim", [2, 3])
def test_fp32_restatement_agrees_with_fp64(dim):
    a, _ = block(dim, "f32")
    b, _ = block(dim, "f64")
    assert (b["acc_eps_p"] != 0).sum() > 50
    for name in ("stresses", "pc", "acc_eps_p", "positions"):
        x, y = np.asarray(a[name], np.float64), np.asarray(b[name], np.float64)
        assert np.abs(x - y).max() / np.abs(y).max() < 2e-3, name
    assert_strain_close(a["eps_e"], b["eps_e"], 2e-3)
