"""CPU checks of the VonMises restatement in the oracle (no GPU): after the
return mapping every particle lies on or inside its yield surface, yielded
particles lie on it with the hardened yield stress, and the elastic strain
gives back the stress."""
import numpy as np

import oracle


def test_von_mises_return_mapping_properties():
    rng = np.random.default_rng(4)
    n = 3000
    x = rng.uniform(0.1, 0.9, (n, 3))
    v = rng.normal(0, 0.3, (n, 3))
    E, nu, sy0, H = 1e5, 0.3, 200.0, 1e3
    o = oracle.OracleSim(dim=3, origin=[0.0] * 3, end=[1.0] * 3, cell_size=0.1, positions=x, velocities=v,
                         shape_function="quadratic", dt=1e-3, particles_per_cell=8,
                         materials=[{"type": "VonMises", "density": 1000.0, "E": E, "pois": nu,
                                     "yield_stress": sy0, "H": H}], precision="f64").initialize()
    o.solve(4)
    S = o["stresses"]
    p = np.trace(S, axis1=1, axis2=2) / 3
    s = S - p[:, None, None] * np.eye(3)
    q = np.sqrt(1.5 * (s * s).sum((1, 2)))
    acc = o["acc_eps_p"]
    sy = sy0 + H * acc
    assert (acc > 0).sum() > 100
    assert (q - sy).max() < 1e-9 * sy0
    yielded = acc > 0
    np.testing.assert_allclose(q[yielded], sy[yielded], rtol=1e-9)
    K, G = E / (3 * (1 - 2 * nu)), E / (2 * (1 + nu))
    eps = o["eps_e"]
    tr = np.trace(eps, axis1=1, axis2=2)
    S2 = 2 * G * (eps - tr[:, None, None] / 3 * np.eye(3)) + K * tr[:, None, None] * np.eye(3)
    np.testing.assert_allclose(S2, S, rtol=0, atol=1e-9 * np.abs(S).max())
