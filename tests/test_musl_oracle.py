"""CPU checks of the MUSL restatement in the oracle (no GPU).

MUSL maps the updated particle momenta back to the grid and takes the
velocity gradient from that field.  For a field the grid represents exactly
(a uniform velocity of a block far from the walls, stress free) the remap
returns the same nodal velocities, so MUSL and USL must agree; for a general
field they differ by a small amount, and MUSL's velocity gradient is the
gradient of a mass-weighted smoothing of the particle velocities."""
import numpy as np

import oracle
from pyroclastmpm_b200 import scenes


def block(v_fn, steps=3):
    h = 0.05
    pts = scenes._lattice(np.array([0.3, 0.3]), np.array([0.6, 0.55]), h / 2)
    base = dict(dim=2, origin=[0.0, 0.0], end=[1.0, 1.0], cell_size=h, shape_function="quadratic", dt=1e-3,
                particles_per_cell=4, alpha=0.99,
                materials=[{"type": "LinearElastic", "density": 1000.0, "E": 1e4, "pois": 0.3}], bcs=[])
    out = []
    for musl in (False, True):
        o = oracle.OracleSim(**base, positions=pts, velocities=v_fn(pts), precision="f64", musl=musl).initialize()
        o.solve(steps)
        out.append(o)
    return out


def test_musl_equals_usl_for_uniform_translation():
    usl, musl = block(lambda p: np.tile([0.3, -0.2], (len(p), 1)))
    for name in ("positions", "velocities", "stresses", "F"):
        np.testing.assert_allclose(musl[name], usl[name], rtol=0, atol=1e-12)


def test_musl_differs_slightly_for_a_shear_field():
    usl, musl = block(lambda p: np.stack([np.sin(6 * p[:, 1]), 0.2 * p[:, 0]], axis=1))
    d = np.abs(musl["stresses"] - usl["stresses"]).max() / np.abs(usl["stresses"]).max()
    assert 0 < d < 0.2
    np.testing.assert_allclose(musl["positions"], usl["positions"], rtol=0, atol=1e-6)
