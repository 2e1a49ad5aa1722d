"""The plain-PyTorch MPM used as the gradient reference (oracle/torch_mpm.py)
against the FP64 C oracle on the same seeded cubes: the forward rollouts
agree to rounding (CPU only)."""
import numpy as np
import pytest
import torch

import oracle
from oracle.torch_mpm import TorchMPM
from pyroclastmpm_b200 import scenes


def cube(kind):
    scene, E, phi, _ = scenes.calibration_cube(n_side=8, cell_size=1.0 / 32, domain=0.5, dt=1e-4)
    v = np.zeros_like(scene["positions"])
    if kind == "flight":
        scene["positions"] = scene["positions"] + np.array([0.0, 0.0, 0.15])
        scene["materials"][0]["cohesion"] = 2e4
        v = np.array([0.7, 0.0, -2.0]) + np.random.default_rng(3).normal(0, 0.05, v.shape)
    else:
        v[:, 0] = 0.7
        v[:, 2] = -2.0
        scene["materials"][0]["cohesion"] = 200.0
    scene["velocities"] = v
    return scene, E, phi


@pytest.mark.parametrize("kind", ["flight", "impact"])
def test_torch_mpm_matches_fp64_oracle(kind):
    scene, E, phi = cube(kind)
    steps = 10
    x0 = np.asarray(scene["positions"], np.float32).astype(np.float64)
    v0 = np.asarray(scene["velocities"], np.float32).astype(np.float64)
    st = TorchMPM(scene).rollout(torch.tensor(x0), torch.tensor(v0), torch.tensor(E.astype(np.float64)),
                                 torch.tensor(phi.astype(np.float64)), steps)
    ref = oracle.OracleSim(**scenes.sim_kwargs(scene), positions=x0, velocities=v0, youngs_modulus=E,
                           friction_angle=phi, precision="f64").initialize()
    ref.solve(steps)
    for name, key in (("positions", "x"), ("velocities", "v"), ("stresses", "sig"), ("F", "F")):
        a = st[key].detach().numpy().reshape(len(x0), -1)
        b = np.asarray(ref[name], np.float64).reshape(len(x0), -1)
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), name
