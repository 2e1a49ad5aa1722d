"""Calibration of per-particle Young's modulus and friction angle with the
adjoint gradients (Adam through pyroclastmpm_b200.autograd.calibrate): a
4,096-particle copy of the calibration cube (16^3 lattice) collapsing under
gravity, started from E log-normal around 5 MPa and friction angles normal
around 25 deg, fitted to the final configuration of a rollout made with the
target E = 10 MPa and 30 deg.  The loss must fall by at least 10x and the
mean parameters move toward the target values."""
import numpy as np
import pytest

from pyroclastmpm_b200 import Simulation, scenes

pytestmark = pytest.mark.gpu


def test_calibration_loss_falls_and_parameters_move_to_target():
    torch = pytest.importorskip("torch")
    from pyroclastmpm_b200.autograd import calibrate

    scene, E0, phi0, (tE, tphi) = scenes.calibration_cube(n_side=16, cell_size=1.0 / 32, domain=0.5, dt=1e-4)
    nsteps, every = 100, 25
    kw = scenes.sim_kwargs(scene)
    tgt = Simulation(**kw)
    tgt.set_particles(scene["positions"], scene["velocities"]).initialize()
    n = len(scene["positions"])
    tgt.set("youngs_modulus", np.full(n, tE, np.float32))
    tgt.set("friction_angle", np.full(n, tphi, np.float32))
    tgt.rollout_forward(nsteps, every)  # the same stepping as the calibration's rollouts
    assert tgt.synchronize() == 0
    target = torch.tensor(tgt.get("positions"), device="cuda")
    tgt.close()
    sim = Simulation(**kw)
    sim.set_particles(scene["positions"], scene["velocities"]).initialize()
    E, phi, losses = calibrate(sim, target, E0, phi0, nsteps, every, iterations=40, lr_log_youngs=0.1,
                               lr_friction=1.0)
    assert sim.synchronize() == 0
    hist = ", ".join(f"{v:.3e}" for v in losses[::5])
    assert losses[-1] <= 0.1 * losses[0], hist
    mE0, mphi0 = float(np.mean(E0)), float(np.mean(phi0))
    mE, mphi = float(E.mean()), float(phi.mean())
    assert abs(mE - tE) < abs(mE0 - tE), (mE0, mE)
    assert abs(mphi - tphi) < abs(mphi0 - tphi), (mphi0, mphi)
