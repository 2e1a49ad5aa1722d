"""Failure paths of the step, made on the host (no GPU fault is provoked):
the key scan's bounded look-back wait running out, non-finite particle state
set from outside, a particle without mass.  The reference has no failure
reporting at all: its CUDA error check calls exit()
(include/pyroclastmpm/common/types_common.h:170-187)."""
import numpy as np
import pytest

from pyroclastmpm_b200 import Batch, Simulation, scenes

pytestmark = pytest.mark.gpu

TIMEOUT, NONFINITE = 19, 17


def column_sim(**extra):
    sc = scenes.granular_column()
    sim = Simulation(**scenes.sim_kwargs(sc), **extra)
    sim.set_particles(sc["positions"], sc["velocities"]).initialize()
    return sc, sim


def test_scan_wait_limit_reports_timeout_and_the_handle_recovers():
    """With the look-back limited to zero polls a scan CTA that finds a
    predecessor not yet published gives up: the step reports
    PMPM_ERR_TIMEOUT, its P2G is skipped (no read through the invalid
    offsets), and after the limit is restored and the state set again the
    handle steps exactly as a fresh one."""
    sc, sim = column_sim()
    assert sim.synchronize() == 0
    sim.set_wait_limit(0)
    seen = False
    for _ in range(20):  # ~540 scan CTAs per step: one of them waits
        sim.solve(1)
        st = sim.synchronize()
        assert st in (0, TIMEOUT)
        if st == TIMEOUT:
            seen = True
            break
    assert seen
    sim.set_wait_limit(1 << 22)
    sim.step = 0
    sim.set_particles(sc["positions"], sc["velocities"]).initialize()
    sim.solve(2)
    assert sim.synchronize() == 0
    _, fresh = column_sim()
    fresh.solve(2)
    assert fresh.synchronize() == 0
    for name in ("positions", "velocities", "stresses"):
        a, b = sim.get(name), fresh.get(name)
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max(), name
    sim.close()
    fresh.close()


def test_batch_scan_wait_limit_reports_timeout():
    insts = scenes.ensemble()[:48]
    b = Batch(insts).initialize()
    assert b.synchronize() == 0
    b.set_wait_limit(0)
    seen = False
    for _ in range(20):
        b.solve(1)
        st = b.synchronize()
        assert st in (0, TIMEOUT)
        if st == TIMEOUT:
            seen = True
            break
    assert seen
    b.close()


@pytest.mark.parametrize("field", ["positions", "velocities"])
def test_nonfinite_state_is_reported(field):
    """A NaN set into one particle's position or velocity spreads through
    its nodes and is reported as PMPM_ERR_NONFINITE by the step."""
    sc = scenes.two_discs()
    sim = Simulation(**scenes.sim_kwargs(sc))
    sim.set_particles(sc["positions"], sc["velocities"]).initialize()
    sim.solve(1)
    assert sim.synchronize() == 0
    vals = sim.get(field)
    vals[5, 0] = np.nan
    sim.set(field, vals)
    sim.solve(2)
    assert sim.synchronize() == NONFINITE
    sim.close()


def test_massless_particle_stays_finite():
    """A particle of zero mass adds nothing to its nodes (the reference's
    1e-9 node-mass cutoff guards the divisions): no fault, finite state."""
    sc = scenes.two_discs()
    sim = Simulation(**scenes.sim_kwargs(sc))
    sim.set_particles(sc["positions"], sc["velocities"]).initialize()
    m = sim.get("masses")
    m[:] = 0.0
    sim.set("masses", m)
    sim.solve(3)
    assert sim.synchronize() == 0
    for name in ("positions", "velocities", "stresses", "F"):
        assert np.isfinite(sim.get(name)).all(), name
