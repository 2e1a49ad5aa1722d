"""CPU-side checks of the native library: it loads without a GPU and exports
every entry point declared in include/pmpm.h; host-side helpers behave."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "pmpm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pmpm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from pyroclastmpm_b200 import _capi

    L = _capi.lib()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(_capi.EXPORTS) == names


def test_status_strings_and_helpers_without_gpu():
    from pyroclastmpm_b200 import _capi

    L = _capi.lib()
    assert L.pmpm_status_string(0) == b"ok"
    assert b"grid" in L.pmpm_status_string(16)
    m = _capi.make_material({"type": "LinearElastic", "density": 1000.0, "E": 1000.0, "pois": 0.3})
    E, nu = np.float32(1000.0), np.float32(0.3)
    assert m.params[3] == pytest.approx(float(E / (np.float32(2) * (np.float32(1) + nu))), rel=0, abs=0)
    dp = _capi.make_material({"type": "DruckerPrager", "density": 1500.0, "E": 1e7, "pois": 0.3,
                              "friction_angle": 30.0, "dilatancy_angle": 0.0, "cohesion": 0.0})
    assert dp.params[2] == pytest.approx(6 * 0.5 / (3 ** 0.5 * 2.5), rel=1e-6)
    assert dp.params[3] == 0.0 and dp.params[4] == 0.0


def test_material_params_match_oracle():
    """The C helpers and the oracle derive identical FP32 constants."""
    import oracle
    from pyroclastmpm_b200 import _capi

    for m in ({"type": "LinearElastic", "density": 1000.0, "E": 1234.5, "pois": 0.27},
              {"type": "NewtonFluid", "density": 1000.0, "viscosity": 1e-3, "bulk_modulus": 2e6, "gamma": 7.0},
              {"type": "DruckerPrager", "density": 1500.0, "E": 1e7, "pois": 0.3, "friction_angle": 33.0,
               "dilatancy_angle": 5.0, "cohesion": 1200.0},
              {"type": "DP_rheo", "density": 1500.0, "E": 1e7, "pois": 0.3, "M": 1.2, "Pt": 50.0,
               "dilatancy_angle": 4.0}):
        c = _capi.make_material(m)
        t, dens, p = oracle.material_params(m, "f32")
        assert c.type == t
        got = np.array(c.params[:7], np.float32)
        want = np.array(p[:7], np.float32)
        np.testing.assert_array_equal(got, want)


def test_create_without_gpu_reports_cuda_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from pyroclastmpm_b200 import _capi

    with pytest.raises(_capi.PmpmError) as e:
        _capi.Simulation(2, [0, 0], [1, 1], 0.1)
    assert e.value.status == 2


def test_scene_particle_counts():
    from pyroclastmpm_b200 import scenes

    assert scenes.two_discs()["positions"].shape == (2528, 2)
    assert scenes.granular_column()["positions"].shape == (1331712, 3)
    s = scenes.granular_column(cell_size=1.0 / 64)
    assert s["positions"].shape == (25 * 32 * 25, 3)


def test_scan_tag_parity_alternates_across_the_wrap():
    """Consecutive key-scan launches alternate the tag's parity (it selects
    the ticket counter the launch before reset) and never publish tag 0,
    also where the tag modulus and the 32-bit launch counter wrap."""
    from pyroclastmpm_b200 import _capi

    starts = [0, 0x3ffffff0, 2 * 0x3ffffffe - 8, 0xfffffff0]
    for s0 in starts:
        prev = None
        for k in range(32):
            launch = (s0 + k) & 0xffffffff
            t = _capi.scan_tag(launch)
            assert 1 <= t <= 0x3ffffffe
            if prev is not None:
                assert (t & 1) != (prev & 1), (hex(launch), t, prev)
            prev = t


def test_resort_interval_rule_ignores_noise_and_follows_real_growth():
    """The autotuner's re-sort interval rule: step times that only scatter
    (no growth beyond the noise of the fitted slope) keep the longest
    interval, whatever the noise draws; a clear growth of the step time
    after a re-sort picks the interval that balances it against the re-sort,
    K = sqrt(2 t_sort / slope) rounded to the candidates."""
    import numpy as np
    from pyroclastmpm_b200 import _capi

    rng = np.random.default_rng(7)
    for _ in range(50):
        flat = 1.71 + rng.normal(0.0, 0.01, 48)
        assert _capi.pick_resort_interval(0.49, flat) == 128
    steps = np.arange(48)
    # slope 2e-3 ms per step: sqrt(2 * 0.49 / 2e-3) = 22 -> 16 or 32 by cost
    grow = 1.70 + 2e-3 * steps + rng.normal(0.0, 0.002, 48)
    k = _capi.pick_resort_interval(0.49, grow)
    costs = {c: 0.49 / c + 2e-3 * c / 2 for c in (8, 16, 32, 64, 128)}
    assert k == min(costs, key=costs.get)
    # steep growth: the shortest candidate
    assert _capi.pick_resort_interval(0.05, 1.7 + 0.05 * steps) == 8
    with pytest.raises(_capi.PmpmError):
        _capi.pick_resort_interval(0.49, [])
