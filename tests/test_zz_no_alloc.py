"""The allocation-free partition entry point (pmpm_partition_noalloc).

Callers that cannot allocate device memory where they need a partition (an
allocator callback, a plug-in on a fixed device-memory budget) use this entry
point: they pass the inputs and outputs, and the
library's temporaries live in a fixed array inside the library.  This test
calls it through the C ABI twice in a row (the second call must not see
leftovers of the first) and checks it against the regular partition entry
point; integer results, so the comparison is exact.  It runs last so a
failure here leaves the rest of the suite already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _regular(dim, x, cell):
    from pyroclastmpm_b200 import Simulation

    sim = Simulation(dim, [0.0] * dim, [1.0] * dim, cell)
    sim.set_particles(x)
    sim.partition()
    out = {k: sim.get(k) for k in ("hash_unsorted", "sorted_index", "cell_start", "cell_end")}
    out["num_cells"] = sim.num_cells
    sim.close()
    return out


def _noalloc(dim, x, cell, num_cells, expect=0, check_memory=False):
    import torch

    from pyroclastmpm_b200 import _capi

    L = _capi.lib()
    n = x.shape[0]
    ncells = int(np.prod(num_cells[:dim]))
    xs = torch.as_tensor(np.ascontiguousarray(x, np.float32), device="cuda")
    hash_u = torch.full((n,), 0xDEAD, dtype=torch.int32, device="cuda")
    sidx = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    cs = torch.full((ncells,), -7, dtype=torch.int32, device="cuda")
    ce = torch.full((ncells,), -7, dtype=torch.int32, device="cuda")
    origin = (ctypes.c_float * 3)(0.0, 0.0, 0.0)
    nc = (ctypes.c_int * 3)(*num_cells)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = L.pmpm_partition_noalloc(dim, origin, ctypes.c_float(cell), nc, ctypes.c_void_p(xs.data_ptr()), n,
                                  ctypes.c_void_p(hash_u.data_ptr()), ctypes.c_void_p(sidx.data_ptr()),
                                  ctypes.c_void_p(cs.data_ptr()), ctypes.c_void_p(ce.data_ptr()), None)
    assert st == expect, _capi.STATUS.get(st, st)
    if check_memory:
        # a call after the first one on this device takes no device memory
        assert torch.cuda.mem_get_info()[0] == free0
    return {"hash_unsorted": hash_u.cpu().numpy().view(np.uint32), "sorted_index": sidx.cpu().numpy(),
            "cell_start": cs.cpu().numpy(), "cell_end": ce.cpu().numpy()}


@pytest.mark.parametrize("dim", [2, 3])
def test_noalloc_partition_matches_regular_twice(dim):
    rng = np.random.default_rng(21 + dim)
    cell = 0.05
    results = []
    for call in range(2):
        n = 20000 if dim == 3 else 6000
        x = rng.uniform(0.0, 1.0, size=(n, dim))
        x[: 1500 + 300 * call] = rng.uniform(0.41, 0.44, size=(1500 + 300 * call, dim))  # cells with > 32 particles
        x[2000:2010] = np.round(x[2000:2010] * 20) / 20  # exact cell faces
        ref = _regular(dim, x, cell)
        got = _noalloc(dim, x, cell, list(ref["num_cells"]), check_memory=call == 1)
        for k in ("hash_unsorted", "sorted_index", "cell_start", "cell_end"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"call {call}: {k}")
        results.append(got)
    assert not np.array_equal(results[0]["sorted_index"], results[1]["sorted_index"])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from pyroclastmpm_b200 import _capi

    L = _capi.lib()
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    origin = (ctypes.c_float * 3)(0.0, 0.0, 0.0)
    nc = (ctypes.c_int * 3)(1024, 1024, 1)  # 1,048,576 cells > the fixed limit
    p = ctypes.c_void_p(buf.data_ptr())
    st = L.pmpm_partition_noalloc(2, origin, ctypes.c_float(0.01), nc, p, 1, p, p, p, p, None)
    assert st == 1


@pytest.mark.parametrize("dim", [2, 3])
def test_noalloc_reports_particles_outside_the_grid(dim):
    """A particle past the +x face whose flat index stays inside the grid and
    a NaN coordinate: binned as the reference's flat hash puts them (the same
    outputs as the regular partition), and reported as out of the domain."""
    rng = np.random.default_rng(31 + dim)
    cell = 0.05
    x = rng.uniform(0.0, 1.0, size=(3000, dim))
    x[7] = [1.07] + [0.5] * (dim - 1)       # column 21 of 21: wraps into the next row
    x[11] = [np.nan] + [0.3] * (dim - 1)
    ref = _regular(dim, x, cell)
    got = _noalloc(dim, x, cell, list(ref["num_cells"]), expect=16)
    for k in ("hash_unsorted", "sorted_index", "cell_start", "cell_end"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    x[11] = [0.3] * dim
    got = _noalloc(dim, x, cell, list(ref["num_cells"]), expect=16)   # the +x particle alone
    x[7] = [0.5] * dim
    _noalloc(dim, x, cell, list(ref["num_cells"]), expect=0)


def test_noalloc_reports_cells_beyond_the_sort():
    """More than 2048 particles in one cell: PMPM_ERR_CELL_OVERFLOW; every
    output but that cell's order inside sorted_index is still the regular
    partition's, and that cell holds the right particles."""
    rng = np.random.default_rng(41)
    cell = 0.05
    x = rng.uniform(0.0, 1.0, size=(8000, 3))
    x[:2100] = rng.uniform(0.4005, 0.4495, size=(2100, 3))
    ref = _regular(3, x, cell)
    got = _noalloc(3, x, cell, list(ref["num_cells"]), expect=18)
    for k in ("hash_unsorted", "cell_start", "cell_end"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    c = int(ref["hash_unsorted"][0])
    lo, hi = int(ref["cell_start"][c]), int(ref["cell_end"][c])
    assert hi - lo >= 2100  # the uniform particles may add one or two
    outside = np.ones(len(x), bool)
    outside[lo:hi] = False
    np.testing.assert_array_equal(got["sorted_index"][outside], ref["sorted_index"][outside])
    np.testing.assert_array_equal(np.sort(got["sorted_index"][lo:hi]), ref["sorted_index"][lo:hi])
