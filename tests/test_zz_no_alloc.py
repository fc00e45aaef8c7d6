"""The allocation-free sort-by-cell (ariel_sort_by_cell_noalloc) against the library's own
SORT stage.

That entry point is for callers that cannot allocate device memory while running (real-time
loops, hosts whose allocator owns all device memory); it keeps its temporaries in one fixed
array inside the library.  Here it is called twice in a row, on two different particle sets,
so that the second call also shows the shared array is reset between calls.  Device buffers
come from torch, the way such a host would pass its own memory.  This file is collected last
so a failure here cannot stop the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

from ariel_b200 import _abi as A
from ariel_b200._lib import lib
from ariel_b200.flipsim import Batch

from helpers import dambreak, params


def _scene_particles(desc):
    b = Batch([desc], params())
    b.init()
    b.step(2)  # move the particles off the seeding lattice
    p = b.get_particles()
    b.close()
    return p


def _reference_binning(desc, p):
    """Cells and per-cell counts from the existing path (set_particles + SORT stage)."""
    b = Batch([desc], params())
    b.set_particles(p["pos"], p["vel"], p["mass"], p["type"])
    b.stage(A.STAGE_SORT)
    cells, counts = b.get_cells()
    b.close()
    return cells.astype(np.int64), counts.astype(np.int64)


def _noalloc(pos, dim):
    import torch
    n = len(pos)
    d_pos = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    d_cell = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_start = torch.zeros(dim ** 3 + 1, dtype=torch.int32, device="cuda")
    d_order = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib().ariel_sort_by_cell_noalloc(C.c_void_p(d_pos.data_ptr()), n, dim, C.c_void_p(d_cell.data_ptr()),
                                          C.c_void_p(d_start.data_ptr()), C.c_void_p(d_order.data_ptr()), None)
    assert rc == A.ARIEL_OK, A.status_name(rc)
    torch.cuda.synchronize()
    as_u = lambda t: t.cpu().numpy().view(np.uint32).astype(np.int64)
    return as_u(d_cell), as_u(d_start), as_u(d_order)


@pytest.mark.gpu
def test_noalloc_sort_matches_sort_stage_twice():
    cases = [dambreak(32, seed=4), dambreak(24, seed=9, hi=(0.5, 0.3, 0.8))]
    for desc in cases:
        p = _scene_particles(desc)
        want_cells, want_counts = _reference_binning(desc, p)
        cells, start, order = _noalloc(p["pos"], desc.dim)
        np.testing.assert_array_equal(cells, want_cells)  # bit-exact cell of every particle
        np.testing.assert_array_equal(np.diff(start), want_counts)
        assert start[0] == 0 and start[-1] == len(cells)
        np.testing.assert_array_equal(order, np.argsort(cells, kind="stable"))


@pytest.mark.gpu
def test_noalloc_rejects_oversize():
    L = lib()
    big_grid = L.ariel_sort_by_cell_noalloc(None, 0, 65, None, C.c_void_p(1), None, None)
    assert big_grid == A.ARIEL_ERR_INVALID_ARG
    too_many = L.ariel_sort_by_cell_noalloc(C.c_void_p(1), (1 << 20) + 1, 16, C.c_void_p(1), C.c_void_p(1),
                                            C.c_void_p(1), None)
    assert too_many == A.ARIEL_ERR_INVALID_ARG
