"""The allocation-free sort-by-cell (ariel_sort_by_cell_noalloc) against the oracle's
ParticleGrid::Sort and the library's own SORT stage.

That entry point is for callers that cannot allocate device memory while running (real-time
loops, hosts whose allocator owns all device memory); it keeps its temporaries in one fixed
array inside the library.  Every case calls it at least twice in a row, on different particle
sets, so the later calls also show that the shared array is reset between calls.  Device
buffers come from torch, the way such a host would pass its own memory.  Checked: the cell of
every particle and the per-cell counts against the oracle (bit-exact), and the grouped order
against a stable argsort (ascending id inside a cell, the order ParticleGrid::Sort appends).
Cases cover the limits (2^20 particles on a 64^3 grid), no particles at all, and crowded cells
that take each of the three in-cell ordering paths.  This file is collected last so a failure
here cannot stop the other GPU tests.
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


def _oracle_binning(dim, pos):
    """Cell of every particle and per-cell counts from the oracle's ParticleGrid::Sort."""
    from oracle.pyoracle import RefSim
    desc = A.scene_dambreak(dim)
    r = RefSim(desc, params())
    n = len(pos)
    r.set_particles(pos, np.zeros((n, 3), np.float32), np.ones(n, np.float32), np.full(n, A.FLUID, np.int32))
    r.stage(A.STAGE_SORT)
    cells, counts = r.get_cells()
    r.close()
    return cells.astype(np.int64), counts.astype(np.int64)


def _sort_stage_binning(desc, p):
    b = Batch([desc], params())
    b.set_particles(p["pos"], p["vel"], p["mass"], p["type"])
    b.stage(A.STAGE_SORT)
    cells, counts = b.get_cells()
    b.close()
    return cells.astype(np.int64), counts.astype(np.int64)


def _noalloc(pos, dim):
    import torch
    n = len(pos)
    d_pos = torch.from_numpy(np.ascontiguousarray(pos, np.float32).reshape(-1)).cuda()
    d_cell = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    d_start = torch.full((dim ** 3 + 1,), -1, dtype=torch.int32, device="cuda")
    d_order = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib().ariel_sort_by_cell_noalloc(C.c_void_p(d_pos.data_ptr()) if n else None, n, dim,
                                          C.c_void_p(d_cell.data_ptr()), C.c_void_p(d_start.data_ptr()),
                                          C.c_void_p(d_order.data_ptr()), None)
    assert rc == A.ARIEL_OK, A.status_name(rc)
    torch.cuda.synchronize()
    as_u = lambda t: t.cpu().numpy().view(np.uint32).astype(np.int64)
    return as_u(d_cell)[:n], as_u(d_start), as_u(d_order)[:n]


def _check(pos, dim):
    cells, start, order = _noalloc(pos, dim)
    want_cells, want_counts = _oracle_binning(dim, pos)
    np.testing.assert_array_equal(cells, want_cells)  # bit-exact cell of every particle
    np.testing.assert_array_equal(np.diff(start), want_counts)
    assert start[0] == 0 and start[-1] == len(pos)
    np.testing.assert_array_equal(order, np.argsort(cells, kind="stable"))
    return want_counts


@pytest.mark.gpu
def test_noalloc_sort_matches_oracle_and_sort_stage_twice():
    cases = [dambreak(32, seed=4), dambreak(24, seed=9, hi=(0.5, 0.3, 0.8))]
    for desc in cases:
        p = _scene_particles(desc)
        _check(p["pos"], desc.dim)
        want_cells, want_counts = _sort_stage_binning(desc, p)
        cells, start, _ = _noalloc(p["pos"], desc.dim)
        np.testing.assert_array_equal(cells, want_cells)
        np.testing.assert_array_equal(np.diff(start), want_counts)


@pytest.mark.gpu
def test_noalloc_at_its_limits_and_empty():
    rng = np.random.default_rng(21)
    full = rng.random((1 << 20, 3), dtype=np.float32)  # 2^20 particles on a 64^3 grid
    _check(full, 64)
    cells, start, order = _noalloc(np.zeros((0, 3), np.float32), 64)
    assert len(cells) == 0 and len(order) == 0 and (start == 0).all()
    _check(rng.random((5000, 3), dtype=np.float32), 64)  # after the full call: counters reset


@pytest.mark.gpu
def test_noalloc_crowded_cells():
    """Cells of 40 (bitonic network), 3,000 (bitonic, largest padding) and 6,000 particles (rank
    path), plus unit-cube violators clamped into the edge cells, in one call; then again with
    the particles shuffled."""
    rng = np.random.default_rng(8)
    dim = 16
    parts = [rng.random((20000, 3), dtype=np.float32)]
    for cnt, cell in ((40, (3, 4, 5)), (3000, (7, 7, 7)), (6000, (10, 2, 9))):
        parts.append(((np.array(cell, np.float32) + rng.random((cnt, 3), dtype=np.float32) * 0.98 + 0.01) / dim)
                     .astype(np.float32))
    parts.append((rng.random((500, 3), dtype=np.float32) * 4.0 - 1.5).astype(np.float32))
    pos = np.concatenate(parts)
    counts = _check(pos, dim)
    assert counts.max() >= 6000
    _check(pos[rng.permutation(len(pos))], dim)


@pytest.mark.gpu
def test_noalloc_rejects_oversize():
    L = lib()
    big_grid = L.ariel_sort_by_cell_noalloc(None, 0, 65, None, C.c_void_p(1), None, None)
    assert big_grid == A.ARIEL_ERR_INVALID_ARG
    too_many = L.ariel_sort_by_cell_noalloc(C.c_void_p(1), (1 << 20) + 1, 16, C.c_void_p(1), C.c_void_p(1),
                                            C.c_void_p(1), None)
    assert too_many == A.ARIEL_ERR_INVALID_ARG
