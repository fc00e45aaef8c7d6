"""Reseeding: on its frames, particles move from FLUID cells above reseed_max to interior FLUID
cells below reseed_min, with the particle count, ids, masses and types kept.  The reference never
adds or removes particles, so the rule is checked against a numpy restatement of it: which
particles move (the highest ids of each crowded cell), into which cells (the r-th given particle
to the r-th received place, cells in index order), and the cell counts after the move.
"""
import numpy as np
import pytest

from ariel_b200 import _abi as A
from ariel_b200.flipsim import Batch

from helpers import assert_bits, dambreak, params


def _cells(pos, n):
    """cell_coord of every particle: truncation of n * x clamped to [0, n - 1], per axis."""
    g = np.clip(np.float32(n) * pos.astype(np.float32), np.float32(0), np.float32(n - 1)).astype(np.int64)
    return (g[:, 0] * n + g[:, 1]) * n + g[:, 2]


def _rule(cell, flags, n, lo, hi):
    """The particles that move (ids, highest first inside each giving cell, cells in index
    order) and the cell each one lands in."""
    nc = n ** 3
    counts = np.bincount(cell, minlength=nc)
    fluid = (flags.reshape(-1) == A.FLUID)
    give = np.where(fluid & (counts > hi), counts - hi, 0)
    f3 = fluid.reshape(n, n, n)
    inner = np.zeros((n, n, n), bool)
    inner[1:-1, 1:-1, 1:-1] = (f3[1:-1, 1:-1, 1:-1] & f3[:-2, 1:-1, 1:-1] & f3[2:, 1:-1, 1:-1] &
                               f3[1:-1, :-2, 1:-1] & f3[1:-1, 2:, 1:-1] & f3[1:-1, 1:-1, :-2] & f3[1:-1, 1:-1, 2:])
    take = np.where(inner.reshape(-1) & (counts < lo), lo - counts, 0)
    movers = []
    for c in np.nonzero(give)[0]:
        ids = np.sort(np.nonzero(cell == c)[0])[::-1]
        movers.extend(ids[:give[c]].tolist())
    places = np.repeat(np.arange(nc), take)
    m = min(len(movers), len(places))
    return np.array(movers[:m], np.int64), places[:m], counts


def _crowded_state(n, big):
    """A 16^3 dam break's initial particles (8 in every cell of the block) and its FLUID flags.
    Either three interior cells are crowded by 4 particles from each of nine others, or one
    interior cell takes every particle of 40 others (328 particles in one cell)."""
    desc = dambreak(n, seed=3)
    b = Batch([desc], params())
    b.init()
    st = b.get_particles()
    b.close()
    pos = st["pos"].copy()
    cell = _cells(pos, n)
    flags = np.where(np.bincount(cell, minlength=n ** 3) > 0, A.FLUID, A.AIR).astype(np.uint8).reshape(n, n, n)
    rng = np.random.default_rng(5)
    if big:
        sinks = [(3, 4, 8)]
        sources = [(i, j, k) for i in (1, 2, 4, 5) for j in (2, 6) for k in (2, 4, 7, 10, 13)]
        take = 8
    else:
        sinks = [(2, 3, 5), (3, 4, 9), (4, 2, 12)]
        sources = [(2, 5, 3), (3, 2, 4), (4, 4, 6), (2, 6, 8), (3, 3, 11), (4, 5, 13), (2, 2, 10), (3, 6, 7),
                   (4, 3, 2)]
        take = 4
    for si, s in enumerate(sources):
        ids = np.nonzero(cell == (s[0] * n + s[1]) * n + s[2])[0][:take]
        t = sinks[si % len(sinks)]
        pos[ids] = (np.array(t, np.float32) + rng.uniform(0.1, 0.9, (len(ids), 3)).astype(np.float32)) / n
    return desc, st, pos, flags


@pytest.mark.gpu
@pytest.mark.parametrize("big", [False, True], ids=["three_cells", "one_cell_of_328"])
def test_reseed_follows_the_rule(big):
    n, lo, hi = 16, 6, 10
    desc, st, pos, flags = _crowded_state(n, big)
    cell = _cells(pos, n)
    counts = np.bincount(cell, minlength=n ** 3)
    movers, places, _ = _rule(cell, flags, n, lo, hi)
    # three cells: the sinks hold 20 (10 to give), the sources 4 (2 to receive), so 18 move and
    # the last sink in index order keeps its crowd.  One cell: it holds 328 (318 to give), the
    # 40 emptied cells receive 6 each
    assert len(movers) == (240 if big else 18)
    prm = params(resample_every=0, reseed_every=1, reseed_min=lo, reseed_max=hi)
    g = Batch([desc], prm)
    g.set_particles(pos, st["vel"], st["mass"], st["type"])
    g.set_grid(A.GRID_A, flags)
    ux = np.full((n + 1, n, n), 0.25, np.float32)
    uy = np.full((n, n + 1, n), -0.5, np.float32)
    uz = np.full((n, n, n + 1), 1.0, np.float32)
    g.set_grid(A.GRID_UX, ux)
    g.set_grid(A.GRID_UY, uy)
    g.set_grid(A.GRID_UZ, uz)
    g.stage(A.STAGE_RESAMPLE)
    out = g.get_particles()
    g.close()
    moved = np.zeros(len(pos), bool)
    moved[movers] = True
    # everything else is untouched, bit for bit
    assert_bits("unmoved pos", out["pos"][~moved], pos[~moved])
    assert_bits("unmoved vel", out["vel"][~moved], st["vel"][~moved])
    assert_bits("mass", out["mass"], st["mass"])
    assert_bits("type", out["type"], st["type"])
    # the moved particles sit in their receiving cells, away from the faces, with the grid's
    # (constant) velocity
    got = _cells(out["pos"][movers], n)
    assert np.array_equal(got, places)
    frac = np.float32(n) * out["pos"][movers] - np.floor(np.float32(n) * out["pos"][movers])
    assert (frac > 0.04).all() and (frac < 0.96).all()
    assert np.allclose(out["vel"][movers], [0.25, -0.5, 1.0], rtol=1e-6, atol=1e-7)
    after = np.bincount(_cells(out["pos"], n), minlength=n ** 3)
    want = counts - np.bincount(cell[movers], minlength=n ** 3) + np.bincount(places, minlength=n ** 3)
    assert np.array_equal(after, want)
    assert after[places].min() == lo

    # frame 1 with reseed_every = 2: nothing moves
    g = Batch([desc], params(resample_every=0, reseed_every=2, reseed_min=lo, reseed_max=hi))
    g.set_particles(pos, st["vel"], st["mass"], st["type"])
    g.set_grid(A.GRID_A, flags)
    g.stage(A.STAGE_BEGIN)
    assert g.stats().frame == 1
    g.stage(A.STAGE_RESAMPLE)
    out = g.get_particles()
    g.close()
    assert_bits("off-frame pos", out["pos"], pos)
    assert_bits("off-frame vel", out["vel"], st["vel"])


@pytest.mark.gpu
def test_reseed_batch_equals_alone():
    """A batch of scenes (one with a solid sphere), resampled and reseeded every second step,
    gives each scene exactly what it gives stepped alone."""
    descs = [dambreak(24, seed=2, hi=(0.35, 0.5, 1.0), spheres=[((0.6, 0.3, 0.5), 0.15)]), dambreak(16, seed=4)]
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1, resample_every=2, reseed_every=2,
                 reseed_min=8, reseed_max=8)
    batch = Batch(descs, prm)
    batch.init()
    batch.step(6)
    for i, d in enumerate(descs):
        alone = Batch([d], prm)
        alone.init()
        alone.step(6)
        a, b = alone.get_particles(), batch.get_particles(i)
        assert_bits("scene %d pos" % i, b["pos"], a["pos"])
        assert_bits("scene %d vel" % i, b["vel"], a["vel"])
        alone.close()
    batch.close()


def test_reseed_arguments():
    """Bounds are checked before any device work: min above max, negative values and more than
    65535 particles per cell are refused."""
    import ctypes as C

    from ariel_b200 import _lib
    L = _lib.lib()
    d = A.scene_dambreak(16)
    h = C.c_void_p()
    for kw in ({"reseed_every": -1}, {"reseed_min": 12, "reseed_max": 8}, {"reseed_min": -2},
               {"reseed_max": 70000}):
        p = A.params_default()
        p.reseed_every = 1
        for k, v in kw.items():
            setattr(p, k, v)
        assert L.ariel_create(C.byref(d), C.byref(p), C.byref(h)) == A.ARIEL_ERR_INVALID_ARG, kw


@pytest.mark.gpu
def test_reseed_moves_particles_in_a_running_scene():
    """In an evolving dam break with bounds of 8 and 8, reseeding frames move particles (the
    positions differ from the same run without reseeding) while the count and the particles'
    masses and types stay."""
    d = dambreak(16, seed=4)
    runs = []
    for every in (0, 2):
        b = Batch([d], params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1, reseed_every=every,
                              reseed_min=8, reseed_max=8))
        b.init()
        b.step(6)
        runs.append(b.get_particles())
        b.close()
    assert len(runs[0]["pos"]) == len(runs[1]["pos"])
    assert not np.array_equal(runs[0]["pos"], runs[1]["pos"])
    assert_bits("mass", runs[1]["mass"], runs[0]["mass"])
    assert_bits("type", runs[1]["type"], runs[0]["type"])
    assert np.isfinite(runs[1]["pos"]).all() and np.isfinite(runs[1]["vel"]).all()
