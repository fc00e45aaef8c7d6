"""CPU checks that pin the oracle (the C++ restatement of the reference step).

The reference ships no tests or golden vectors and cannot be built here, so the oracle is
pinned by: published Philox4x32-10 known answers, the reference's lattice-seeding count,
golden stage outputs from an independent numpy restatement (tests/golden/make_golden.py),
and hand-derived physical answers.
"""
import os

import numpy as np
import pytest

from ariel_b200 import _abi as A
from oracle.pyoracle import RefSim, philox

from helpers import assert_bits, dambreak, params

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "stages_n8.npz")


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32-10
    assert list(philox([0, 0, 0, 0], [0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(philox([0xffffffff] * 4, [0xffffffff] * 2)) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0])) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_dambreak_lattice_count():
    # Scene::GenerateParticles' sub-cell lattice (scene.cpp:283-304) inside x<.4, y<.6, z<1 at
    # density .5: 51 x 77 x 128 lattice points on a 64^3 grid.
    r = RefSim(dambreak(64), params())
    r.init()
    assert r.count() == 51 * 77 * 128
    flags = r.get_grid(A.GRID_A)
    # Init's MarkCellTypes runs with the seeding density 10 (scene.cpp:448): every occupied
    # cell is FLUID, the block covers cells x<26, y<39
    assert flags[:25, :38, :].min() == A.FLUID and flags[27:, :, :].max() == A.AIR


def _golden_oracle():
    g = np.load(GOLDEN)
    n = int(g["n"])
    desc = A.scene_dambreak(n)
    desc.density = float(g["density"])
    prm = params()
    r = RefSim(desc, prm)
    r.set_particles(g["pos"], g["vel"], g["mass"], g["type"])
    return g, r


def test_oracle_matches_numpy_golden():
    g, r = _golden_oracle()
    assert r.max_density() == float(g["max_density"])
    r.stage(A.STAGE_SORT)
    pc, cc = r.get_cells()
    assert_bits("particle cell", pc, g["particle_cell"])
    assert_bits("cell counts", cc, g["cell_count"])
    r.stage(A.STAGE_DENSITY)
    assert_bits("density", r.get_particles()["density"], g["dens"])
    r.stage(A.STAGE_FORCES)
    assert_bits("velocity after forces", r.get_particles()["vel"], g["vel_forced"])
    r.stage(A.STAGE_P2G)
    for w, k in [(A.GRID_UX, "ux"), (A.GRID_UY, "uy"), (A.GRID_UZ, "uz")]:
        assert_bits(k, r.get_grid(w), g[k])
    r.stage(A.STAGE_CLASSIFY)
    assert_bits("flags", r.get_grid(A.GRID_A), g["flags"])
    assert_bits("L", r.get_grid(A.GRID_L), g["L"])
    r.stage(A.STAGE_BOUNDARY_DIV)
    for w, k in [(A.GRID_PREV_UX, "pux"), (A.GRID_PREV_UY, "puy"), (A.GRID_PREV_UZ, "puz"),
                 (A.GRID_UX, "ex"), (A.GRID_UY, "ey"), (A.GRID_UZ, "ez"), (A.GRID_D, "D")]:
        assert_bits(k, r.get_grid(w), g[k])


def test_single_particle_splat():
    """One FLUID particle: a face takes exactly the particle's velocity component when the
    particle lies in the face's 2x4x4 cell block within the Sharpen radius 1.4 cells, else 0
    (particlegridoperations.inl:146-249)."""
    n = 8
    r = RefSim(dambreak(n), params())
    p = np.array([[0.43, 0.52, 0.37]], np.float32)
    u = np.array([[0.7, -1.25, 2.5]], np.float32)
    r.set_particles(p, u, np.ones(1, np.float32), np.array([A.FLUID], np.int32))
    r.stage(A.STAGE_SORT)
    r.stage(A.STAGE_P2G)
    gp = p[0] * n
    cell = np.floor(gp).astype(int)
    for axis, w in enumerate((A.GRID_UX, A.GRID_UY, A.GRID_UZ)):
        grid = r.get_grid(w)
        for idx in np.ndindex(grid.shape):
            fc = np.array(idx, np.float64) + 0.5
            fc[axis] -= 0.5
            lo = np.array(idx) - 2
            lo[axis] = idx[axis] - 1
            hi = np.array(idx) + 1
            hi[axis] = idx[axis]
            inside = np.all(cell >= lo) and np.all(cell <= hi)
            near = ((gp - fc) ** 2).sum() < 1.4 ** 2 - 1e-4
            far = ((gp - fc) ** 2).sum() > 1.4 ** 2 + 1e-4
            if inside and near:
                # (w*u)/w: two fp32 roundings, so within an ulp of u
                assert abs(grid[idx] - u[0, axis]) <= 2.5e-7 * abs(u[0, axis]), (axis, idx, grid[idx])
            elif (not inside) or far:
                assert grid[idx] == 0.0, (axis, idx, grid[idx])


def test_hydrostatic_pressure_profile():
    """A liquid layer at rest over the full floor: after one step the pressure solve cancels
    gravity, so inside the layer P(j) - P(j-1) = -g dt h per cell (u_y(j) = -g dt,
    u_y -= (P(j) - P(j-1)) / h, flip.cpp:568-680).  The free surface comes from the particle
    density field (CellSDF, particlegrid.cpp:75-90), which is lower next to the walls, so the
    ghost-fluid surface and hence the slope vary by a few tenths of a percent across x/z."""
    n = 16
    desc = dambreak(n, hi=(1.0, 0.5, 1.0), jitter=0.0)
    prm = params(precision=A.PREC_FP64, stop=A.STOP_REL, tol=1e-10, resample_every=0)
    r = RefSim(desc, prm)
    r.init()
    for g in range(A.STAGE_GRADIENT):
        r.stage(g)
    P = r.get_grid(A.GRID_P).astype(np.float64)
    dP = P[:, 1:, :] - P[:, :-1, :]
    expect = -9.8 * (1.0 / 240.0) * (1.0 / n)
    core = dP[3:-3, 2:5, 3:-3]
    np.testing.assert_allclose(core, expect, rtol=1e-2)
    # and the projected interior vertical velocity nearly vanishes (g dt = 0.041)
    r.stage(A.STAGE_GRADIENT)
    uy = r.get_grid(A.GRID_UY)
    assert np.abs(uy[3:-3, 2:6, 3:-3]).max() < 1e-2 * 9.8 / 240.0
