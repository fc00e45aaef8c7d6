"""Stage outputs of the reference's own FLIP step, committed as fixtures (tests/golden/
reference_*.npz, written by tests/golden/make_reference_golden.py from the reference's sources
compiled into oracle/_ref/), replayed on the oracle (CPU) and on the CUDA library (GPU).

Every stage must reproduce the reference bit for bit -- cell indices and counts, densities, face
velocities, flags, liquid SDF, divergence, particle positions and velocities -- except the pressure
solve.  The oracle, run in the reference's configuration, reproduces the pressure bit for bit too.
The CUDA library's REF32 solve runs the reference's algorithm and absolute stop rule in fp32 but
accumulates its dot products in fp64, so its pressure agrees to within the solve's rounding; after
the solve the reference's pressure is loaded so that the later stages start from the same state.
"""
import os

import numpy as np
import pytest

from ariel_b200 import _abi as A

from helpers import assert_bits

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["dambreak16", "sphere16"]
GRID_KEYS = {A.GRID_UX: "ux", A.GRID_UY: "uy", A.GRID_UZ: "uz", A.GRID_PREV_UX: "pux",
             A.GRID_PREV_UY: "puy", A.GRID_PREV_UZ: "puz", A.GRID_D: "D", A.GRID_P: "P", A.GRID_L: "L",
             A.GRID_A: "A"}
FACES = (A.GRID_UX, A.GRID_UY, A.GRID_UZ)
PREV = (A.GRID_PREV_UX, A.GRID_PREV_UY, A.GRID_PREV_UZ)


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", "reference_%s.npz" % name)))


def desc_of(g):
    spheres = [((float(s[0]), float(s[1]), float(s[2])), float(s[3])) for s in g["spheres"]]
    return A.scene_dambreak(int(g["n"]), liquid_hi=tuple(float(v) for v in g["hi"]), seed=int(g["seed"]),
                            spheres=spheres, dt=float(g["dt"]))


def params_of(g, precision=A.PREC_REF32):
    p = A.params_default()
    p.precision = precision
    p.precond = A.PRECOND_REF
    p.stop_rule = A.STOP_REF_ABS
    p.resample_every = 1
    p.rng_seed = int(g["rng_seed"])
    p.use_graph = 0
    return p


def replay(sim, g, name, check_solve):
    """Runs the 12 stages on `sim` (oracle or CUDA handle) from the fixture's input state and
    compares each stage with the reference's outputs."""
    sim.set_particles(g["in_pos"], g["in_vel"], g["in_mass"], g["in_type"])
    sim.set_grid(A.GRID_P, g["in_P"])
    assert sim.max_density() == float(g["max_density"]), name + " density normaliser"

    def grids(stage, which):
        for w in which:
            key = "%s_%s" % (stage, GRID_KEYS[w])
            assert_bits("%s %s" % (name, key), sim.get_grid(w), g[key])

    for stage in range(A.STAGE_COUNT):
        sim.stage(stage)
        s = A.STAGE_NAMES[stage]
        tag = "%s/%s" % (name, s)
        if stage in (A.STAGE_BEGIN, A.STAGE_G2P_ADVECT, A.STAGE_RESAMPLE):
            p = sim.get_particles()
            assert_bits(tag + " pos", p["pos"], g[s + "_pos"])
            assert_bits(tag + " vel", p["vel"], g[s + "_vel"])
        elif stage == A.STAGE_SORT:
            pc, cc = sim.get_cells()
            assert_bits(tag + " particle->cell", pc, g["sort_particle_cell"])
            assert_bits(tag + " per-cell counts", cc, g["sort_cell_count"])
        elif stage == A.STAGE_DENSITY:
            assert_bits(tag + " density", sim.get_particles()["density"], g["density_density"])
        elif stage == A.STAGE_FORCES:
            assert_bits(tag + " vel", sim.get_particles()["vel"], g["forces_vel"])
        elif stage == A.STAGE_P2G:
            grids(s, FACES)
        elif stage == A.STAGE_CLASSIFY:
            grids(s, (A.GRID_A, A.GRID_L))
        elif stage == A.STAGE_BOUNDARY_DIV:
            grids(s, FACES + PREV + (A.GRID_D,))
        elif stage == A.STAGE_SOLVE:
            check_solve(tag, sim.get_grid(A.GRID_P), g["solve_P"], g["classify_A"])
            sim.set_grid(A.GRID_P, g["solve_P"])
        elif stage == A.STAGE_GRADIENT:
            grids(s, FACES)
        elif stage == A.STAGE_EXTRAPOLATE:
            grids(s, FACES + PREV)


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_fixture(name):
    from oracle.pyoracle import RefSim
    g = load(name)
    ora = RefSim(desc_of(g), params_of(g))

    def exact(tag, got, want, flags):
        assert_bits(tag + " P", got, want)

    replay(ora, g, name, exact)
    ora.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cuda_reproduces_reference_fixture(name):
    from ariel_b200.flipsim import Batch
    g = load(name)
    gpu = Batch([desc_of(g)], params_of(g))

    def close(tag, got, want, flags):
        fl = flags == A.FLUID
        assert (got[~fl] == 0).all(), tag + ": non-FLUID pressure must be 0 (solver.inl:160-176)"
        scale = float(np.abs(want[fl]).max())
        err = float(np.abs(got[fl].astype(np.float64) - want[fl]).max()) / scale
        # same algorithm, same fp32 vectors and stop rule; only the dot-product rounding differs
        assert err <= 1e-4, "%s P: max relative difference %.3e" % (tag, err)

    replay(gpu, g, name, close)
    gpu.close()
