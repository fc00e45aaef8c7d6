"""GPU-vs-oracle parity at the benchmark configurations' sizes.

The stage-by-stage comparison of tests/test_parity_stages.py, run where the size-dependent paths
of the CUDA library engage:
  * the 64^3 dam break (502,656 particles) straight from Init and after ten
    oracle steps, and one whole step from Init;
  * the 128^3 dam break (4,021,248 particles) from Init;
  * the sphere scene's shape -- liquid beside a static solid sphere c = (.6,.3,.5), r = .15, dt = 1/480,
    resampling every 5th step -- at 64^3, evolved to frame 4 and compared across a resampling
    step;
  * the pressure solve's streamed chunks (each persistent block holds only its first chunk's
    records in shared memory; capping the solve grid at 24 blocks makes most chunks stream).
The neighbour kernels' power-of-two shortcuts (h^2 of the density kernel, re of the resampler)
are taken at n = 64 and 128, and evolved dam breaks hold cells of more than 16 particles.
"""
import numpy as np
import pytest

from ariel_b200 import _abi as A
from ariel_b200.flipsim import Batch
from oracle.pyoracle import RefSim

from helpers import assert_bits, dambreak, params, stage_parity


def _pair_from(st, P, P64, desc, prm):
    ora = RefSim(desc, prm)
    ora.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
    ora.set_grid(A.GRID_P, P)
    ora.set_grid(A.GRID_P64, P64)
    gpu = Batch([desc], prm)
    gpu.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
    gpu.set_grid(A.GRID_P, P)
    gpu.set_grid(A.GRID_P64, P64)
    return ora, gpu


def _evolve(desc, prm, steps):
    r = RefSim(desc, prm)
    r.init()
    if steps:
        r.step(steps)
    out = r.get_particles(), r.get_grid(A.GRID_P), r.get_grid(A.GRID_P64)
    r.close()
    return out


def _max_cell_count(h):
    return int(h.get_cells()[1].max())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 96, 128])
def test_stage_parity_from_init(n):
    """The 64^3 and 128^3 dam breaks, and 96^3, whose grid index divisors (n, n + 1, n^2,
    n (n + 1)) have inexact reciprocals: both sides run their own Init (seeding, density
    normaliser, first sort and classification), then every stage of the first step is compared."""
    desc = dambreak(n, seed=1)
    prm = params(stop=A.STOP_REL, tol=1e-6)
    ora = RefSim(desc, prm)
    ora.init()
    gpu = Batch([desc], prm)
    gpu.init()
    assert gpu.count() == ora.count()
    if n in (64, 128):
        assert gpu.count() == {64: 502656, 128: 4021248}[n]
    assert gpu.max_density() == ora.max_density()
    assert_bits("init pos", gpu.get_particles()["pos"], ora.get_particles()["pos"])
    assert_bits("init flags", gpu.get_grid(A.GRID_A), ora.get_grid(A.GRID_A))
    stage_parity("dambreak%d_init" % n, gpu, ora)
    ora.close()
    gpu.close()


@pytest.mark.gpu
@pytest.mark.parametrize("grid_blocks", [0, 24], ids=["resident_grid", "streamed_chunks"])
def test_stage_parity_64_evolved(grid_blocks):
    """The 64^3 dam break after ten oracle steps (a sloshing state with crowded cells)."""
    desc = dambreak(64, seed=1)
    prm = params(stop=A.STOP_REL, tol=1e-6, pcg_grid_blocks=grid_blocks)
    st, P, P64 = _evolve(desc, prm, 10)
    ora, gpu = _pair_from(st, P, P64, desc, prm)
    stage_parity("dambreak64_evolved", gpu, ora)
    assert _max_cell_count(ora) > 16
    ora.close()
    gpu.close()


@pytest.mark.gpu
def test_whole_step_from_init_64():
    """The 64^3 dam break: one full step from Init on both sides; flags and SDF are decided before the solve and
    are bit-exact, particle state after the solve agrees to the solve's tolerance."""
    desc = dambreak(64, seed=1)
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-6, graph=1)
    ora = RefSim(desc, params(stop=A.STOP_REL, tol=1e-6))
    ora.init()
    gpu = Batch([desc], prm)
    gpu.init()
    ora.step(1)
    gpu.step(1)
    assert_bits("step-1 flags", gpu.get_grid(A.GRID_A), ora.get_grid(A.GRID_A))
    assert_bits("step-1 L", gpu.get_grid(A.GRID_L), ora.get_grid(A.GRID_L))
    gp, op = gpu.get_particles(), ora.get_particles()
    vscale = np.abs(op["vel"]).max()
    np.testing.assert_allclose(gp["vel"] / vscale, op["vel"] / vscale, rtol=0, atol=1e-4)
    np.testing.assert_allclose(gp["pos"], op["pos"], rtol=0, atol=1e-6)
    ora.close()
    gpu.close()


@pytest.mark.gpu
def test_stage_parity_sphere_resample_64():
    """The sphere scene (dam break with a solid sphere at (.6, .3, .5), r .15, dt 1/480) at 64^3:
    evolved by the oracle to frame 4 with resampling every 5th step,
    then one step with resampling on, stage by stage (sphere push-out, solid constraints and the
    resampler's springs and jitter included)."""
    desc = dambreak(64, seed=3, hi=(0.35, 0.5, 1.0), spheres=[((0.6, 0.3, 0.5), 0.15)])
    desc.stepsize = 1.0 / 480.0
    st, P, P64 = _evolve(desc, params(stop=A.STOP_REL, tol=1e-6, resample_every=5), 4)
    assert (st["type"] == A.SOLID).any()
    prm = params(stop=A.STOP_REL, tol=1e-6, resample_every=1)
    ora, gpu = _pair_from(st, P, P64, desc, prm)
    stage_parity("sphere64_resample", gpu, ora)
    flags = ora.get_grid(A.GRID_A)
    assert (flags == A.SOLID).any()
    ora.close()
    gpu.close()
