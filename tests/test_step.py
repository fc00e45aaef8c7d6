"""Whole-step parity (GPU vs oracle) and batch equivalence."""
import numpy as np
import pytest

from ariel_b200 import _abi as A
from ariel_b200.flipsim import Batch, FlipSim
from oracle.pyoracle import RefSim

from helpers import assert_bits, dambreak, params


@pytest.mark.gpu
@pytest.mark.parametrize("n,graph", [(16, 0), (16, 1), (32, 1)])
def test_first_step_matches_oracle(n, graph):
    """From Init, one full step: the flags are decided before the pressure solve and must be
    bit-exact; particle state after the solve agrees to the solve's tolerance."""
    desc = dambreak(n, seed=2)
    prm = params(stop=A.STOP_REL, tol=1e-6, graph=graph)
    ora = RefSim(desc, prm)
    ora.init()
    gpu = Batch([desc], prm)
    gpu.init()
    assert gpu.count() == ora.count()
    assert_bits("init positions", gpu.get_particles()["pos"], ora.get_particles()["pos"])
    assert_bits("init flags", gpu.get_grid(A.GRID_A), ora.get_grid(A.GRID_A))
    ora.step(1)
    gpu.step(1)
    assert_bits("step-1 flags", gpu.get_grid(A.GRID_A), ora.get_grid(A.GRID_A))
    assert_bits("step-1 L", gpu.get_grid(A.GRID_L), ora.get_grid(A.GRID_L))
    gp, op = gpu.get_particles(), ora.get_particles()
    vscale = np.abs(op["vel"]).max()
    np.testing.assert_allclose(gp["vel"] / vscale, op["vel"] / vscale, rtol=0, atol=1e-3)
    np.testing.assert_allclose(gp["pos"], op["pos"], rtol=0, atol=1e-5)
    assert gpu.stats().frame == ora.stats().frame == 1


@pytest.mark.gpu
def test_multistep_properties():
    """Size-independent properties over many steps at 64^3: particle count conserved, every
    FLUID particle inside [1/n, 1-1/n] after advection, pressure solved each step, and the
    flag field stays a valid cell-type field."""
    n = 64
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1)
    sim = FlipSim(n, 0.5, 1.0 / 240.0, dambreak(n), params=prm)
    sim.Init()
    n0 = sim.batch.count()
    for _ in range(10):
        sim.Step()
    st = sim.batch.stats()
    assert st.pcg_converged and st.pcg_rel_residual <= 1e-5 * 1.01
    p = sim.GetParticles()
    assert len(p["pos"]) == n0 and np.isfinite(p["pos"]).all() and np.isfinite(p["vel"]).all()
    flags = sim.batch.get_grid(A.GRID_A)
    assert set(np.unique(flags)) <= {A.AIR, A.FLUID}
    assert sim.m_frame == 10 and st.frame == 10
    # the liquid falls: mean y velocity negative, mean height decreased
    assert p["vel"][:, 1].mean() < 0


@pytest.mark.gpu
@pytest.mark.parametrize("p2g_faces", [0, 2, 4])
def test_batch_equals_alone(p2g_faces):
    """Scenes of different sizes stepped in one batch give bit-identical results to each scene
    stepped alone (chunked reductions depend only on each scene's own cells), also when the
    batch's grid transfer runs several faces per thread across row and scene boundaries."""
    descs = [dambreak(16, seed=1), dambreak(24, seed=2, hi=(0.3, 0.5, 1.0)), dambreak(12, seed=3)]
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1)
    batch = Batch(descs, params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1, p2g_faces=p2g_faces))
    batch.init()
    batch.step(4)
    for i, d in enumerate(descs):
        alone = Batch([d], prm)
        alone.init()
        alone.step(4)
        a, b = alone.get_particles(), batch.get_particles(i)
        assert_bits("scene %d pos" % i, b["pos"], a["pos"])
        assert_bits("scene %d vel" % i, b["vel"], a["vel"])
        assert_bits("scene %d P" % i, batch.get_grid(A.GRID_P, i), alone.get_grid(A.GRID_P))
        assert batch.stats(i).pcg_iterations == alone.stats().pcg_iterations
        alone.close()
    batch.close()


@pytest.mark.gpu
def test_graph_survives_state_rebuild():
    """Step graphs captured before the state is rebuilt (set_particles re-allocates every buffer)
    are updated to the new buffers before their next replay: the run matches an ungraphed one."""
    d = dambreak(16, seed=2)
    runs = []
    for graph in (1, 0):
        b = Batch([d], params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=graph))
        b.init()
        b.step(2)
        p = b.get_particles()
        b.set_particles(p["pos"], p["vel"], p["mass"], p["type"])
        b.step(2)
        runs.append(b.get_particles())
        b.close()
    assert_bits("pos", runs[0]["pos"], runs[1]["pos"])
    assert_bits("vel", runs[0]["vel"], runs[1]["vel"])
