"""Edge cases of the step: empty and ragged inputs, particles on the domain's faces and corners,
coincident particles, a full domain, batches past the fast solve kernel's scene limit, and the
argument limits."""
import ctypes as C
import os

import numpy as np
import pytest

from ariel_b200 import _abi as A
from ariel_b200 import _lib
from ariel_b200.flipsim import Batch
from oracle.pyoracle import RefSim

from helpers import assert_bits, dambreak, params, stage_parity


def _empty(n=12):
    d = dambreak(n)
    d.n_liquid = 0
    return d


@pytest.mark.gpu
def test_empty_scene_alone_and_in_a_batch():
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1)
    b = Batch([_empty()], prm)
    b.init()
    b.step(3)
    assert b.count() == 0
    st = b.stats()
    assert st.frame == 3 and st.pcg_converged == 1 and st.n_fluid_cells == 0
    assert not b.get_grid(A.GRID_P).any()
    b.close()
    # an empty scene between two others changes nothing for them
    descs = [dambreak(16, seed=1), _empty(), dambreak(12, seed=2)]
    batch = Batch(descs, prm)
    batch.init()
    batch.step(3)
    for i in (0, 2):
        alone = Batch([descs[i]], prm)
        alone.init()
        alone.step(3)
        assert_bits("scene %d pos" % i, batch.get_particles(i)["pos"], alone.get_particles()["pos"])
        alone.close()
    batch.close()


def _awkward_particles(n, seed=4):
    """Liquid on every face, edge and corner of the domain, a stack of coincident particles,
    and an ordinary block -- all FLUID, unit mass."""
    rng = np.random.default_rng(seed)
    pts = []
    for x in (0.0, 1.0, 1.0 - 1e-7):
        for y in (0.0, 0.5, 1.0):
            for z in (0.0, 1.0, 0.25):
                pts.append((x, y, z))
    # coincident: the resampler's jitter branch; 23 particles in one cell also take the sort's
    # path for cells of more than 16 particles
    pts += [(0.5, 0.5, 0.5)] * 20
    pts += [(0.5 + 1e-7, 0.5, 0.5)] * 3
    blk = rng.uniform(0.05, 0.45, size=(400, 3))
    blk[:, 1] *= 0.5
    pts = np.concatenate([np.array(pts, np.float32), blk.astype(np.float32)])
    vel = rng.uniform(-0.5, 0.5, size=pts.shape).astype(np.float32)
    return pts, vel, np.ones(len(pts), np.float32), np.full(len(pts), A.FLUID, np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [8, 13])
def test_boundary_and_coincident_particles_bit_exact(n):
    """Stage-by-stage parity with the oracle when particles sit exactly on the domain's faces
    and corners (clamps and truncations at 0 and n) and when many share one position."""
    prm = params(stop=A.STOP_REL, tol=1e-6)
    desc = dambreak(n)
    pos, vel, mass, typ = _awkward_particles(n)
    ora = RefSim(desc, prm)
    ora.set_particles(pos, vel, mass, typ)
    gpu = Batch([desc], prm)
    gpu.set_particles(pos, vel, mass, typ)
    assert gpu.max_density() == ora.max_density()
    stage_parity("awkward%d" % n, gpu, ora)
    ora.close()
    gpu.close()


@pytest.mark.gpu
def test_full_domain_liquid_steps():
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1)
    b = Batch([dambreak(12, hi=(1.0, 1.0, 1.0))], prm)
    b.init()
    b.step(2)
    st = b.stats()
    assert st.pcg_converged == 1 and st.n_fluid_cells > 0.9 * 12 ** 3
    p = b.get_particles()
    assert np.isfinite(p["pos"]).all() and np.isfinite(p["vel"]).all()
    assert (p["pos"] >= 0).all() and (p["pos"] <= 1).all()
    b.close()


@pytest.mark.gpu
def test_batch_past_fast_kernel_limit():
    """130 scenes exceed the fast solve kernel's 128-scene limit, so the general kernel solves
    them; each scene still converges and matches the same scene solved alone within the solve
    tolerance."""
    descs = [dambreak(8 + (i % 5), seed=i + 1) for i in range(130)]
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-6, graph=1)
    batch = Batch(descs, prm)
    batch.init()
    batch.step(2)
    for i in (0, 64, 129):
        st = batch.stats(i)
        assert st.pcg_converged == 1 and st.pcg_rel_residual <= 1e-6
        alone = Batch([descs[i]], prm)
        alone.init()
        alone.step(2)
        pa, pb = alone.get_particles()["pos"], batch.get_particles(i)["pos"]
        assert np.abs(pa - pb).max() < 1e-5
        alone.close()
    batch.close()


def test_argument_limits():
    L = _lib.lib()
    p = A.params_default()
    h = C.c_void_p()
    big = A.scene_dambreak(1025)
    assert L.ariel_create(C.byref(big), C.byref(p), C.byref(h)) == A.ARIEL_ERR_INVALID_ARG
    d = A.scene_dambreak(16)
    d.n_liquid = A.MAX_BOXES + 1
    assert L.ariel_create(C.byref(d), C.byref(p), C.byref(h)) == A.ARIEL_ERR_INVALID_ARG
    d = A.scene_dambreak(16)
    d.stepsize = 0.0
    assert L.ariel_create(C.byref(d), C.byref(p), C.byref(h)) == A.ARIEL_ERR_INVALID_ARG
    arr = (A.AsimSceneDesc * 1025)(*([A.scene_dambreak(8)] * 1025))
    assert L.ariel_create_batch(arr, 1025, C.byref(p), C.byref(h)) == A.ARIEL_ERR_INVALID_ARG
    d = A.scene_dambreak(16)
    q = A.params_default()
    q.p2g_faces = 3
    assert L.ariel_create(C.byref(d), C.byref(q), C.byref(h)) == A.ARIEL_ERR_INVALID_ARG
