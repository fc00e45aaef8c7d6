"""Request server (continuous batching): scenes that join and leave a running batch give the
same particles as the same scene stepped alone, admission respects the device-byte budget, and
the accounting adds up.

The tolerance of the served-vs-alone comparison is zero: every reduction of the step is
chunked per scene, so a scene's arithmetic does not depend on which other scenes share the
launches or where its cells sit in the packed layout.
"""
import os
import time

import pytest

from ariel_b200 import _abi as A
from ariel_b200.flipsim import Batch, Server, state_bytes

from helpers import assert_bits, dambreak, params


def _alone(desc, prm, nsteps):
    b = Batch([desc], prm)
    b.init()
    b.step(nsteps)
    p = b.get_particles()
    b.close()
    return p["pos"], p["vel"]


def _wait_steps(srv, rid, k, timeout_s=120.0):
    t = time.time()
    while srv.poll(rid).steps_done < k:
        assert time.time() - t < timeout_s, "request %d never reached step %d" % (rid, k)
        time.sleep(0.002)


def _scenes():
    return [
        (dambreak(16, seed=1), 14),
        (dambreak(24, seed=2, hi=(0.3, 0.5, 1.0)), 6),
        (dambreak(20, seed=3, spheres=[((0.6, 0.3, 0.5), 0.15)]), 9),
        (dambreak(12, seed=4), 5),
    ]


@pytest.mark.gpu
@pytest.mark.parametrize("reseed_every", [0, 2])
def test_served_equals_alone(reseed_every):
    # with reseeding (bounds of 8 and 8, so that the evolving dam breaks do move particles),
    # each scene reseeds on its own frames whatever batch it runs in
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1, reseed_every=reseed_every,
                 reseed_min=8, reseed_max=8)
    scenes = _scenes()
    with Server(prm, max_live=8) as srv:
        ids = [srv.submit(*scenes[0])]
        _wait_steps(srv, ids[0], 3)            # joins a running batch
        ids.append(srv.submit(*scenes[1]))
        ids.append(srv.submit(*scenes[2]))
        srv.wait(ids[1])                       # a scene leaves while others run
        ids.append(srv.submit(*scenes[3]))
        srv.drain()
        st = srv.stats()
        for rid, (d, n) in zip(ids, scenes):
            info = srv.poll(rid)
            assert info.state == A.REQ_DONE and info.steps_done == n
            assert info.stats.frame == n
            pos, vel = srv.fetch(rid)
            apos, avel = _alone(d, prm, n)
            assert_bits("request %d pos" % rid, pos, apos)
            assert_bits("request %d vel" % rid, vel, avel)
        assert st.finished == 4 and st.failed == 0
        assert st.max_live_seen >= 2            # the work really overlapped
        assert st.relayouts >= 4
        # every scene stepped exactly its own number of steps
        assert st.particle_steps == sum(srv.poll(r).n_particles * n for r, (_, n) in zip(ids, scenes))
        assert st.timed_steps == st.batch_steps
        assert 0 < st.step_ms_p50 <= st.step_ms_p99 <= st.step_ms_max
        assert st.hbm_peak_bytes <= st.hbm_budget_bytes


@pytest.mark.gpu
def test_admission_respects_budget():
    """With room for one scene at a time the server runs them one after the other."""
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1)
    scenes = [(dambreak(16, seed=1), 4), (dambreak(16, seed=5), 3), (dambreak(12, seed=6), 5)]
    one = max(state_bytes([d], prm) for d, _ in scenes)
    with Server(prm, hbm_budget_bytes=int(one * 1.3), max_live=8) as srv:
        ids = [srv.submit(d, n) for d, n in scenes]
        srv.drain()
        st = srv.stats()
        assert st.finished == 3 and st.max_live_seen == 1
        assert st.hbm_peak_bytes <= one
        for rid, (d, n) in zip(ids, scenes):
            pos, vel = srv.fetch(rid)
            apos, avel = _alone(d, prm, n)
            assert_bits("request %d pos" % rid, pos, apos)
            assert_bits("request %d vel" % rid, vel, avel)


@pytest.mark.gpu
def test_oversize_request_fails_others_served():
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1)
    small = dambreak(12, seed=1)
    with Server(prm, hbm_budget_bytes=int(state_bytes([small], prm) * 1.2)) as srv:
        big = srv.submit(dambreak(48, seed=2), 2)
        ok = srv.submit(small, 3)
        srv.drain()
        assert srv.poll(big).state == A.REQ_FAILED and srv.poll(big).status == A.ARIEL_ERR_OOM
        with pytest.raises(Exception):
            srv.wait(big)
        assert srv.poll(ok).state == A.REQ_DONE
        srv.release(ok)


@pytest.mark.gpu
def test_state_bytes_matches_allocation():
    """The admission estimate equals what a handle allocates (the server's own accounting)."""
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1)
    scenes = [dambreak(16, seed=1), dambreak(20, seed=3, spheres=[((0.6, 0.3, 0.5), 0.15)])]
    est = state_bytes(scenes, prm)
    with Server(prm) as srv:
        ids = [srv.submit(d, 30) for d in scenes]   # long enough to be live together
        srv.drain()
        peak = srv.stats().hbm_peak_bytes
    # the estimate rounds each buffer up to 256 bytes; the server sums the unrounded sizes
    assert peak <= est <= peak + 256 * 80


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-GPU behaviour")
def test_server_without_device_and_footprint_on_host():
    import ctypes as C
    from ariel_b200 import _lib
    L = _lib.lib()
    cfg = A.AsimServerConfig()
    L.ariel_server_config_default(C.byref(cfg))
    p = A.params_default()
    h = C.c_void_p()
    assert L.ariel_server_create(C.byref(p), C.byref(cfg), C.byref(h)) == A.ARIEL_ERR_NO_DEVICE
    mixed = params(precision=A.PREC_MIXED)
    fp64 = params(precision=A.PREC_FP64)
    b16, b32 = state_bytes([dambreak(16)], mixed), state_bytes([dambreak(32)], mixed)
    assert 0 < b16 < b32
    assert state_bytes([dambreak(32)], fp64) > b32
    both = state_bytes([dambreak(16), dambreak(32)], mixed)
    assert abs(both - (b16 + b32)) <= 64 * 256  # per-handle buffers counted once
    # reseeding adds its per-cell counts and their scans, each rounded to 256 bytes
    nc = 16 ** 3
    r256 = lambda b: (b + 255) // 256 * 256
    reseed = state_bytes([dambreak(16)], params(precision=A.PREC_MIXED, reseed_every=2))
    assert reseed - b16 == 2 * r256(4 * nc) + 2 * r256(4 * (nc + 1))
