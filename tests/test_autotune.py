"""Autotuner: its candidate list respects the library's limits, and a tuned setting computes
the same pressure as the default one (tuning changes speed only)."""
import ctypes as C
import os

import numpy as np
import pytest

from ariel_b200 import _abi as A
from ariel_b200 import _lib, autotune

from helpers import dambreak, params


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="uses the no-GPU status to see the argument check")
def test_brick_limits_agree_with_library():
    L = _lib.lib()
    d = A.scene_dambreak(16)
    shapes = list(autotune.BRICKS) + [(31, 8, 8), (8, 8, 33), (32, 2, 2), (2, 2, 64), (16, 16, 9), (13, 13, 13)]
    for b in shapes:
        p = A.params_default()
        p.sweep_brick[:] = b
        h = C.c_void_p()
        st = L.ariel_create(C.byref(d), C.byref(p), C.byref(h))
        assert (st == A.ARIEL_ERR_NO_DEVICE) == autotune.brick_ok(b), (b, st)
    for bps, b in autotune.candidates(params(precond=A.PRECOND_MIC0)):
        assert autotune.brick_ok(b) and bps in (1, 2)


@pytest.mark.gpu
def test_tuned_setting_is_timed_and_equivalent(tmp_path, monkeypatch):
    monkeypatch.setenv("ARIEL_TUNE_CACHE", str(tmp_path / "tune.json"))
    from ariel_b200.flipsim import Batch
    desc = dambreak(24, seed=3)
    prm = params(precision=A.PREC_MIXED, precond=A.PRECOND_MIC0, stop=A.STOP_REL, tol=1e-6, graph=1)
    tuned, rep = autotune.tune([desc], prm, steps=1, warmup=1)
    assert not rep["cached"] and len(rep["timings"]) == len(autotune.candidates(prm))
    assert all(t["solve_ms"] > 0 for t in rep["timings"])
    assert (tuned.pcg_blocks_per_sm, tuple(tuned.sweep_brick)) in autotune.candidates(prm)
    _, rep2 = autotune.tune([desc], prm)
    assert rep2["cached"] and rep2["chosen"] == rep["chosen"]
    out = []
    for p in (prm, tuned):
        b = Batch([desc], p)
        b.init()
        b.step(3)
        out.append(b.get_grid(A.GRID_P64))
        b.close()
    assert np.array_equal(out[0].view(np.uint8), out[1].view(np.uint8))
