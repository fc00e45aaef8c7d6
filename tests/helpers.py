"""Shared helpers for the parity tests (GPU library vs CPU oracle on identical inputs)."""
import numpy as np

from ariel_b200 import _abi as A


def dambreak(n, seed=1, spheres=(), hi=(0.4, 0.6, 1.0), jitter=1.0):
    return A.scene_dambreak(n, liquid_hi=hi, seed=seed, jitter=jitter, spheres=spheres)


def params(precision=A.PREC_REF32, precond=A.PRECOND_REF, stop=A.STOP_REF_ABS, tol=1e-5, graph=0, **kw):
    p = A.params_default()
    p.precision = precision
    p.precond = precond
    p.stop_rule = stop
    p.tol = tol
    p.use_graph = graph
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def evolved_state(desc, prm, steps):
    """Particles (and pressure) after `steps` oracle steps from the scene's Init state."""
    from oracle.pyoracle import RefSim
    r = RefSim(desc, prm)
    r.init()
    if steps:
        r.step(steps)
    st = r.get_particles()
    P = r.get_grid(A.GRID_P)
    P64 = r.get_grid(A.GRID_P64)
    return st, P, P64


def assert_bits(name, got, want):
    """Bit-exact comparison (NaN-aware) with a short diagnostic."""
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, "%s: shape %s vs %s" % (name, got.shape, want.shape)
    if got.dtype.kind == "f":
        same = (got == want) | (np.isnan(got) & np.isnan(want))
    else:
        same = got == want
    if not same.all():
        bad = np.argwhere(~same)
        i = tuple(bad[0])
        diff = np.abs(got.astype(np.float64) - want.astype(np.float64))
        raise AssertionError("%s: %d of %d entries differ; first at %s: got %r want %r; max |diff| %.3e"
                             % (name, (~same).sum(), same.size, i, got[i], want[i], np.nanmax(diff)))


def assert_close(name, got, want, rtol, atol=0.0):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    err = np.abs(got - want)
    lim = atol + rtol * np.abs(want)
    if not (err <= lim).all():
        i = np.unravel_index(np.argmax(err - lim), err.shape)
        raise AssertionError("%s: max |diff| %.3e at %s (got %r want %r, rtol %g atol %g)"
                             % (name, err.max(), i, got[i], want[i], rtol, atol))
