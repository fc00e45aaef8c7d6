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


FACE_GRIDS = (A.GRID_UX, A.GRID_UY, A.GRID_UZ)
PREV_GRIDS = (A.GRID_PREV_UX, A.GRID_PREV_UY, A.GRID_PREV_UZ)


def _particles(tag, g, o, fields=("pos", "vel", "mass", "type")):
    gp, op = g.get_particles(), o.get_particles()
    for f in fields:
        assert_bits("%s %s" % (tag, f), gp[f], op[f])


def stage_parity(name, gpu, ora):
    """Runs the 12 FlipSim stages on both sides from identical state and compares every stage's
    output bit for bit; after the solve (which differs only in summation order) the oracle's
    pressure is copied into the GPU state."""
    for stage in range(A.STAGE_COUNT):
        ora.stage(stage)
        gpu.stage(stage)
        tag = "%s/%s" % (name, A.STAGE_NAMES[stage])
        if stage in (A.STAGE_BEGIN, A.STAGE_FORCES, A.STAGE_G2P_ADVECT, A.STAGE_RESAMPLE):
            _particles(tag, gpu, ora)
        elif stage == A.STAGE_SORT:
            gc, gn = gpu.get_cells()
            oc, on = ora.get_cells()
            assert_bits(tag + " particle->cell", gc, oc)
            assert_bits(tag + " per-cell counts", gn, on)
        elif stage == A.STAGE_DENSITY:
            assert_bits(tag + " density", gpu.get_particles()["density"], ora.get_particles()["density"])
        elif stage == A.STAGE_P2G:
            for w in FACE_GRIDS:
                assert_bits("%s face %d" % (tag, w), gpu.get_grid(w), ora.get_grid(w))
        elif stage == A.STAGE_CLASSIFY:
            assert_bits(tag + " flags", gpu.get_grid(A.GRID_A), ora.get_grid(A.GRID_A))
            assert_bits(tag + " L", gpu.get_grid(A.GRID_L), ora.get_grid(A.GRID_L))
        elif stage == A.STAGE_BOUNDARY_DIV:
            for w in FACE_GRIDS + PREV_GRIDS:
                assert_bits("%s grid %d" % (tag, w), gpu.get_grid(w), ora.get_grid(w))
            assert_bits(tag + " D", gpu.get_grid(A.GRID_D), ora.get_grid(A.GRID_D))
        elif stage == A.STAGE_SOLVE:
            Pg, Po = gpu.get_grid(A.GRID_P), ora.get_grid(A.GRID_P)
            flags = ora.get_grid(A.GRID_A)
            fl = flags == A.FLUID
            assert (Pg[~fl] == 0).all() and (Po[~fl] == 0).all()
            sg, so = gpu.stats(), ora.stats()
            assert sg.pcg_converged and so.pcg_converged
            if fl.any():
                scale = np.abs(Po[fl]).max() + 1e-30
                assert_close(tag + " P", Pg[fl] / scale, Po[fl] / scale, rtol=0, atol=1e-3)
            # identical inputs for the following stages
            gpu.set_grid(A.GRID_P, Po)
        elif stage in (A.STAGE_GRADIENT, A.STAGE_EXTRAPOLATE):
            for w in FACE_GRIDS + PREV_GRIDS:
                assert_bits("%s grid %d" % (tag, w), gpu.get_grid(w), ora.get_grid(w))


def icosphere(subdiv=2):
    """A closed triangle mesh of the unit sphere: an icosahedron subdivided `subdiv` times, its
    vertices pushed onto the sphere.  Returns (vertices (V,3) float32, triangles (T,3) int32)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache, nf = {}, []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts, np.float32), np.array(faces, np.int32)


def box_mesh():
    """A closed triangle mesh of the cube [-1, 1]^3 (12 triangles)."""
    v = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float32)
    idx = lambda x, y, z: x * 4 + y * 2 + z
    quads = [(idx(0, 0, 0), idx(0, 1, 0), idx(0, 1, 1), idx(0, 0, 1)), (idx(1, 0, 0), idx(1, 0, 1), idx(1, 1, 1), idx(1, 1, 0)),
             (idx(0, 0, 0), idx(0, 0, 1), idx(1, 0, 1), idx(1, 0, 0)), (idx(0, 1, 0), idx(1, 1, 0), idx(1, 1, 1), idx(0, 1, 1)),
             (idx(0, 0, 0), idx(1, 0, 0), idx(1, 1, 0), idx(0, 1, 0)), (idx(0, 0, 1), idx(0, 1, 1), idx(1, 1, 1), idx(1, 0, 1))]
    tris = []
    for a, b, c, d in quads:
        tris += [(a, b, c), (a, c, d)]
    return v, np.array(tris, np.int32)
