"""TEST INFRASTRUCTURE ONLY: ctypes loader of the CPU oracle (oracle/ariel_oracle.cpp).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg -- never by the
product package.  Pinned to the reference's own code (see ariel_oracle.h).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from ariel_b200 import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libariel_oracle.so")
_lib = None


def build(quiet=True):
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        vp = C.c_void_p
        L.ariel_ref_create.argtypes = [C.POINTER(A.AsimSceneDesc), C.POINTER(A.AsimParams), C.POINTER(vp)]
        L.ariel_ref_destroy.argtypes = [vp]
        L.ariel_ref_destroy.restype = None
        L.ariel_ref_add_mesh.argtypes = [vp, vp, C.c_int32, vp, C.c_int32, vp, C.c_float]
        L.ariel_ref_tri_ray.argtypes = [vp, vp, vp, vp]
        L.ariel_ref_tri_ray.restype = C.c_int32
        L.ariel_ref_set_faithful.argtypes = [vp, C.c_int32]
        L.ariel_ref_set_faithful.restype = None
        L.ariel_ref_set_threads.argtypes = [C.c_int32]
        L.ariel_ref_set_threads.restype = None
        L.ariel_ref_max_threads.restype = C.c_int32
        for name in ("ariel_ref_init",):
            getattr(L, name).argtypes = [vp]
        L.ariel_ref_step.argtypes = [vp, C.c_int32]
        L.ariel_ref_stage.argtypes = [vp, C.c_int32]
        L.ariel_ref_particle_count.argtypes = [vp, C.POINTER(C.c_int64)]
        L.ariel_ref_get_particles.argtypes = [vp, vp, vp, vp, vp, vp]
        L.ariel_ref_set_particles.argtypes = [vp, C.c_int64, vp, vp, vp, vp]
        L.ariel_ref_get_cells.argtypes = [vp, vp, vp]
        L.ariel_ref_get_grid.argtypes = [vp, C.c_int32, vp, C.c_int64]
        L.ariel_ref_set_grid.argtypes = [vp, C.c_int32, vp, C.c_int64]
        L.ariel_ref_stats.argtypes = [vp, C.POINTER(A.AsimStats)]
        L.ariel_ref_get_max_density.argtypes = [vp, C.POINTER(C.c_float)]
        L.ariel_ref_stage_ms.argtypes = [vp, vp]
        L.ariel_ref_solve_fp64.argtypes = [C.c_int32, vp, vp, vp, vp, C.c_double, C.c_int32,
                                           C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.ariel_ref_apply_fp64.argtypes = [C.c_int32, vp, vp, vp, vp]
        L.ariel_ref_level_set.argtypes = [vp, vp, C.c_int64]
        L.ariel_ref_surface_mesh.argtypes = [vp, vp, C.c_int64, vp, C.c_int64, C.POINTER(C.c_int64),
                                             C.POINTER(C.c_int64)]
        L.ariel_ref_philox4x32_10.argtypes = [vp, vp, vp]
        L.ariel_ref_philox4x32_10.restype = None
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _check(code, what):
    if code != A.ARIEL_OK:
        raise RuntimeError("%s -> %s" % (what, A.status_name(code)))


def grid_shape(n, which):
    if which in (A.GRID_UX, A.GRID_PREV_UX):
        return (n + 1, n, n), np.float32
    if which in (A.GRID_UY, A.GRID_PREV_UY):
        return (n, n + 1, n), np.float32
    if which in (A.GRID_UZ, A.GRID_PREV_UZ):
        return (n, n, n + 1), np.float32
    if which == A.GRID_A:
        return (n, n, n), np.int32
    if which == A.GRID_P64:
        return (n, n, n), np.float64
    return (n, n, n), np.float32


class RefSim:
    """CPU oracle handle mirroring the product's FlipSim-like surface."""

    def __init__(self, desc, params, faithful=False):
        self.L = lib()
        h = C.c_void_p()
        _check(self.L.ariel_ref_create(C.byref(desc), C.byref(params), C.byref(h)), "ariel_ref_create")
        self.h = h
        self.n = desc.dim
        self.L.ariel_ref_set_faithful(self.h, 1 if faithful else 0)

    def close(self):
        if self.h:
            self.L.ariel_ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_mesh(self, vertices, triangles, translate=(0.0, 0.0, 0.0), scale=1.0):
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, np.int32).reshape(-1, 3)
        tr = np.ascontiguousarray(translate, np.float32).reshape(3)
        _check(self.L.ariel_ref_add_mesh(self.h, _p(v), len(v), _p(t), len(t), _p(tr), float(scale)), "add_mesh")

    def init(self):
        _check(self.L.ariel_ref_init(self.h), "ariel_ref_init")

    def step(self, n=1):
        _check(self.L.ariel_ref_step(self.h, n), "ariel_ref_step")

    def stage(self, s):
        _check(self.L.ariel_ref_stage(self.h, s), "ariel_ref_stage")

    def count(self):
        n = C.c_int64()
        _check(self.L.ariel_ref_particle_count(self.h, C.byref(n)), "count")
        return n.value

    def get_particles(self):
        n = self.count()
        pos = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        den = np.zeros(n, np.float32)
        mass = np.zeros(n, np.float32)
        typ = np.zeros(n, np.int32)
        _check(self.L.ariel_ref_get_particles(self.h, _p(pos), _p(vel), _p(den), _p(mass), _p(typ)), "get_particles")
        return dict(pos=pos, vel=vel, density=den, mass=mass, type=typ)

    def set_particles(self, pos, vel, mass, typ):
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        mass = np.ascontiguousarray(mass, np.float32)
        typ = np.ascontiguousarray(typ, np.int32)
        _check(self.L.ariel_ref_set_particles(self.h, len(mass), _p(pos), _p(vel), _p(mass), _p(typ)), "set_particles")

    def get_cells(self):
        n = self.count()
        pc = np.zeros(n, np.int32)
        cc = np.zeros(self.n ** 3, np.int32)
        _check(self.L.ariel_ref_get_cells(self.h, _p(pc), _p(cc)), "get_cells")
        return pc, cc

    def get_grid(self, which):
        shape, dt = grid_shape(self.n, which)
        a = np.zeros(shape, dt)
        _check(self.L.ariel_ref_get_grid(self.h, which, _p(a), a.nbytes), "get_grid")
        return a

    def set_grid(self, which, a):
        shape, dt = grid_shape(self.n, which)
        a = np.ascontiguousarray(a, dt).reshape(shape)
        _check(self.L.ariel_ref_set_grid(self.h, which, _p(a), a.nbytes), "set_grid")

    def stats(self):
        st = A.AsimStats()
        _check(self.L.ariel_ref_stats(self.h, C.byref(st)), "stats")
        return st

    def max_density(self):
        v = C.c_float()
        _check(self.L.ariel_ref_get_max_density(self.h, C.byref(v)), "max_density")
        return v.value

    def level_set(self):
        N = self.n + 5
        phi = np.zeros((N, N, N), np.float32)
        _check(self.L.ariel_ref_level_set(self.h, _p(phi), phi.nbytes), "level_set")
        return phi

    def surface_mesh(self):
        nv, nq = C.c_int64(), C.c_int64()
        _check(self.L.ariel_ref_surface_mesh(self.h, None, 0, None, 0, C.byref(nv), C.byref(nq)), "surface_mesh")
        v = np.zeros((nv.value, 3), np.float32)
        q = np.zeros((nq.value, 4), np.int32)
        _check(self.L.ariel_ref_surface_mesh(self.h, _p(v), nv.value, _p(q), nq.value, C.byref(nv), C.byref(nq)),
               "surface_mesh")
        return v, q

    def stage_ms(self):
        a = np.zeros(A.STAGE_COUNT, np.float64)
        _check(self.L.ariel_ref_stage_ms(self.h, _p(a)), "stage_ms")
        return a


def solve_fp64(n, flags, L, b, x0=None, tol=1e-12, max_iters=0):
    """Tight FP64 PCG on the reference operator; returns (x, iterations, rel_residual)."""
    flags = np.ascontiguousarray(flags, np.int32)
    L = np.ascontiguousarray(L, np.float32)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(n ** 3, np.float64) if x0 is None else np.array(x0, np.float64).ravel().copy()
    it = C.c_int32()
    rel = C.c_double()
    lib().ariel_ref_solve_fp64(n, _p(flags), _p(L), _p(b), _p(x), tol, max_iters, C.byref(it), C.byref(rel))
    return x.reshape(n, n, n), it.value, rel.value


def apply_fp64(n, flags, L, x):
    flags = np.ascontiguousarray(flags, np.int32)
    L = np.ascontiguousarray(L, np.float32)
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(n ** 3, np.float64)
    _check(lib().ariel_ref_apply_fp64(n, _p(flags), _p(L), _p(x), _p(y)), "apply_fp64")
    return y.reshape(n, n, n)


def tri_ray(v, o, d):
    """The mesh queries' ray-triangle test: (hit, hit point o + d t) for the triangle v (3x3)."""
    import numpy as np
    v = np.ascontiguousarray(v, np.float32).ravel()
    o = np.ascontiguousarray(o, np.float32)
    d = np.ascontiguousarray(d, np.float32)
    pt = np.zeros(3, np.float32)
    hit = lib().ariel_ref_tri_ray(_p(v), _p(o), _p(d), _p(pt))
    return bool(hit), pt


def philox(counter, key):
    c = np.ascontiguousarray(counter, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().ariel_ref_philox4x32_10(_p(c), _p(k), _p(o))
    return o
