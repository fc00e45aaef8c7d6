"""TEST INFRASTRUCTURE ONLY: ctypes loader of betajippity/Ariel's own FLIP step, compiled from the
reference's sources into oracle/_ref/ by `make -C oracle reference` (see oracle/ref_driver.cpp).

It exists to pin the oracle (oracle/ariel_oracle.cpp) to the reference's arithmetic.  The sources
are read where they lie under the reference checkout, so the library can be built only where that
checkout exists; `available()` says whether it is built or buildable.  Imported by tests only.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from ariel_b200 import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.environ.get("ARIEL_REFERENCE_DIR", "/root/reference")
_SO = {
    "default": os.path.join(_HERE, "_ref", "libariel_reference.so"),
    "glm096": os.path.join(_HERE, "_ref", "libariel_reference_glm096.so"),
    # TBB's parallel_for spread over OpenMP threads: the benchmark's CPU reference arm (timed only)
    "omp": os.path.join(_HERE, "_ref", "libariel_reference_omp.so"),
    # the reference's mesh sources (oracle/ref_mesh_driver.cpp): its ray-triangle test
    "mesh": os.path.join(_HERE, "_ref", "libariel_reference_mesh.so"),
}
_libs = {}

# Stage cuts of oracle/ref_driver.cpp's ariel_pin_stage (0-11 as include/ariel.h's ARIEL_STAGE_*
# where the reference allows the same cut; 6 = StorePreviousGrid + EnforceBoundaryVelocity only;
# 7 = Solve including FlipGrid; 12 = stages 6-8 as the reference's Project runs them).
STAGE_BOUNDARY = 6
STAGE_SOLVE_WITH_FLIP = 7
STAGE_PROJECT = 12


def sources_present():
    return os.path.isfile(os.path.join(REF_DIR, "src", "sim", "flip.cpp"))


def build():
    out = subprocess.run(["make", "-C", _HERE, "reference", "REF=" + REF_DIR], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("reference build failed:\n" + out.stdout + out.stderr)


def available(variant="default"):
    if os.path.exists(_SO[variant]) and not sources_present():
        return True
    if not sources_present():
        return False
    build()
    return os.path.exists(_SO[variant])


def lib(variant="default"):
    if variant not in _libs:
        if not available(variant):
            raise RuntimeError("the reference's sources are not here and oracle/_ref is not built")
        L = C.CDLL(_SO[variant])
        vp = C.c_void_p
        L.ariel_pin_create.restype = vp
        L.ariel_pin_create.argtypes = [C.c_int32, C.c_float, C.c_float, vp, C.c_int32, vp, C.c_int32, C.c_uint64]
        L.ariel_pin_destroy.argtypes = [vp]
        L.ariel_pin_destroy.restype = None
        L.ariel_pin_set_scene_particles.argtypes = [vp, C.c_int64, vp, vp, vp, vp]
        L.ariel_pin_init.argtypes = [vp]
        L.ariel_pin_step.argtypes = [vp, C.c_int32]
        L.ariel_pin_stage.argtypes = [vp, C.c_int32]
        L.ariel_pin_particle_count.argtypes = [vp]
        L.ariel_pin_particle_count.restype = C.c_int64
        L.ariel_pin_get_particles.argtypes = [vp, vp, vp, vp, vp, vp]
        L.ariel_pin_set_particles.argtypes = [vp, C.c_int64, vp, vp, vp, vp]
        L.ariel_pin_get_cells.argtypes = [vp, vp, vp]
        L.ariel_pin_get_grid.argtypes = [vp, C.c_int32, vp]
        L.ariel_pin_set_grid.argtypes = [vp, C.c_int32, vp]
        L.ariel_pin_max_density.argtypes = [vp]
        L.ariel_pin_max_density.restype = C.c_float
        L.ariel_pin_frame.argtypes = [vp]
        L.ariel_pin_threads.restype = C.c_int32
        L.ariel_pin_philox4x32_10.argtypes = [vp, vp, vp]
        L.ariel_pin_philox4x32_10.restype = None
        _libs[variant] = L
    return _libs[variant]


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _ok(code, what):
    if code != 0:
        raise RuntimeError("%s failed" % what)


class ReferenceSim:
    """The reference's FlipSim driven through oracle/ref_driver.cpp.

    Fixed by the reference: PIC/FLIP 0.95, subcell 1, its own preconditioner, fp32 PCG with the
    absolute stop rule r.r <= 1e-2 n^3, resampling every step (src/sim/flip.cpp:15-30, 121;
    src/sim/solver.inl:289-354).
    """

    def __init__(self, desc, rng_seed, variant="default"):
        self.L = lib(variant)
        self.n = desc.dim
        forces = np.array([desc.forces[i][d] for i in range(desc.n_forces) for d in range(3)], np.float32)
        spheres = np.array([[desc.solid[i].center[0], desc.solid[i].center[1], desc.solid[i].center[2],
                             desc.solid[i].radius] for i in range(desc.n_solid)], np.float32).ravel()
        self.h = self.L.ariel_pin_create(desc.dim, desc.density, desc.stepsize, _p(forces), desc.n_forces,
                                         _p(spheres) if spheres.size else None, desc.n_solid, rng_seed)
        if not self.h:
            raise RuntimeError("ariel_pin_create refused the scene")

    def close(self):
        if self.h:
            self.L.ariel_pin_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_with(self, st):
        """FlipSim::Init, with Scene::GenerateParticles handing over the particles of `st`."""
        pos, vel, mass, typ = _arrays(st)
        _ok(self.L.ariel_pin_set_scene_particles(self.h, len(mass), _p(pos), _p(vel), _p(mass), _p(typ)),
            "set_scene_particles")
        _ok(self.L.ariel_pin_init(self.h), "init")

    def step(self, n=1):
        _ok(self.L.ariel_pin_step(self.h, n), "step")

    def stage(self, s):
        _ok(self.L.ariel_pin_stage(self.h, s), "stage %d" % s)

    def frame(self):
        return self.L.ariel_pin_frame(self.h)

    def count(self):
        return self.L.ariel_pin_particle_count(self.h)

    def max_density(self):
        return self.L.ariel_pin_max_density(self.h)

    def get_particles(self):
        n = self.count()
        pos = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        den = np.zeros(n, np.float32)
        mass = np.zeros(n, np.float32)
        typ = np.zeros(n, np.int32)
        _ok(self.L.ariel_pin_get_particles(self.h, _p(pos), _p(vel), _p(den), _p(mass), _p(typ)), "get_particles")
        return dict(pos=pos, vel=vel, density=den, mass=mass, type=typ)

    def set_particles(self, pos, vel, mass, typ):
        pos, vel, mass, typ = _arrays(dict(pos=pos, vel=vel, mass=mass, type=typ))
        _ok(self.L.ariel_pin_set_particles(self.h, len(mass), _p(pos), _p(vel), _p(mass), _p(typ)), "set_particles")

    def get_cells(self):
        pc = np.zeros(self.count(), np.int32)
        cc = np.zeros(self.n ** 3, np.int32)
        _ok(self.L.ariel_pin_get_cells(self.h, _p(pc), _p(cc)), "get_cells")
        return pc, cc

    def get_grid(self, which):
        from oracle.pyoracle import grid_shape
        shape, dt = grid_shape(self.n, which)
        a = np.zeros(shape, dt)
        _ok(self.L.ariel_pin_get_grid(self.h, which, _p(a)), "get_grid")
        return a

    def set_grid(self, which, a):
        from oracle.pyoracle import grid_shape
        shape, dt = grid_shape(self.n, which)
        a = np.ascontiguousarray(a, dt).reshape(shape)
        _ok(self.L.ariel_pin_set_grid(self.h, which, _p(a)), "set_grid")


def _arrays(st):
    return (np.ascontiguousarray(st["pos"], np.float32), np.ascontiguousarray(st["vel"], np.float32),
            np.ascontiguousarray(st["mass"], np.float32), np.ascontiguousarray(st["type"], np.int32))


def threads(variant="default"):
    return lib(variant).ariel_pin_threads()


def philox(counter, key, variant="default"):
    c = np.ascontiguousarray(counter, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib(variant).ariel_pin_philox4x32_10(_p(c), _p(k), _p(o))
    return o


def ray_triangle(v, o, d):
    """Obj::RayTriangleTest (src/geom/obj/obj.cpp:354-398) of the reference's own build:
    (hit, hit point) for the triangle v (3x3) and the ray (o, d)."""
    if "mesh" not in _libs:
        if not available("mesh"):
            raise RuntimeError("the reference's sources are not here and oracle/_ref is not built")
        L = C.CDLL(_SO["mesh"])
        L.ariel_pin_ray_triangle.argtypes = [C.c_void_p] * 4
        L.ariel_pin_ray_triangle.restype = C.c_int32
        _libs["mesh"] = L
    v = np.ascontiguousarray(v, np.float32).ravel()
    o = np.ascontiguousarray(o, np.float32)
    d = np.ascontiguousarray(d, np.float32)
    pt = np.zeros(3, np.float32)
    hit = _libs["mesh"].ariel_pin_ray_triangle(_p(v), _p(o), _p(d), _p(pt))
    return bool(hit), pt


def reference_params():
    """Oracle parameters equal to what the reference's FlipSim hard-codes."""
    p = A.params_default()
    p.precision = A.PREC_REF32
    p.precond = A.PRECOND_REF
    p.stop_rule = A.STOP_REF_ABS
    p.resample_every = 1
    p.picflip = 0.95
    p.subcell = 1
    return p
