"""Python mirror of the reference's `fluidCore::FlipSim` (src/sim/flip.hpp:20-66) over the C ABI.

    sim = FlipSim(maxres=64, density=0.5, stepsize=1/240, scene=dambreak(64), verbose=False)
    sim.Init(); sim.Step(False, False, False); particles = sim.GetParticles()

Construction, Init and Step follow the reference's names and meaning; the state lives on the
B200 and GetParticles copies it to host numpy arrays.  `Batch` steps several scenes together.
"""
import ctypes as C

import numpy as np

from . import _abi as A
from ._lib import ArielError, check, lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


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


class Batch:
    """k scenes stepped together (one launch per stage over a packed index space)."""

    def __init__(self, descs, params=None):
        self.L = lib()
        if params is None:
            params = A.params_default()
        self.params = params
        arr = (A.AsimSceneDesc * len(descs))(*descs)
        h = C.c_void_p()
        if len(descs) == 1:
            check(self.L.ariel_create(C.byref(arr[0]), C.byref(params), C.byref(h)), "ariel_create")
        else:
            check(self.L.ariel_create_batch(arr, len(descs), C.byref(params), C.byref(h)), "ariel_create_batch")
        self.h = h
        self.descs = list(descs)
        self.k = len(descs)

    def close(self):
        if getattr(self, "h", None):
            self.L.ariel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- lifecycle ---------------------------------------------------------------------
    def init(self):
        check(self.L.ariel_init(self.h), "ariel_init")

    def step(self, n=1):
        check(self.L.ariel_step(self.h, n), "ariel_step")

    def stage(self, s):
        check(self.L.ariel_stage(self.h, s), "ariel_stage")

    def synchronize(self):
        check(self.L.ariel_synchronize(self.h), "ariel_synchronize")

    # -- accessors ---------------------------------------------------------------------
    def dim(self, scene=0):
        return self.descs[scene].dim

    def count(self, scene=0):
        n = C.c_int64()
        check(self.L.ariel_particle_count(self.h, scene, C.byref(n)), "ariel_particle_count")
        return n.value

    def get_particles(self, scene=0):
        n = self.count(scene)
        pos = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        den = np.zeros(n, np.float32)
        mass = np.zeros(n, np.float32)
        typ = np.zeros(n, np.int32)
        check(self.L.ariel_get_particles(self.h, scene, _p(pos), _p(vel), _p(den), _p(mass), _p(typ)),
              "ariel_get_particles")
        return dict(pos=pos, vel=vel, density=den, mass=mass, type=typ)

    def get_positions_velocities(self, pos, vel, scene=0):
        check(self.L.ariel_get_particles(self.h, scene, _p(pos), _p(vel), None, None, None), "ariel_get_particles")

    def set_particles(self, pos, vel, mass, typ, scene=0):
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        mass = np.ascontiguousarray(mass, np.float32)
        typ = np.ascontiguousarray(typ, np.int32)
        check(self.L.ariel_set_particles(self.h, scene, len(mass), _p(pos), _p(vel), _p(mass), _p(typ)),
              "ariel_set_particles")

    def get_cells(self, scene=0):
        n = self.count(scene)
        d = self.dim(scene)
        pc = np.zeros(n, np.int32)
        cc = np.zeros(d ** 3, np.int32)
        check(self.L.ariel_get_cells(self.h, scene, _p(pc), _p(cc)), "ariel_get_cells")
        return pc, cc

    def get_grid(self, which, scene=0):
        shape, dt = grid_shape(self.dim(scene), which)
        a = np.zeros(shape, dt)
        check(self.L.ariel_get_grid(self.h, scene, which, _p(a), a.nbytes), "ariel_get_grid")
        return a

    def set_grid(self, which, a, scene=0):
        shape, dt = grid_shape(self.dim(scene), which)
        a = np.ascontiguousarray(a, dt).reshape(shape)
        check(self.L.ariel_set_grid(self.h, scene, which, _p(a), a.nbytes), "ariel_set_grid")

    def stats(self, scene=0):
        st = A.AsimStats()
        check(self.L.ariel_stats(self.h, scene, C.byref(st)), "ariel_stats")
        return st

    def max_density(self, scene=0):
        v = C.c_float()
        check(self.L.ariel_get_max_density(self.h, scene, C.byref(v)), "ariel_get_max_density")
        return v.value

    def upload_state(self, pos, vel, scene=0):
        """Asynchronous H2D of xyz positions/velocities (keep the buffers alive until the
        next synchronising call)."""
        check(self.L.ariel_upload_state(self.h, scene, _p(pos), _p(vel)), "ariel_upload_state")

    def download_state(self, pos, vel, scene=0):
        check(self.L.ariel_download_state(self.h, scene, _p(pos), _p(vel)), "ariel_download_state")

    def timing_reset(self):
        check(self.L.ariel_timing_reset(self.h), "ariel_timing_reset")

    def timing(self, max_steps=4096):
        ms = np.zeros(A.STAGE_COUNT, np.float64)
        solve_k = C.c_double()
        steps = np.zeros(max_steps, np.float64)
        n = C.c_int32()
        check(self.L.ariel_timing_get(self.h, _p(ms), C.byref(solve_k), _p(steps), max_steps, C.byref(n)),
              "ariel_timing_get")
        return dict(stage_ms=ms, solve_kernel_ms=solve_k.value, steps=n.value,
                    step_ms=steps[:min(n.value, max_steps)].copy())

    def level_set(self, scene=0):
        """The liquid surface's level set ((n+5)^3 samples, sample (i,j,k) at grid point
        (i-2, j-2, k-2))."""
        N = self.dim(scene) + 5
        phi = np.zeros((N, N, N), np.float32)
        check(self.L.ariel_get_level_set(self.h, scene, _p(phi), phi.nbytes), "ariel_get_level_set")
        return phi

    def surface_mesh(self, scene=0):
        """(vertices (V,3) in grid units, quads (Q,4) 0-based) of the liquid surface."""
        nv, nq = C.c_int64(), C.c_int64()
        check(self.L.ariel_surface_mesh(self.h, scene, None, 0, None, 0, C.byref(nv), C.byref(nq)),
              "ariel_surface_mesh")
        v = np.zeros((nv.value, 3), np.float32)
        q = np.zeros((nq.value, 4), np.int32)
        check(self.L.ariel_surface_mesh(self.h, scene, _p(v), nv.value, _p(q), nq.value, C.byref(nv), C.byref(nq)),
              "ariel_surface_mesh")
        return v, q

    def export_surface(self, path, frame, scene=0):
        check(self.L.ariel_export_surface(self.h, scene, str(path).encode(), frame), "ariel_export_surface")

    def checkpoint_save(self, path):
        check(self.L.ariel_checkpoint_save(self.h, str(path).encode()), "ariel_checkpoint_save")

    def checkpoint_load(self, path):
        check(self.L.ariel_checkpoint_load(self.h, str(path).encode()), "ariel_checkpoint_load")

    def export_particles(self, path, frame, scene=0):
        """Scene::ExportParticles' particle file (Houdini ASCII .geo, or .geo.gz); returns the
        written path."""
        check(self.L.ariel_export_particles(self.h, scene, str(path).encode(), frame), "ariel_export_particles")
        p = str(path)
        gz = p.endswith(".gz")
        stem, ext = (p[:-3] if gz else p).rsplit(".", 1)
        return "%s.%04d.%s%s" % (stem, frame, ext, ".gz" if gz else "")

    def solver_totals(self, scene=0):
        t = A.AsimSolverTotals()
        check(self.L.ariel_solver_totals(self.h, scene, C.byref(t)), "ariel_solver_totals")
        return t

    def timer_begin(self):
        check(self.L.ariel_timer_begin(self.h), "ariel_timer_begin")

    def timer_end(self):
        ms = C.c_double()
        check(self.L.ariel_timer_end(self.h, C.byref(ms)), "ariel_timer_end")
        return ms.value


class FlipSim:
    """FlipSim(maxres, density, stepsize, scene, verbose) -- src/sim/flip.hpp:22-23.

    `scene` is an AsimSceneDesc (the synthetic stand-in for sceneCore::Scene); maxres, density
    and stepsize override its grid size, lattice density and time step like the reference's
    constructor arguments do.
    """

    def __init__(self, maxres, density, stepsize, scene, verbose=False, params=None):
        desc = A.AsimSceneDesc()
        C.pointer(desc)[0] = scene
        desc.dim = int(maxres)
        desc.density = float(density)
        desc.stepsize = float(stepsize)
        self._b = Batch([desc], params)
        self.m_frame = 0
        self.verbose = verbose

    def Init(self):
        """FlipSim::Init (src/sim/flip.cpp:42-77)."""
        self._b.init()
        self.m_frame = 0

    def Step(self, saveVDB=False, saveOBJ=False, savePARTIO=False):
        """FlipSim::Step (src/sim/flip.cpp:92-128).  The export flags are accepted for
        interface parity; particle export is GetParticles()."""
        self._b.step(1)
        self.m_frame += 1

    def GetParticles(self):
        """FlipSim::GetParticles (src/sim/flip.hpp:29): host copies of the particle state."""
        return self._b.get_particles(0)

    def GetDimensions(self):
        """FlipSim::GetDimensions (src/sim/flip.hpp:30)."""
        n = self._b.dim(0)
        return (n, n, n)

    def GetScene(self):
        return self._b.descs[0]

    @property
    def batch(self):
        return self._b


def state_bytes(descs, params=None):
    """Device bytes a handle or server batch holds for these scenes."""
    L = lib()
    if params is None:
        params = A.params_default()
    arr = (A.AsimSceneDesc * len(descs))(*descs)
    b = C.c_int64()
    check(L.ariel_state_bytes(arr, len(descs), C.byref(params), C.byref(b)), "ariel_state_bytes")
    return b.value


class Server:
    """Request server: scenes of any size arrive as (scene, steps) requests and are stepped
    together, re-packed at step boundaries as they arrive and finish (ariel_server_*)."""

    def __init__(self, params=None, hbm_budget_bytes=0, max_live=0, prepare_threads=0, keep_results=1,
                 reserve_budget=0):
        self.L = lib()
        if params is None:
            params = A.params_default()
        cfg = A.AsimServerConfig()
        self.L.ariel_server_config_default(C.byref(cfg))
        cfg.hbm_budget_bytes = hbm_budget_bytes
        if max_live:
            cfg.max_live = max_live
        if prepare_threads:
            cfg.prepare_threads = prepare_threads
        cfg.keep_results = keep_results
        cfg.reserve_budget = reserve_budget
        h = C.c_void_p()
        check(self.L.ariel_server_create(C.byref(params), C.byref(cfg), C.byref(h)), "ariel_server_create")
        self.h = h

    def submit(self, desc, nsteps):
        i = C.c_int64()
        check(self.L.ariel_server_submit(self.h, C.byref(desc), nsteps, C.byref(i)), "ariel_server_submit")
        return i.value

    def poll(self, rid):
        info = A.AsimRequestInfo()
        check(self.L.ariel_server_poll(self.h, rid, C.byref(info)), "ariel_server_poll")
        return info

    def wait(self, rid, timeout_ms=600000.0):
        check(self.L.ariel_server_wait(self.h, rid, timeout_ms), "ariel_server_wait")

    def drain(self, timeout_ms=600000.0):
        check(self.L.ariel_server_drain(self.h, timeout_ms), "ariel_server_drain")

    def fetch(self, rid):
        n = self.poll(rid).n_particles
        pos = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        check(self.L.ariel_server_fetch(self.h, rid, _p(pos), _p(vel)), "ariel_server_fetch")
        return pos, vel

    def release(self, rid):
        check(self.L.ariel_server_release(self.h, rid), "ariel_server_release")

    def stats(self):
        st = A.AsimServerStats()
        check(self.L.ariel_server_stats(self.h, C.byref(st)), "ariel_server_stats")
        return st

    def shutdown(self):
        if getattr(self, "h", None):
            check(self.L.ariel_server_shutdown(self.h), "ariel_server_shutdown")
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.shutdown()

    def __del__(self):
        try:
            self.shutdown()
        except Exception:
            pass


class Mesh:
    """A static solid mesh registered with the library (ariel_mesh_create): triangles in object
    space placed in the unit cube as object * scale + translate; reference it from a scene with
    `_abi.add_mesh(desc, mesh.id)`."""

    def __init__(self, vertices, triangles, translate=(0.0, 0.0, 0.0), scale=1.0):
        self.L = lib()
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, np.int32).reshape(-1, 3)
        tr = np.ascontiguousarray(translate, np.float32).reshape(3)
        mid = C.c_int32()
        check(self.L.ariel_mesh_create(_p(v), len(v), _p(t), len(t), _p(tr), float(scale), C.byref(mid)),
              "ariel_mesh_create")
        self.id = mid.value
        self.vertices, self.triangles, self.translate, self.scale = v, t, tr, float(scale)

    @classmethod
    def adopt(cls, mesh_id):
        """Takes ownership of a mesh the library registered itself (ariel_scene_load): its id,
        placement and counts; it is destroyed with this object."""
        m = cls.__new__(cls)
        m.L = lib()
        nv, nt, sc = C.c_int32(), C.c_int32(), C.c_float()
        tr = np.zeros(3, np.float32)
        check(m.L.ariel_mesh_info(mesh_id, C.byref(nv), C.byref(nt), _p(tr), C.byref(sc)), "ariel_mesh_info")
        m.id = mesh_id
        m.translate, m.scale = tr, float(sc.value)
        m.n_vertices, m.n_triangles = nv.value, nt.value
        m.vertices = m.triangles = None  # held by the library
        return m

    def close(self):
        if getattr(self, "id", None) is not None:
            self.L.ariel_mesh_destroy(self.id)
            self.id = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
