"""ctypes mirror of include/ariel.h (structs, enums, status codes).

The layouts here must match include/ariel.h field for field; tests/test_abi.py checks the
sizes and field offsets against the C compiler.s view of the header.
"""
import ctypes as C

ARIEL_OK = 0
ARIEL_ERR_INVALID_ARG = 1
ARIEL_ERR_OOM = 2
ARIEL_ERR_NOT_CONVERGED = 3
ARIEL_ERR_DEVICE_TIMEOUT = 4
ARIEL_ERR_CUDA = 5
ARIEL_ERR_STATE = 6
ARIEL_ERR_NO_DEVICE = 7
ARIEL_ERR_NAN = 8
ARIEL_ERR_PENDING = 9

STATUS_NAMES = {
    0: "ARIEL_OK", 1: "ARIEL_ERR_INVALID_ARG", 2: "ARIEL_ERR_OOM", 3: "ARIEL_ERR_NOT_CONVERGED",
    4: "ARIEL_ERR_DEVICE_TIMEOUT", 5: "ARIEL_ERR_CUDA", 6: "ARIEL_ERR_STATE",
    7: "ARIEL_ERR_NO_DEVICE", 8: "ARIEL_ERR_NAN", 9: "ARIEL_ERR_PENDING",
}

AIR, FLUID, SOLID = 0, 1, 2          # src/grid/macgrid.inl:13

PRECOND_REF, PRECOND_MIC0 = 0, 1
PREC_REF32, PREC_FP64, PREC_MIXED = 0, 1, 2
STOP_REF_ABS, STOP_REL = 0, 1

(STAGE_BEGIN, STAGE_SORT, STAGE_DENSITY, STAGE_FORCES, STAGE_P2G, STAGE_CLASSIFY,
 STAGE_BOUNDARY_DIV, STAGE_SOLVE, STAGE_GRADIENT, STAGE_EXTRAPOLATE, STAGE_G2P_ADVECT,
 STAGE_RESAMPLE) = range(12)
STAGE_COUNT = 12
STAGE_NAMES = ["begin", "sort", "density", "forces", "p2g", "classify", "boundary_div", "solve",
               "gradient", "extrapolate", "g2p_advect", "resample"]

(GRID_UX, GRID_UY, GRID_UZ, GRID_PREV_UX, GRID_PREV_UY, GRID_PREV_UZ, GRID_D, GRID_P, GRID_L,
 GRID_A, GRID_P64) = range(11)

MAX_BOXES = 8
MAX_SPHERES = 8
MAX_FORCES = 4
MAX_MESHES = 8


class AsimBox(C.Structure):
    _fields_ = [("lo", C.c_float * 3), ("hi", C.c_float * 3), ("vel", C.c_float * 3)]


class AsimSphere(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("radius", C.c_float)]


class AsimSceneDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("density", C.c_float), ("stepsize", C.c_float),
        ("n_forces", C.c_int32), ("forces", (C.c_float * 3) * MAX_FORCES),
        ("n_liquid", C.c_int32), ("liquid", AsimBox * MAX_BOXES),
        ("n_solid", C.c_int32), ("solid", AsimSphere * MAX_SPHERES),
        ("seed", C.c_uint64), ("jitter", C.c_float), ("reserved", C.c_int32),
        ("n_mesh", C.c_int32), ("mesh", C.c_int32 * MAX_MESHES),
    ]


class AsimSceneInfo(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("reserved", C.c_int32), ("density", C.c_double), ("step_size", C.c_double),
        ("partio_output", C.c_char * 512), ("vdb_output", C.c_char * 512), ("mesh_output", C.c_char * 512),
    ]


class AsimParams(C.Structure):
    _fields_ = [
        ("picflip", C.c_float), ("subcell", C.c_int32), ("precond", C.c_int32),
        ("precision", C.c_int32), ("stop_rule", C.c_int32), ("max_iters", C.c_int32),
        ("tol", C.c_double), ("inner_tol", C.c_double), ("max_outer", C.c_int32),
        ("resample_every", C.c_int32), ("mic_tau", C.c_double), ("mic_sigma", C.c_double),
        ("rng_seed", C.c_uint64), ("use_graph", C.c_int32), ("timing", C.c_int32),
        ("barrier_timeout_ms", C.c_double), ("fail_on_not_converged", C.c_int32),
        ("pcg_blocks_per_sm", C.c_int32), ("pcg_grid_blocks", C.c_int32), ("sweep_brick", C.c_int32 * 3),
        ("p2g_faces", C.c_int32), ("reseed_every", C.c_int32), ("reseed_min", C.c_int32),
        ("reseed_max", C.c_int32),
    ]


class AsimStats(C.Structure):
    _fields_ = [
        ("frame", C.c_int64), ("n_particles", C.c_int64), ("n_fluid_cells", C.c_int64),
        ("pcg_iterations", C.c_int32), ("pcg_outer", C.c_int32),
        ("pcg_rel_residual", C.c_double), ("pcg_rr", C.c_double),
        ("pcg_converged", C.c_int32), ("precond_exact_path", C.c_int32),
        ("stage_ms", C.c_double * STAGE_COUNT), ("step_ms", C.c_double),
        ("last_status", C.c_int32), ("reserved", C.c_int32),
    ]


class AsimSolverTotals(C.Structure):
    _fields_ = [
        ("solves", C.c_int64), ("iterations", C.c_int64), ("outer", C.c_int64),
        ("cell_iterations", C.c_double), ("cell_outer", C.c_double),
        ("not_converged", C.c_int64), ("reserved", C.c_int64),
    ]


REQ_QUEUED, REQ_READY, REQ_RUNNING, REQ_DONE, REQ_FAILED = range(5)


class AsimServerConfig(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_int64), ("max_live", C.c_int32), ("prepare_threads", C.c_int32),
        ("keep_results", C.c_int32), ("max_ready", C.c_int32), ("reserve_budget", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class AsimRequestInfo(C.Structure):
    _fields_ = [
        ("state", C.c_int32), ("status", C.c_int32), ("nsteps", C.c_int32), ("steps_done", C.c_int32),
        ("n_particles", C.c_int64), ("state_bytes", C.c_int64),
        ("submit_ms", C.c_double), ("admit_ms", C.c_double), ("done_ms", C.c_double),
        ("stats", AsimStats),
    ]


class AsimServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64), ("admitted", C.c_int64), ("finished", C.c_int64),
        ("failed", C.c_int64), ("live", C.c_int64), ("waiting", C.c_int64),
        ("batch_steps", C.c_int64), ("particle_steps", C.c_int64), ("timed_steps", C.c_int64),
        ("wall_ms", C.c_double), ("busy_ms", C.c_double),
        ("step_ms_p50", C.c_double), ("step_ms_p99", C.c_double), ("step_ms_max", C.c_double),
        ("latency_ms_p50", C.c_double), ("latency_ms_p99", C.c_double),
        ("relayouts", C.c_int64), ("relayout_ms", C.c_double),
        ("hbm_budget_bytes", C.c_int64), ("hbm_in_use_bytes", C.c_int64), ("hbm_peak_bytes", C.c_int64),
        ("max_live_seen", C.c_int32), ("last_error", C.c_int32),
        ("relayout_wait_ms", C.c_double), ("relayout_build_ms", C.c_double), ("graph_build_ms", C.c_double),
        ("staged", C.c_int64),
    ]


def params_default():
    """The reference's constants (flip.cpp:26-27, solver.inl:107,322-325)."""
    p = AsimParams()
    p.picflip = 0.95
    p.subcell = 1
    p.precond = PRECOND_REF
    p.precision = PREC_REF32
    p.stop_rule = STOP_REF_ABS
    p.max_iters = 0
    p.tol = 1e-5
    p.inner_tol = 1e-6
    p.max_outer = 8
    p.resample_every = 1
    p.mic_tau = 0.97
    p.mic_sigma = 0.25
    p.rng_seed = 0x5EED
    p.use_graph = 1
    p.timing = 0
    p.barrier_timeout_ms = 2000.0
    p.fail_on_not_converged = 0
    return p


def scene_dambreak(n, liquid_hi=(0.4, 0.6, 1.0), dt=1.0 / 240.0, density=0.5, seed=1,
                   jitter=1.0, spheres=()):
    """Synthetic dam break: axis-aligned liquid block from the origin, gravity -9.8 in y."""
    d = AsimSceneDesc()
    d.dim = n
    d.density = density
    d.stepsize = dt
    d.n_forces = 1
    d.forces[0][0], d.forces[0][1], d.forces[0][2] = 0.0, -9.8, 0.0
    d.n_liquid = 1
    for a in range(3):
        d.liquid[0].lo[a] = 0.0
        d.liquid[0].hi[a] = liquid_hi[a]
        d.liquid[0].vel[a] = 0.0
    d.n_solid = len(spheres)
    for i, (c, r) in enumerate(spheres):
        for a in range(3):
            d.solid[i].center[a] = c[a]
        d.solid[i].radius = r
    d.seed = seed
    d.jitter = jitter
    return d


def add_mesh(desc, mesh_id):
    """References a solid mesh (an ariel_mesh_create id) from a scene description."""
    if desc.n_mesh >= MAX_MESHES:
        raise ValueError("at most %d meshes per scene" % MAX_MESHES)
    desc.mesh[desc.n_mesh] = mesh_id
    desc.n_mesh += 1
    return desc


def status_name(code):
    return STATUS_NAMES.get(code, "ARIEL_STATUS_%d" % code)
