/*
 * ariel.h -- C ABI of the B200-native FLIP step (sm_100a CUDA behind plain C).
 *
 * This library replaces the hot path of betajippity/Ariel, `fluidCore::FlipSim::Step`
 * (src/sim/flip.cpp:92-128), and the free functions it calls:
 *   SplatParticlesToMACGrid / SplatMACGridToParticles / EnforceBoundaryVelocity /
 *   InterpolateVelocity   (src/sim/particlegridoperations.inl:23-29),
 *   Solve                 (src/sim/solver.inl:23),
 *   ResampleParticles     (src/sim/particleresampler.inl:23-26),
 *   ParticleGrid::Sort / MarkCellTypes / BuildSDF (src/grid/particlegrid.hpp:28-39).
 *
 * One handle (`ariel_sim`) owns 1..k scenes that are stepped together.  All grid and
 * particle state stays resident in device memory; the caller owns every host buffer
 * passed in or out.  Calls on one handle are not thread-safe; distinct handles are.
 * Every entry point returns an `ariel_status`.
 *
 * Units and layouts follow the reference:
 *   - particle positions are in the unit cube [0,1]^3 (src/grid/macgrid.inl:36-50),
 *     host particle buffers are xyz-interleaved float triples in particle-id order;
 *   - grids are cubic, n cells per axis (the reference's G2P assumes a cube:
 *     src/sim/particlegridoperations.inl:121-124);
 *   - cell (i,j,k) is stored at (i*n + j)*n + k; the x-face grid has (n+1)*n*n entries at
 *     (i*n + j)*n + k, the y-face grid n*(n+1)*n at (i*(n+1) + j)*n + k and the z-face
 *     grid n*n*(n+1) at (i*n + j)*(n+1) + k  (src/grid/macgrid.inl:72-84).
 */
#ifndef ARIEL_H
#define ARIEL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ARIEL_ABI_VERSION 2

typedef enum ariel_status {
    ARIEL_OK = 0,
    ARIEL_ERR_INVALID_ARG = 1,    /* bad pointer, size, mode or scene index */
    ARIEL_ERR_OOM = 2,            /* device allocation refused or HBM budget exceeded */
    ARIEL_ERR_NOT_CONVERGED = 3,  /* pressure solve hit its iteration cap above tolerance */
    ARIEL_ERR_DEVICE_TIMEOUT = 4, /* a bounded device-side wait ran out (grid barrier, flag) */
    ARIEL_ERR_CUDA = 5,           /* a CUDA runtime call failed */
    ARIEL_ERR_STATE = 6,          /* call out of order (e.g. step before init) */
    ARIEL_ERR_NO_DEVICE = 7,      /* no usable sm_100 device */
    ARIEL_ERR_NAN = 8,            /* non-finite value in host input */
    ARIEL_ERR_PENDING = 9         /* server request not finished within the wait */
} ariel_status;

/* Cell types: enum geomtype {SOLID=2, FLUID=1, AIR=0} (src/grid/macgrid.inl:13). */
enum { ARIEL_AIR = 0, ARIEL_FLUID = 1, ARIEL_SOLID = 2 };

/* Preconditioner.
 * REF : the reference's BuildPreconditioner/ApplyPreconditioner (src/sim/solver.inl:104-135,
 *       232-286) including its PRef value==1.0f test (solver.inl:72-78).
 * MIC0: modified incomplete Cholesky MIC(0) with tau/sigma (Bridson), FP64 factorisation,
 *       forward/backward substitution as i+j+k wavefront sweeps. */
enum { ARIEL_PRECOND_REF = 0, ARIEL_PRECOND_MIC0 = 1 };

/* Pressure-solve precision.
 * REF32: every vector in fp32, the reference's own operator expression (solver.inl:196-230).
 * FP64 : every PCG vector, coefficient and scalar in fp64 (the plain FP64 GPU path).
 * MIXED: fp32 SpMV / preconditioner / vector updates inside an fp64 iterative-refinement
 *        outer loop; fp64 dots, alpha/beta, outer true residual and MIC(0) diagonal. */
enum { ARIEL_PREC_REF32 = 0, ARIEL_PREC_FP64 = 1, ARIEL_PREC_MIXED = 2 };

/* Stop rule. REF_ABS: r.r <= 1e-2*n^3 (solver.inl:322,339).  REL: |r|/|b| <= tol. */
enum { ARIEL_STOP_REF_ABS = 0, ARIEL_STOP_REL = 1 };

/* Stages of FlipSim::Step, in call order (src/sim/flip.cpp:92-128).  `ariel_stage` runs one;
 * `ariel_step` runs all of them and advances the frame counter. */
enum {
    ARIEL_STAGE_BEGIN = 0,        /* frame++, AdjustParticlesStuckInSolids, StoreTemp (:93-103) */
    ARIEL_STAGE_SORT = 1,         /* ParticleGrid::Sort (:104) */
    ARIEL_STAGE_DENSITY = 2,      /* ComputeDensity (:105) */
    ARIEL_STAGE_FORCES = 3,       /* ApplyExternalForces (:106) */
    ARIEL_STAGE_P2G = 4,          /* SplatParticlesToMACGrid (:107) */
    ARIEL_STAGE_CLASSIFY = 5,     /* MarkCellTypes (:108) + the BuildSDF of Project (:440) */
    ARIEL_STAGE_BOUNDARY_DIV = 6, /* StorePreviousGrid, EnforceBoundaryVelocity, divergence,
                                     FlipGrid (:109-110, :420-437, solver.inl:365) */
    ARIEL_STAGE_SOLVE = 7,        /* BuildPreconditioner + SolveConjugateGradient (solver.inl:356) */
    ARIEL_STAGE_GRADIENT = 8,     /* SubtractPressureGradient + EnforceBoundaryVelocity (:449,:112) */
    ARIEL_STAGE_EXTRAPOLATE = 9,  /* ExtrapolateVelocity + SubtractPreviousGrid (:113-114) */
    ARIEL_STAGE_G2P_ADVECT = 10,  /* SolvePicFlip + AdvectParticles + CheckParticleSolidConstraints
                                     (:115-118) */
    ARIEL_STAGE_RESAMPLE = 11,    /* StoreTemp + ResampleParticles + CheckParticleSolidConstraints
                                     (:119-123) */
    ARIEL_STAGE_COUNT = 12
};

/* Grid selectors for ariel_get_grid / ariel_set_grid. */
enum {
    ARIEL_GRID_UX = 0, ARIEL_GRID_UY = 1, ARIEL_GRID_UZ = 2,          /* m_mgrid faces, f32 */
    ARIEL_GRID_PREV_UX = 3, ARIEL_GRID_PREV_UY = 4, ARIEL_GRID_PREV_UZ = 5, /* m_mgrid_previous */
    ARIEL_GRID_D = 6,   /* divergence (negated after FlipGrid), f32 n^3 */
    ARIEL_GRID_P = 7,   /* pressure, f32 n^3 */
    ARIEL_GRID_L = 8,   /* liquid SDF, f32 n^3 */
    ARIEL_GRID_A = 9,   /* cell types, int32 n^3 */
    ARIEL_GRID_P64 = 10 /* fp64 pressure kept for FP64/MIXED warm starts, f64 n^3 */
};

#define ARIEL_MAX_BOXES 8
#define ARIEL_MAX_SPHERES 8
#define ARIEL_MAX_FORCES 4
#define ARIEL_MAX_MESHES 8

/* Axis-aligned liquid block in unit coordinates (a `mesh_gen` box of the reference's scenes,
 * src/scene/sceneloader.cpp:346-398), with its starting velocity (scene.cpp:280). */
typedef struct AsimBox {
    float lo[3];
    float hi[3];
    float vel[3];
} AsimBox;

/* Static solid sphere in unit coordinates; becomes SOLID particles of mass 10 at the lattice
 * points inside it (src/scene/scene.cpp:457-477), and the analytic surface for the ray and
 * point-inside tests of the solid constraints (flip.cpp:130-227). */
typedef struct AsimSphere {
    float center[3];
    float radius;
} AsimSphere;

typedef struct AsimSceneDesc {
    int32_t dim;          /* n: cubic grid of n^3 cells (FlipSim maxres) */
    float density;        /* lattice spacing in cells: 0.5 -> 8 particles/cell (sceneloader.cpp:411) */
    float stepsize;       /* dt (FlipSim stepsize) */
    int32_t n_forces;     /* external forces, applied in order (flip.cpp:682-695) */
    float forces[ARIEL_MAX_FORCES][3];
    int32_t n_liquid;
    AsimBox liquid[ARIEL_MAX_BOXES];
    int32_t n_solid;
    AsimSphere solid[ARIEL_MAX_SPHERES];
    uint64_t seed;        /* seeds the in-sub-cell jitter of the initial liquid lattice */
    float jitter;         /* 1: uniform jitter inside each lattice sub-cell; 0: sub-cell centres */
    int32_t reserved;
    int32_t n_mesh;       /* static solid meshes (ariel_mesh_create ids), after the spheres */
    int32_t mesh[ARIEL_MAX_MESHES];
} AsimSceneDesc;

typedef struct AsimParams {
    float picflip;            /* FLIP fraction of the PIC/FLIP blend (flip.cpp:27: .95) */
    int32_t subcell;          /* ghost-fluid pressure boundary (flip.cpp:26: 1) */
    int32_t precond;          /* ARIEL_PRECOND_* */
    int32_t precision;        /* ARIEL_PREC_* */
    int32_t stop_rule;        /* ARIEL_STOP_* */
    int32_t max_iters;        /* PCG iteration cap; 0 -> n^3 (solver.inl:325) */
    double tol;               /* relative tolerance for ARIEL_STOP_REL */
    double inner_tol;         /* MIXED: relative reduction asked of each fp32 inner solve (1e-6) */
    int32_t max_outer;        /* MIXED: cap on refinement sweeps */
    int32_t resample_every;   /* resample every k-th step; 1 = every step as the reference
                                 (flip.cpp:121); 0 = never */
    double mic_tau;           /* MIC(0) tau (0.97) */
    double mic_sigma;         /* MIC(0) safety (0.25) */
    uint64_t rng_seed;        /* counter-based RNG seed for the resampling jitter, which
                                 replaces rand() (particleresampler.inl:69-71) */
    int32_t use_graph;        /* capture one step per CUDA graph and replay it */
    int32_t timing;           /* record per-stage CUDA-event times (adds event records) */
    double barrier_timeout_ms;/* bound of every device-side spin wait */
    int32_t fail_on_not_converged; /* return ARIEL_ERR_NOT_CONVERGED from step when a solve
                                      stops at max_iters above tolerance */
    int32_t pcg_blocks_per_sm;  /* blocks per SM of the persistent solve kernel; 0 = default (2) */
    int32_t pcg_grid_blocks;    /* >0: cap on the solve kernel's blocks in all (results do not
                                   depend on it; tests and tuning); 0 = one grid of resident blocks */
    int32_t sweep_brick[3];     /* brick (i, j, k extents in cells) of the ordered wavefront sweeps
                                   (MIC(0) and the reference's PRef==1 path); results do not depend
                                   on it.  0,0,0 = default 12,12,12.  Limits: i,j <= 31, k <= 63,
                                   product <= 2048, (i+1)(j+1)(k+1) <= 2744 */
    int32_t p2g_faces;          /* faces of one row each thread of the grid transfer (P2G) takes:
                                   1, 2 or 4; 0 = chosen by the number of faces.  Results do not
                                   depend on it */
    int32_t reseed_every;       /* 0 = off; else, on frames divisible by it and after resampling,
                                   particles above reseed_max in a FLUID cell move to interior FLUID
                                   cells (all six neighbours FLUID) below reseed_min.  The particle
                                   count is kept.  No counterpart in the reference, which never
                                   adds or removes particles */
    int32_t reseed_min;         /* 0 -> 6 */
    int32_t reseed_max;         /* 0 -> 10 */
} AsimParams;

typedef struct AsimStats {
    int64_t frame;            /* FlipSim::m_frame */
    int64_t n_particles;
    int64_t n_fluid_cells;    /* FLUID cells at the last solve */
    int32_t pcg_iterations;   /* last solve: CG iterations (sum of inner iterations for MIXED) */
    int32_t pcg_outer;        /* last solve: refinement sweeps (MIXED), else 1 */
    double pcg_rel_residual;  /* last solve: final |r|/|b| (true residual for FP64/MIXED) */
    double pcg_rr;            /* last solve: final r.r as tested by the stop rule */
    int32_t pcg_converged;    /* last solve met its stop rule */
    int32_t precond_exact_path; /* last solve needed the ordered (wavefront) REF preconditioner */
    double stage_ms[ARIEL_STAGE_COUNT]; /* last step, per stage (when timing is on) */
    double step_ms;           /* last step, device time (when timing is on) */
    int32_t last_status;
    int32_t reserved;
} AsimStats;

/* Pressure-solve totals accumulated on the device since the last ariel_timing_reset. */
typedef struct AsimSolverTotals {
    int64_t solves;
    int64_t iterations;        /* CG iterations (inner iterations for MIXED) */
    int64_t outer;             /* refinement sweeps (MIXED), else one per solve */
    double cell_iterations;    /* sum over solves of FLUID cells x iterations */
    double cell_outer;         /* sum over solves of FLUID cells x sweeps */
    int64_t not_converged;
    int64_t reserved;
} AsimSolverTotals;

typedef struct ariel_sim ariel_sim;

/* Defaults: the reference's constants, REF preconditioner, REF32 precision, REF_ABS stop. */
void ariel_params_default(AsimParams* params);
/* Dam break: liquid block x in [0,.4], y in [0,.6], z in [0,1], gravity -9.8 y, dt 1/240. */
void ariel_scene_dambreak(AsimSceneDesc* desc, int32_t n);
const char* ariel_status_string(ariel_status status);
int32_t ariel_abi_version(void);

/* FlipSim(maxres, density, stepsize, scene, verbose) (src/sim/flip.hpp:22-23). */
ariel_status ariel_create(const AsimSceneDesc* desc, const AsimParams* params, ariel_sim** out);
/* k scenes of any sizes stepped together over one packed cell/particle index space. */
ariel_status ariel_create_batch(const AsimSceneDesc* descs, int32_t k, const AsimParams* params,
                                ariel_sim** out);
ariel_status ariel_destroy(ariel_sim* sim);
ariel_status ariel_scene_count(ariel_sim* sim, int32_t* k);

/* FlipSim::Init (src/sim/flip.cpp:42-77): density normaliser from a 10^3 lattice, particle
 * seeding (src/scene/scene.cpp:257-360), Sort and MarkCellTypes. */
ariel_status ariel_init(ariel_sim* sim);
/* FlipSim::Step (src/sim/flip.cpp:92-128) n times for every scene of the handle. */
ariel_status ariel_step(ariel_sim* sim, int32_t nsteps);
/* One stage (ARIEL_STAGE_*) for every scene; does not advance the frame except BEGIN. */
ariel_status ariel_stage(ariel_sim* sim, int32_t stage);
ariel_status ariel_synchronize(ariel_sim* sim);

/* FlipSim::GetParticles (src/sim/flip.hpp:29). Any output pointer may be NULL. */
ariel_status ariel_particle_count(ariel_sim* sim, int32_t scene, int64_t* n);
ariel_status ariel_get_particles(ariel_sim* sim, int32_t scene, float* pos, float* vel,
                                 float* density, float* mass, int32_t* type);
/* Replace a scene's particles (positions/velocities xyz-interleaved, unit coordinates). */
ariel_status ariel_set_particles(ariel_sim* sim, int32_t scene, int64_t n, const float* pos,
                                 const float* vel, const float* mass, const int32_t* type);
/* Particle-to-cell index (per particle, id order) and per-cell counts from the last Sort. */
ariel_status ariel_get_cells(ariel_sim* sim, int32_t scene, int32_t* particle_cell,
                             int32_t* cell_count);
ariel_status ariel_get_grid(ariel_sim* sim, int32_t scene, int32_t which, void* buf,
                            int64_t nbytes);
ariel_status ariel_set_grid(ariel_sim* sim, int32_t scene, int32_t which, const void* buf,
                            int64_t nbytes);
ariel_status ariel_get_dimensions(ariel_sim* sim, int32_t scene, int32_t* n);
ariel_status ariel_stats(ariel_sim* sim, int32_t scene, AsimStats* stats);
/* Normaliser m_max_density computed by Init (flip.cpp:62-70). */
ariel_status ariel_get_max_density(ariel_sim* sim, int32_t scene, float* max_density);

/* Per-step particle I/O through host buffers (the reference's GetParticles use, with the
 * particles kept by the caller): xyz-interleaved positions and velocities of the scene's
 * current particles, in id order.  Upload is asynchronous on the handle's stream (pinned host
 * memory makes it a true async copy; the buffers must stay valid until the next synchronising
 * call); download returns when the data is in `pos`/`vel`. */
ariel_status ariel_upload_state(ariel_sim* sim, int32_t scene, const float* pos, const float* vel);
ariel_status ariel_download_state(ariel_sim* sim, int32_t scene, float* pos, float* vel);

/* Device timing of whole steps on the handle's stream (CUDA events). */
ariel_status ariel_timer_begin(ariel_sim* sim);
ariel_status ariel_timer_end(ariel_sim* sim, double* ms);

/* Per-stage device times accumulated over every step run since the last reset (requires
 * params.timing = 1, which keeps graph replay and double-buffers the stage events so the
 * device is never idle while they are read).  ms[ARIEL_STAGE_COUNT] receives the per-stage
 * sums, solve_kernel_ms the persistent solve kernel alone, step_ms (may be NULL) the
 * per-step totals of the last `max_steps` steps; *nsteps the number of steps summed. */
ariel_status ariel_timing_reset(ariel_sim* sim);
ariel_status ariel_solver_totals(ariel_sim* sim, int32_t scene, AsimSolverTotals* totals);
ariel_status ariel_timing_get(ariel_sim* sim, double* ms, double* solve_kernel_ms, double* step_ms,
                              int32_t max_steps, int32_t* nsteps);

/* Device-side failure detection: runs the bounded grid barrier with one arrival missing so
 * that it must time out after `timeout_ms`; returns ARIEL_ERR_DEVICE_TIMEOUT when the bound
 * worked and ARIEL_OK if the barrier (wrongly) completed. */
ariel_status ariel_selftest_barrier_timeout(double timeout_ms);

/* Static solid meshes: the reference's solid mesh geoms (Scene's solids built from OBJ files,
 * src/scene/scene.cpp:362-434, src/geom/obj/obj.cpp) for scenes that reference them through
 * AsimSceneDesc.mesh.  `vertices` holds n_vertices xyz triples in object space, `triangles`
 * n_triangles index triples (0-based, quads split by the caller); the mesh is placed in the unit
 * cube as object * scale + translate (uniform scale and translation; rotations are not
 * supported).  A solid mesh contains a point when a ray from it along +z crosses the mesh an odd
 * number of times (Scene::CheckPointInsideSolidGeom, scene.cpp:382-402); it yields SOLID
 * particles at the lattice points inside it and takes part in the solid constraints.  The
 * library keeps its own copy; host-side only (no device needed), thread-safe.  Limits: at most
 * 2^24 triangles per mesh.  A scene keeps working with a mesh destroyed after its handle was
 * created, but new handles referencing a destroyed id are refused. */
ariel_status ariel_mesh_create(const float* vertices, int32_t n_vertices, const int32_t* triangles,
                               int32_t n_triangles, const float* translate, float scale, int32_t* mesh_id);
ariel_status ariel_mesh_destroy(int32_t mesh_id);
/* A registered mesh's vertex and triangle counts and placement (any pointer may be null). */
ariel_status ariel_mesh_info(int32_t mesh_id, int32_t* n_vertices, int32_t* n_triangles, float* translate,
                             float* scale);

/* Scene files (SceneLoader, src/scene/sceneloader.cpp:11-131, 346-443): the reference's JSON
 * scene (settings, globalforces, transforms, meshfiles, geoms, sim) into *desc.  A box liquid
 * becomes an AsimBox, a sphere solid an AsimSphere; box solids and solids read from OBJ files
 * (paths relative to the scene file, src/geom/obj/obj.cpp) are registered as static meshes
 * (ariel_mesh_create), listed in desc->mesh, and stay registered until ariel_mesh_destroy.
 * What the path cannot represent (liquids from meshes, animated meshes, rotations, non-uniform
 * scaling of spheres or meshes, geometry appearing after frame 0, non-cubic grids, more boxes,
 * spheres, meshes or forces than the ABI holds, missing ids, unreadable files) returns
 * ARIEL_ERR_INVALID_ARG with the reason in `error` (when given) and registers nothing.  The
 * reference seeds liquid particles at lattice-cell centres: pass jitter 0 to match it.
 * Host-side only (no device needed). */
typedef struct AsimSceneInfo {
    int32_t dim;
    int32_t reserved;
    double density;           /* settings.density as written (desc->density is its float) */
    double step_size;
    char partio_output[512];  /* settings' output paths ("" when absent) */
    char vdb_output[512];
    char mesh_output[512];
} AsimSceneInfo;
ariel_status ariel_scene_load(const char* path, float jitter, uint64_t seed, AsimSceneDesc* desc,
                              AsimSceneInfo* info, char* error, int32_t error_len);
/* The same from the file's text; `base_dir` resolves OBJ paths. */
ariel_status ariel_scene_parse(const char* json_text, const char* base_dir, float jitter, uint64_t seed,
                               AsimSceneDesc* desc, AsimSceneInfo* info, char* error, int32_t error_len);

/* Checkpoints: every piece of state a step reads from the previous one (particles, pressure
 * warm start, frame counter, density normaliser) of every scene of the handle, in one file.
 * Loading needs a handle created with the same scene descriptions and continues
 * bit-identically.  Replaces no reference function: the reference's only output is the particle
 * export below. */
ariel_status ariel_checkpoint_save(ariel_sim* sim, const char* path);
ariel_status ariel_checkpoint_load(ariel_sim* sim, const char* path);
/* Scene::ExportParticles' particle branch (src/scene/scene.cpp:35-80): FLUID particles with
 * position (grid units), v and id, to `path` with ".%04d" of `frame` inserted before the
 * extension (".gz" counted as part of it).  Written as Houdini classic ASCII geometry; `path`
 * must end in ".geo", or ".geo.gz" for gzip-compressed output. */
ariel_status ariel_export_particles(ariel_sim* sim, int32_t scene, const char* path, int32_t frame);

/* Count of this library's kernel launches issued so far (all handles). */
int64_t ariel_kernel_launches(void);

/* Liquid surface of one scene, for output: the reference's LevelSet(particles) (OpenVDB
 * ParticlesToLevelSet, src/grid/levelset.cpp:101-111) and LevelSet::WriteObjToFile (OpenVDB
 * VolumeToMesh, levelset.cpp:113-172), which Scene::ExportParticles' VDB/OBJ branch calls
 * (src/scene/scene.cpp:84-100).  The level set: FLUID particles as spheres of radius 0.5 cells
 * rasterised on the integer points of the grid, padded 2 cells beyond each wall; a sample holds
 * the smallest (distance to a particle - 0.5) within 2 cells, else 1.5.  The mesh: surface nets
 * at level 0 (one vertex per sign-changing grid cube, one quad per sign-changing grid edge,
 * normals from inside to outside), in grid units.  Temporaries are allocated for the call.
 *
 * ariel_get_level_set: N^3 floats, N = n + 5, sample (i, j, k) at grid point (i-2, j-2, k-2),
 *   i slowest.
 * ariel_surface_mesh: the counts, and -- when the buffers are given and large enough --
 *   vertices (xyz floats) and quads (4 vertex indices each, 0-based).  Buffers too small:
 *   ARIEL_ERR_INVALID_ARG with the counts set.
 * ariel_export_surface: the mesh as a Wavefront OBJ at `path` (ending in ".obj") with ".%04d" of
 *   `frame` inserted before the extension (Scene::ExportParticles' naming, scene.cpp:89-90). */
ariel_status ariel_get_level_set(ariel_sim* sim, int32_t scene, float* phi, int64_t nbytes);
ariel_status ariel_surface_mesh(ariel_sim* sim, int32_t scene, float* vertices, int64_t max_vertices, int32_t* quads,
                                int64_t max_quads, int64_t* n_vertices, int64_t* n_quads);
ariel_status ariel_export_surface(ariel_sim* sim, int32_t scene, const char* path, int32_t frame);

/* Text of the last CUDA failure seen by this thread (the failing call and CUDA's message). */
const char* ariel_last_error(void);

/* Sort-by-cell without any device allocation.  No counterpart in the reference: it serves
 * callers that cannot call cudaMalloc once running -- real-time loops that must not stall on an
 * allocation, and hosts whose own allocator owns all device memory and only hands out its
 * buffers.  Same binning as ARIEL_STAGE_SORT: for `n` particles at device positions `pos`
 * (xyz-interleaved floats in the unit cube; coordinates outside it are clamped into the edge
 * cells, as ParticleGrid::Sort does) on a `dim`^3 grid it writes, into caller-provided device
 * memory, the cell of every particle (particle_cell[n]), the exclusive prefix of per-cell counts
 * (cell_start[dim^3 + 1]) and the particle ids grouped by cell, ascending inside a cell
 * (order[n]).  Work is queued on `stream` (a cudaStream_t; NULL for the default stream) and the
 * call returns without waiting.
 * Limits: n <= 1,048,576 and dim^3 <= 262,144 (a 64^3 grid); larger requests return
 * ARIEL_ERR_INVALID_ARG.  Temporaries live in one fixed array of about 5.2 MB inside the
 * library, held on every GPU that loads it until the process exits.  Under CUDA's default lazy
 * module loading that array is allocated when the library's module first loads on a device,
 * i.e. by the first call there: make one call on each device at start-up, before any stream
 * capture and before the caller's allocator takes over the device's memory (or run with
 * CUDA_MODULE_LOADING=EAGER).  The array's device address is looked up on every call, so the
 * entry point keeps working after the caller resets the device.
 * Every call reuses the array (per-cell counters are cleared by each call): calls that may
 * overlap on the GPU race and must be serialised by the caller.  Cost is linear in n except for
 * cells of more than 4,096 particles, which are ordered in time quadratic in their size. */
ariel_status ariel_sort_by_cell_noalloc(const float* pos, int64_t n, int32_t dim, uint32_t* particle_cell,
                                        uint32_t* cell_start, uint32_t* order, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Request server (continuous batching).  No counterpart in the reference, whose viewer steps one
 * scene in a loop (src/viewer/viewer.cpp:66-87).  Scenes arrive as requests of a number of
 * steps; host threads seed their particles while the device steps the live ones; between two
 * batch steps the server retires finished scenes (copying their particles out) and admits
 * waiting ones, oldest first, while the device bytes of the re-packed layout fit the budget.
 * All live scenes share each stage's launch.  A scene's results are the same as when it is
 * stepped alone with the same AsimParams.
 * ------------------------------------------------------------------------------------------- */
typedef struct ariel_server ariel_server;

typedef struct AsimServerConfig {
    int64_t hbm_budget_bytes; /* device bytes for scene state; 0: 85% of the free memory */
    int32_t max_live;         /* scenes stepped together at most (<= 1024); 0: 32 */
    int32_t prepare_threads;  /* host threads seeding arriving scenes; 0: 4 */
    int32_t keep_results;     /* 1: keep each finished scene's particles for fetch */
    int32_t max_ready;        /* seeded scenes waiting for admission at most (their particles are
                                 uploaded ahead to device memory when the budget allows); 0: 8 */
    int32_t reserve_budget;   /* 1: map the whole budget into the server's memory pool at creation,
                                 so that no re-packing waits for the pool to grow */
    int32_t reserved[5];
} AsimServerConfig;

enum { ARIEL_REQ_QUEUED = 0, ARIEL_REQ_READY = 1, ARIEL_REQ_RUNNING = 2, ARIEL_REQ_DONE = 3, ARIEL_REQ_FAILED = 4 };

typedef struct AsimRequestInfo {
    int32_t state;        /* ARIEL_REQ_* */
    int32_t status;       /* failure status when FAILED */
    int32_t nsteps;
    int32_t steps_done;   /* steps queued for this scene so far */
    int64_t n_particles;  /* known once seeded */
    int64_t state_bytes;  /* device bytes of the scene alone */
    double submit_ms, admit_ms, done_ms; /* since server creation; -1 until reached */
    AsimStats stats;      /* the scene's stats after its last step (DONE) */
} AsimRequestInfo;

typedef struct AsimServerStats {
    int64_t submitted, admitted, finished, failed, live, waiting;
    int64_t batch_steps;      /* steps of the whole batch */
    int64_t particle_steps;   /* sum over batch steps of the particles stepped */
    int64_t timed_steps;      /* batch steps with a device time below */
    double wall_ms;           /* since server creation */
    double busy_ms;           /* device time of all batch steps */
    double step_ms_p50, step_ms_p99, step_ms_max; /* device time per batch step */
    double latency_ms_p50, latency_ms_p99;        /* submit -> done per finished request */
    int64_t relayouts;
    double relayout_ms;       /* host time spent re-packing (includes admission copies) */
    int64_t hbm_budget_bytes, hbm_in_use_bytes, hbm_peak_bytes;
    int32_t max_live_seen;
    int32_t last_error;
    double relayout_wait_ms;  /* part of relayout_ms spent waiting for the batch step in flight */
    double relayout_build_ms; /* part of relayout_ms spent allocating and filling the new layout */
    double graph_build_ms;    /* host time capturing and instantiating step graphs */
    int64_t staged;           /* scenes whose particles were uploaded ahead of admission */
} AsimServerStats;

void ariel_server_config_default(AsimServerConfig* config);
ariel_status ariel_server_create(const AsimParams* params, const AsimServerConfig* config, ariel_server** out);
/* Queues a scene for `nsteps` steps; returns at once with its id. */
ariel_status ariel_server_submit(ariel_server* server, const AsimSceneDesc* desc, int32_t nsteps, int64_t* id);
ariel_status ariel_server_poll(ariel_server* server, int64_t id, AsimRequestInfo* info);
/* ARIEL_OK when the request is done, its failure status when it failed, ARIEL_ERR_PENDING
 * when `timeout_ms` passed first. */
ariel_status ariel_server_wait(ariel_server* server, int64_t id, double timeout_ms);
/* Waits until every submitted request is done or failed (ARIEL_ERR_PENDING on timeout). */
ariel_status ariel_server_drain(ariel_server* server, double timeout_ms);
/* A finished request's particles, id order, xyz-interleaved (3 * n_particles floats each). */
ariel_status ariel_server_fetch(ariel_server* server, int64_t id, float* pos, float* vel);
/* Forgets a finished request and its results. */
ariel_status ariel_server_release(ariel_server* server, int64_t id);
ariel_status ariel_server_stats(ariel_server* server, AsimServerStats* stats);
/* Stops the server; requests not finished fail with ARIEL_ERR_STATE.  Frees the handle. */
ariel_status ariel_server_shutdown(ariel_server* server);
/* Device bytes a handle (or a server batch) holds for these scenes (seeds them on the host to
 * count their particles). */
ariel_status ariel_state_bytes(const AsimSceneDesc* descs, int32_t k, const AsimParams* params, int64_t* bytes);

#ifdef __cplusplus
}
#endif

#endif /* ARIEL_H */
