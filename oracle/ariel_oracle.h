/*
 * ariel_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of betajippity/Ariel's FLIP step (src/sim/flip.cpp:92-128 and everything it
 * calls), used as the parity checker of the CUDA library and as the timed CPU baseline.
 * Nothing in the product links or calls this code.
 *
 * PINNED to the reference's own code: oracle/Makefile's `reference` target compiles the
 * reference's FLIP step from its unmodified sources (src/sim/flip.cpp with the .inl files it
 * includes, src/grid/particlegrid.cpp) against stand-in headers for the absent glm, TBB and
 * OpenVDB (oracle/refshim/, oracle/ref_driver.cpp) into oracle/_ref/.  tests/test_reference_pin.py
 * holds this restatement bit-identical to it, whole steps and stage by stage, in the reference's
 * configuration (fp32 PCG, its preconditioner and absolute stop rule).  Analytic solid spheres
 * stand in for the reference's mesh solids on both sides.
 *
 * The entry points mirror the product's C ABI (include/ariel.h) with the prefix ariel_ref_.
 */
#ifndef ARIEL_ORACLE_H
#define ARIEL_ORACLE_H

#include "../include/ariel.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ariel_ref ariel_ref;

ariel_status ariel_ref_create(const AsimSceneDesc* desc, const AsimParams* params,
                              ariel_ref** out);
void ariel_ref_destroy(ariel_ref* r);
/* A static solid mesh (before init): triangles in object space placed at object * scale +
 * translate in the unit cube, after the scene's spheres; queried by brute force. */
ariel_status ariel_ref_add_mesh(ariel_ref* r, const float* vertices, int32_t n_vertices, const int32_t* triangles,
                                int32_t n_triangles, const float* translate, float scale);
/* The mesh queries' ray-triangle test for one triangle v[0..8] and ray (o, d): 1 on a hit, with
 * the hit point o + d t in point[0..2] (the value the nearest-hit query records). */
int32_t ariel_ref_tri_ray(const float* v, const float* o, const float* d, float* point);
/* 1: the reference's own parallel granularity (one parallel region per (j,k) line in Op,
 *    the S copy and the backward sweep, serial Sort and Product) -- the timed CPU baseline.
 * 0: one parallel region per loop nest (same results, faster; used by the tests). */
void ariel_ref_set_faithful(ariel_ref* r, int32_t faithful);
void ariel_ref_set_threads(int32_t nthreads);
int32_t ariel_ref_max_threads(void);

ariel_status ariel_ref_init(ariel_ref* r);
ariel_status ariel_ref_step(ariel_ref* r, int32_t nsteps);
ariel_status ariel_ref_stage(ariel_ref* r, int32_t stage);

ariel_status ariel_ref_particle_count(ariel_ref* r, int64_t* n);
ariel_status ariel_ref_get_particles(ariel_ref* r, float* pos, float* vel, float* density,
                                     float* mass, int32_t* type);
ariel_status ariel_ref_set_particles(ariel_ref* r, int64_t n, const float* pos, const float* vel,
                                     const float* mass, const int32_t* type);
ariel_status ariel_ref_get_cells(ariel_ref* r, int32_t* particle_cell, int32_t* cell_count);
ariel_status ariel_ref_get_grid(ariel_ref* r, int32_t which, void* buf, int64_t nbytes);
ariel_status ariel_ref_set_grid(ariel_ref* r, int32_t which, const void* buf, int64_t nbytes);
ariel_status ariel_ref_stats(ariel_ref* r, AsimStats* stats);
ariel_status ariel_ref_get_max_density(ariel_ref* r, float* max_density);
/* Per-stage wall time of the last step (ms, host clock). */
ariel_status ariel_ref_stage_ms(ariel_ref* r, double* ms);

/* Stand-alone FP64 PCG on the reference's ghost-fluid operator: flags (int32 n^3), L (f32 n^3),
 * b (f64 n^3, the negated divergence), x (f64 n^3, warm start in / solution out).  Diagonal
 * (reference) preconditioner, stop at |r|/|b| <= tol.  Returns iterations and the final relative
 * true residual.  Used to report the error of the GPU solves. */
ariel_status ariel_ref_solve_fp64(int32_t n, const int32_t* flags, const float* L, const double* b,
                                  double* x, double tol, int32_t max_iters, int32_t* iterations,
                                  double* rel_residual);
/* FP64 operator apply y = A x on the same operator (non-fluid rows 0). */
ariel_status ariel_ref_apply_fp64(int32_t n, const int32_t* flags, const float* L, const double* x,
                                  double* y);

/* The liquid surface of the oracle's particles: the level set and the surface-nets mesh of
 * ariel_get_level_set / ariel_surface_mesh (include/ariel.h), computed by serial loops. */
ariel_status ariel_ref_level_set(ariel_ref* r, float* phi, int64_t nbytes);
ariel_status ariel_ref_surface_mesh(ariel_ref* r, float* vertices, int64_t max_vertices, int32_t* quads,
                                    int64_t max_quads, int64_t* n_vertices, int64_t* n_quads);

/* Philox4x32-10 block (counter c[4], key k[2]) -> out[4]; exposed for known-answer tests. */
void ariel_ref_philox4x32_10(const uint32_t* c, const uint32_t* k, uint32_t* out);

#ifdef __cplusplus
}
#endif

#endif
