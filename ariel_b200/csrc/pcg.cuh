// pcg.cuh -- pressure-solve data shared by pcg.cu and host.cu.
#pragma once

#include <algorithm>

#include "state.cuh"

namespace ariel {

enum PcgMode { kRef32 = 0, kFp64 = 1, kMixed = 2 };

// Per-scene solver scalars, written by the leader block of each grid barrier.
struct PcgScene {
    double bb;        // |b|^2 over FLUID cells
    double rr;        // r.r of the working (inner) residual
    double rho;       // z.r
    double alpha, beta;
    double rr_out;    // |b - A x|^2 at the last outer residual (FP64/MIXED true residual)
    double target;    // stop threshold on rr of the current (inner) solve
    float alpha32, beta32, rho32, pad32;
    int iters;        // CG iterations (summed over inner solves)
    int outer;        // refinement sweeps
    int done;         // whole solve finished
    int inner_done;   // current inner solve finished
    int converged;
    int ordered;      // preconditioner needs the ordered (wavefront) path
    int ones;         // FLUID cells whose order-free REF preconditioner value is exactly 1
    int nf;           // FLUID cells
    int csize;        // this scene's chunk size (FLUID cells per chunk)
    int pad;
};
static_assert(sizeof(PcgScene) % 16 == 0, "PcgScene is copied as 16-byte words");

// Accumulated over solves (reset by the host); written by the leader when a scene finishes.
struct PcgTotals {
    long long solves, iterations, outer;
    double cell_iterations, cell_outer;
    long long not_converged, pad;
};

struct PcgCtl {
    int all_done;
    int all_inner_done;
    int any_ordered;
    int pad;
};

struct Barrier {
    unsigned count;
    unsigned gen;
    int error;
    int pad;
};

struct PcgArgs {
    DevState S;
    int mode;
    int fast;            // k_pcg_fast handles launches without an ordered preconditioner
    int may_be_ordered;  // the general kernel must also be launched (see launch_pcg_solve)
    int precond;
    int stop_rule;
    int max_iters;     // <=0: n^3 per scene
    int max_outer;
    double tol;
    double inner_tol;
    double tau, sigma;
    unsigned long long timeout_ns;
    // FLUID list
    const uint32_t* fl;        // packed FLUID cells, scene by scene, ascending
    uint4* rec;                // per FLUID-list entry: (cell, neighbour mask, diagonal bits)
    const long long* fl_pref;  // k+1
    const long long* ch_pref;  // k+1 chunk begins
    // per-cell operator data (dense over packed cells)
    uint8_t* mask;   // bit d set: neighbour d (-x,+x,-y,+y,-z,+z) is FLUID
    double* diag;    // ADiag (fp32 value for REF32, fp64 otherwise)
    double* pc64;    // preconditioner values
    float* pc32;
    // vectors (dense over packed cells); element type per mode
    void* r;
    void* z;
    void* s0;
    void* s1;
    void* q;
    void* ordq;      // forward-sweep scratch of the ordered preconditioner
    void* u;         // single-reduction PCG: preconditioned residual
    void* p;         // single-reduction PCG: search direction
    void* va0;       // fast single-reduction PCG: packed (r, w, s, pc), two parities
    void* va1;
    void* vb;        // fast single-reduction PCG: packed (p, x)
    double* r64;     // MIXED outer residual
    float* d32;      // MIXED inner correction
    double* partial; // 3 * max chunks (three dot products per reduction)
    long long max_chunks;
    // ordered wavefront sweeps: bricks of every scene sorted by level I+J+K (then scene, I, J,
    // K), each scene's brick grid starting at brick_base[s], one progress flag per brick
    const int4* bricks;
    const int* brick_base;
    unsigned* bflag;
    int nbricks;
    int bx, by, bz;
    PcgScene* sc;
    PcgTotals* totals;
    PcgCtl* ctl;
    Barrier* bar;
};

// Build the FLUID list, per-cell operator data and chunk table; zero non-FLUID pressure.
cudaError_t launch_pcg_prepare(const PcgArgs& A, uint32_t* pred, uint32_t* scan, void* scan_tmp, cudaStream_t st);
// The cooperative persistent PCG kernel.
cudaError_t launch_pcg_solve(const PcgArgs& A, int nblocks, cudaStream_t st);
// Blocks of the persistent kernel that fit on the device at once.
int pcg_max_blocks(int device, int mode, int per_sm_cap);
// Bounded-wait self test (one arrival missing).
cudaError_t launch_barrier_selftest(Barrier* bar, int* err, unsigned long long timeout_ns, cudaStream_t st);

constexpr int kPcgThreads = 256;
// Chunks of the FLUID list, the unit of every reduction's partial sums.  Each scene's chunk size
// is the FLUID count split kChunkTarget ways (the persistent solve's resident blocks on a B200: 2
// per SM x 148 SMs), rounded up to a multiple of kChunkAlign and kept within [kChunkMin,
// kChunkMax]: a large scene then gives every resident block one chunk and every SM about the same
// number of cells (with power-of-two sizes a 128^3 dam break left 79 SMs with twice the cells of
// the others), a small one still spreads over as many blocks as 512-cell chunks allow, and a huge
// one keeps chunks that fit the shared-memory record cache.  The size depends on the scene alone,
// so a scene's bits do not depend on the batch it is solved in or on the grid.
constexpr int kChunkMin = 512;
constexpr int kChunkMax = 2048;
constexpr int kChunkAlign = 64;
constexpr long long kChunkTarget = 296;
__host__ __device__ inline int chunk_size(long long nf) {
    long long c = (nf + kChunkTarget - 1) / kChunkTarget;
    c = (c + kChunkAlign - 1) / kChunkAlign * kChunkAlign;
    return (int)(c < kChunkMin ? kChunkMin : (c > kChunkMax ? kChunkMax : c));
}
// Most chunks a scene of `cells` cells can have (its FLUID count is at most `cells`).
inline long long chunk_bound(long long cells) {
    const long long lo = (cells + kChunkMin - 1) / kChunkMin;
    const long long hi = (cells + kChunkMax - 1) / kChunkMax;
    return std::min(lo, std::max(kChunkTarget, hi));
}
constexpr int kBrickMaxCells = 2048;
constexpr int kBrickMaxExt = 2744;
constexpr int kBrickMaxLevels = 128;
// Dynamic shared memory of the general solve kernel (the ordered wavefront sweeps' boxes).
size_t brick_dyn_smem();
bool brick_shape_ok(int bx, int by, int bz);

}  // namespace ariel
