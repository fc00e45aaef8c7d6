// pcg.cu -- the pressure Poisson solve (Solve, src/sim/solver.inl:356-379) on sm_100a.
//
// One cooperative, persistent kernel runs the whole solve for every scene of the handle:
// FLUID cells are split into fixed-size chunks that belong to exactly one scene; each chunk
// writes its partial dot products; the last block to arrive at a grid barrier reduces each
// scene's chunk partials in a fixed order and updates that scene's alpha/beta/stop state.
// Results therefore do not depend on block scheduling, nor on which other scenes share the
// launch (a scene's chunk boundaries depend only on its own FLUID count).
//
// Precision modes:
//   kRef32 -- the reference's fp32 arithmetic: ComputeAx's exact expression (solver.inl:196-230),
//             Op's x + alpha*y updates (:157-177), fp32 alpha/beta; dots accumulate in fp64 and
//             are rounded to fp32 (the reference's serial float Product is only less accurate).
//   kFp64  -- every vector and scalar fp64 (the plain FP64 GPU path).
//   kMixed -- fp64 iterative refinement: true residual, x and dots in fp64; each correction
//             solve's SpMV, preconditioner apply and vector updates in fp32.
// Preconditioner: the reference's (elementwise unless a FLUID value is exactly 1.0, then an
// ordered i+j+k hyperplane sweep), or MIC(0) (ordered sweeps).
//
// Every wait is bounded by a globaltimer budget; on expiry the kernel records an error word
// and all blocks return.
#include <cooperative_groups.h>

#include "pcg.cuh"

namespace ariel {

namespace {

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier for co-resident blocks.  The last block to arrive runs `leader` (all of its
// threads) before releasing the others.  Returns false if the wait ran out of time or another
// block reported an error; the caller must then return.
// Memory ordering: the block's writes are ordered before its arrival by __syncthreads plus one
// gpu-scope fence by thread 0 (fences are cumulative); after the release is observed, thread 0
// fences again (acquire), so every thread of the block may read other blocks' writes with
// ordinary cached loads after the closing __syncthreads -- the same guarantee grid-wide
// cooperative-group synchronisation gives.
template <class F>
__device__ bool grid_barrier(Barrier* bar, int* dev_error, unsigned long long timeout_ns, F&& leader) {
    __shared__ int s_last, s_ok;
    __shared__ unsigned s_gen;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned g = *(volatile unsigned*)&bar->gen;
        s_gen = g;
        __threadfence();
        unsigned arrived = atomicAdd(&bar->count, 1u);
        s_last = (arrived == gridDim.x - 1);
        s_ok = 1;
        if (!s_last) {
            unsigned long long t0 = gtimer();
            while (*(volatile unsigned*)&bar->gen == g) {
                if (*(volatile int*)&bar->error) {
                    s_ok = 0;
                    break;
                }
                if (gtimer() - t0 > timeout_ns) {
                    atomicExch(&bar->error, 1);
                    if (dev_error) atomicExch(dev_error, 1);
                    s_ok = 0;
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
    }
    __syncthreads();
    if (s_last) {
        leader();
        __syncthreads();
        if (threadIdx.x == 0) {
            bar->count = 0;
            __threadfence();
            st_release_u32(&bar->gen, s_gen + 1);
        }
        __syncthreads();
    }
    return s_ok != 0;
}

struct NoLeader {
    __device__ void operator()() const {}
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block reduction of two values; result valid in thread 0.
__device__ __forceinline__ void block_sum2(double& a, double& b) {
    __shared__ double sa[kPcgThreads / 32], sb[kPcgThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) {
        sa[wid] = a;
        sb[wid] = b;
    }
    __syncthreads();
    if (wid == 0) {
        a = lane < kPcgThreads / 32 ? sa[lane] : 0.0;
        b = lane < kPcgThreads / 32 ? sb[lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
    }
    __syncthreads();
}

// Sum of partial[b..e) by one warp in a fixed tree that depends only on e-b (so a scene's
// result does not depend on which scenes share the launch); valid in every lane.  Loads are
// issued 16 per lane before any add so that the leader pays about one L2 round trip.
__device__ __forceinline__ double scene_sum(const double* part, long long b, long long e) {
    const int lane = threadIdx.x & 31;
    double v = 0.0;
    for (long long base = b; base < e; base += 32 * 16) {
        double x[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            long long c = base + (long long)u * 32 + lane;
            x[u] = c < e ? part[c] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) v += x[u];
    }
    v = warp_sum(v);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Whole-struct copy of a scene's solver state (read after a grid barrier).
__device__ __forceinline__ PcgScene load_sc(const PcgScene* p) {
    PcgScene v;
    const int4* src = reinterpret_cast<const int4*>(p);
    int4* dst = reinterpret_cast<int4*>(&v);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(PcgScene) / 16); ++i) dst[i] = src[i];
    return v;
}

template <int MODE>
struct VT {
    using T = float;
};
template <>
struct VT<kFp64> {
    using T = double;
};

// ------------------------------------------------------------------------------------------
// Preparation: per-cell operator data, order-free preconditioner, FLUID predicate.
// ------------------------------------------------------------------------------------------
__global__ void k_prep_cells(PcgArgs A, uint32_t* pred) {
    const DevState& S = A.S;
    __shared__ long long pref_s[kMaxScenes + 1];
    load_prefix<kMaxScenes>(pref_s, S.c_pref, S.k);
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= S.nc) return;
    int s = find_scene(pref_s, S.k, c);
    const SceneDev& D = S.scenes[s];
    const int n = D.n;
    const uint8_t flag = S.flags[c];
    pred[c] = flag == ARIEL_FLUID;
    if (flag != ARIEL_FLUID) {
        S.P[c] = 0.0f;
        if (S.P64) S.P64[c] = 0.0;
        A.mask[c] = 0;
        A.diag[c] = 0.0;
        A.pc64[c] = 0.0;
        A.pc32[c] = 0.0f;
        return;
    }
    int i, j, k;
    cell_ijk(D, c - D.c_begin, i, j, k);
    const int q[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
    const float Lc = S.L[c];
    float d32 = 6.0f;
    double d64 = 6.0;
    uint8_t m = 0;
    for (int d = 0; d < 6; ++d) {
        int qi = q[d][0], qj = q[d][1], qk = q[d][2];
        if (qi < 0 || qi > n - 1 || qj < 0 || qj > n - 1 || qk < 0 || qk > n - 1) {
            d32 -= 1.0f;
            d64 -= 1.0;
            continue;
        }
        long long qc = D.c_begin + ((long long)qi * n + qj) * n + qk;
        uint8_t tq = S.flags[qc];
        if (tq == ARIEL_SOLID) {
            d32 -= 1.0f;
            d64 -= 1.0;
        } else if (tq == ARIEL_FLUID) {
            m |= (uint8_t)(1u << d);
        } else if (D.subcell) {
            // ADiag (solver.inl:95-96): diag -= L_q / min(1e-6, L_c)
            d32 -= S.L[qc] / gmin(1.0e-6f, Lc);
            d64 -= (double)S.L[qc] / (double)gmin(1.0e-6f, Lc);
        }
    }
    A.mask[c] = m;
    int one = 0;
    if (A.mode == kRef32) {
        // BuildPreconditioner (solver.inl:113-128) with its neighbour terms zero
        float e = d32 - (0.0f * 0.0f) - (0.0f * 0.0f) - (0.0f * 0.0f);
        float pc = 0.0f;
        if (d32 > 0) {
            if (e < 0.25f * d32) e = d32;
            pc = 1.0f / sqrtf(e);
        }
        A.diag[c] = (double)d32;
        A.pc32[c] = pc;
        A.pc64[c] = (double)pc;
        one = pc == 1.0f;
    } else {
        double pc = d64 > 0 ? 1.0 / sqrt(d64) : 0.0;
        A.diag[c] = d64;
        A.pc64[c] = pc;
        A.pc32[c] = (float)pc;
        one = pc == 1.0;
    }
    if (one) atomicAdd(&A.sc[s].ones, 1);
}

// FLUID list, plus one 16-byte record per entry holding everything the solve needs about the
// cell besides its vectors: index, neighbour mask and ADiag (fp32 bits for the fp32 modes, fp64
// bits otherwise), so that a single load starts a cell's update.
__global__ void k_fl_write(PcgArgs A, const uint32_t* pred, const uint32_t* scan) {
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.S.nc) return;
    if (!pred[c]) return;
    const uint32_t t = scan[c];
    const_cast<uint32_t*>(A.fl)[t] = (uint32_t)c;
    uint4 r;
    r.x = (uint32_t)c;
    r.y = (uint32_t)A.mask[c];
    if (A.mode == kFp64) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(A.diag[c]);
        r.z = (uint32_t)b;
        r.w = (uint32_t)(b >> 32);
    } else {
        r.z = __float_as_uint((float)A.diag[c]);
        r.w = 0u;
    }
    A.rec[t] = r;
}

__global__ void k_pcg_tables(PcgArgs A, const uint32_t* scan) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int k = A.S.k;
    long long* flp = const_cast<long long*>(A.fl_pref);
    long long* chp = const_cast<long long*>(A.ch_pref);
    long long acc = 0;
    int any_ordered = 0;
    for (int s = 0; s <= k; ++s) flp[s] = scan[A.S.c_pref[s]];
    for (int s = 0; s < k; ++s) {
        chp[s] = acc;
        long long nf = flp[s + 1] - flp[s];
        const int cs = chunk_size(nf);
        acc += (nf + cs - 1) / cs;
        PcgScene& P = A.sc[s];
        P.nf = (int)nf;
        P.csize = cs;
        P.ordered = nf > 0 && (A.precond == ARIEL_PRECOND_MIC0 || P.ones > 0);
        any_ordered |= P.ordered;
    }
    chp[k] = acc;
    A.ctl->all_done = 0;
    A.ctl->all_inner_done = 0;
    A.ctl->any_ordered = any_ordered;
}

// Data written by other blocks is read only after a grid barrier (whose acquire makes ordinary
// loads observe it) or, inside an ordered sweep, through L2 after the producer's release flag.
template <class T>
__device__ __forceinline__ T ldv(const T* p) {
    return *p;
}

// ------------------------------------------------------------------------------------------
// Ordered wavefront sweeps over bricks (all blocks of the persistent kernel).
//
// The ordered preconditioners (MIC(0), and the reference's PRef == 1 path) need every cell's
// lower neighbours (i-1, j-1, k-1) before the cell itself (upper ones for the backward
// sweep).  Each scene's grid is cut into bx*by*bz bricks; a brick depends only on its three
// upstream bricks, so the bricks of all scenes are listed by level I+J+K and block b takes list
// positions b, b + G, b + 2G, ...  A brick waits (bounded) for its upstream bricks' progress
// flags, loads its cells and one face of halo per upstream brick into shared memory, sweeps its
// own i+j+k levels there, writes the results and publishes its flag.  Every wait points to an
// earlier list position and every block walks its positions in order, so with all blocks
// resident (cooperative launch) the sweep always completes.  A cell's arithmetic is the same
// for any brick shape or grid size.
// ------------------------------------------------------------------------------------------
enum BrickKind { kBuild = 0, kFwd = 1, kBwd = 2 };

struct BrickSmem {
    double* box0;      // [kBrickMaxExt] apply: q (forward) or z (backward) as T; build: pc (double)
    double* box1;      // [kBrickMaxExt] apply: pc as T
    double* inb;       // [kBrickMaxCells] interior input: r (forward), q (backward) as T; diag (build)
    int* lstart;       // [kBrickMaxLevels + 1] first table entry of each level
    uint16_t* ltab;    // [kBrickMaxCells] packed x << 11 | y << 6 | z, sorted by level x+y+z
    uint8_t* mbox;     // [kBrickMaxExt] FLUID-neighbour mask | 64 when the cell is FLUID
};

__device__ BrickSmem brick_smem(unsigned char* dyn) {
    BrickSmem B;
    B.box0 = reinterpret_cast<double*>(dyn);
    B.box1 = B.box0 + kBrickMaxExt;
    B.inb = B.box1 + kBrickMaxExt;
    B.lstart = reinterpret_cast<int*>(B.inb + kBrickMaxCells);
    B.ltab = reinterpret_cast<uint16_t*>(B.lstart + kBrickMaxLevels + 1);
    B.mbox = reinterpret_cast<uint8_t*>(B.ltab + kBrickMaxCells);
    return B;
}

// The brick's cells grouped by level (built once per launch).
__device__ void brick_levels(const PcgArgs& A, BrickSmem& B) {
    const int bx = A.bx, by = A.by, bz = A.bz, nl = bx + by + bz - 2, ncell = bx * by * bz;
    int* cur = reinterpret_cast<int*>(B.box0);
    for (int l = threadIdx.x; l <= nl; l += blockDim.x) B.lstart[l] = 0;
    __syncthreads();
    for (int li = threadIdx.x; li < ncell; li += blockDim.x) {
        const int x = li / (by * bz), y = (li / bz) % by, z = li % bz;
        atomicAdd(&B.lstart[x + y + z + 1], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int l = 1; l <= nl; ++l) B.lstart[l] += B.lstart[l - 1];
    __syncthreads();
    for (int l = threadIdx.x; l < nl; l += blockDim.x) cur[l] = B.lstart[l];
    __syncthreads();
    for (int li = threadIdx.x; li < ncell; li += blockDim.x) {
        const int x = li / (by * bz), y = (li / bz) % by, z = li % bz;
        const int pos = atomicAdd(&cur[x + y + z], 1);
        B.ltab[pos] = (uint16_t)((x << 11) | (y << 6) | z);
    }
    __syncthreads();
}

// Thread 0: bounded wait until *f >= val.
__device__ bool brick_wait(const unsigned* f, unsigned val, Barrier* bar, int* dev_error, unsigned long long tmo) {
    const unsigned long long t0 = gtimer();
    while (ld_acquire_u32(f) < val) {
        if (*(volatile int*)&bar->error) return false;
        if (gtimer() - t0 > tmo) {
            atomicExch(&bar->error, 1);
            if (dev_error) atomicExch(dev_error, 1);
            return false;
        }
        __nanosleep(32);
    }
    return true;
}

// One sweep over the bricks of every ordered scene (apply sweeps skip scenes whose inner solve
// is done).  KIND kBuild: the preconditioner values (pc64 / pc32); kFwd: out = q from in = r;
// kBwd: out = z from in = q.  `val` is this sweep's flag value (the forward sweep's is val - 1
// for kBwd).  Returns false when a wait gave up.
template <int KIND, class T>
__device__ bool brick_sweep(const PcgArgs& A, const BrickSmem& B, unsigned val, const T* in, T* out, const T* pcv,
                            unsigned long long tmo) {
    const DevState& S = A.S;
    const bool mic = A.precond == ARIEL_PRECOND_MIC0;
    const bool ref32 = A.mode == kRef32;
    const int bx = A.bx, by = A.by, bz = A.bz;
    const int ey = by + 1, ez = bz + 1;
    const int sx = ey * ez, sy = ez;
    const int lo = KIND == kBwd ? 0 : 1;  // halo below (build, forward) or above (backward)
    const int nl = bx + by + bz - 2, ncell = bx * by * bz;
    const int nb = A.nbricks;
    T* const vbox = reinterpret_cast<T*>(B.box0);
    T* const pbox = reinterpret_cast<T*>(B.box1);
    double* const cbox = B.box0;
    T* const vin = reinterpret_cast<T*>(B.inb);
    double* const din = B.inb;
    const int nfx = by * bz, nfy = bx * bz, nfz = bx * by, nh = nfx + nfy + nfz;
    const int hx = KIND == kBwd ? bx : -1, hy = KIND == kBwd ? by : -1, hz = KIND == kBwd ? bz : -1;
    auto bidx = [&](int x, int y, int z) { return ((x + lo) * ey + (y + lo)) * ez + (z + lo); };
    __shared__ int s_ok;
    for (int p = blockIdx.x; p < nb; p += gridDim.x) {
        const int pp = KIND == kBwd ? nb - 1 - p : p;
        const int4 br = A.bricks[pp];
        const int s = br.x;
        if (!ldv(&A.sc[s].ordered)) continue;
        if (KIND != kBuild && ldv(&A.sc[s].inner_done)) continue;
        const SceneDev& D = S.scenes[s];
        const int n = D.n;
        const int I0 = br.y * bx, J0 = br.z * by, K0 = br.w * bz;
        const int nbJ = (n + by - 1) / by, nbK = (n + bz - 1) / bz, nbI = (n + bx - 1) / bx;
        unsigned* const fb = A.bflag + A.brick_base[s];
        auto flag_of = [&](int I, int J, int K) { return fb + ((long long)I * nbJ + J) * nbK + K; };
        auto inside = [&](int i, int j, int k) { return i >= 0 && j >= 0 && k >= 0 && i < n && j < n && k < n; };
        auto cid = [&](int i, int j, int k) { return D.c_begin + ((long long)i * n + j) * n + k; };
        auto halo_cell = [&](int h, int& x, int& y, int& z) -> bool {
            if (h < nfx) {
                x = hx;
                y = h / bz;
                z = h % bz;
            } else if (h < nfx + nfy) {
                h -= nfx;
                x = h / bz;
                y = hy;
                z = h % bz;
            } else {
                h -= nfx + nfy;
                x = h / by;
                y = h % by;
                z = hz;
            }
            return inside(I0 + x, J0 + y, K0 + z);
        };
        // 1. data that does not change during the sweep: masks, r (forward), pc, diagonal
        for (int li = threadIdx.x; li < ncell; li += blockDim.x) {
            const int x = li / (by * bz), y = (li / bz) % by, z = li % bz;
            const int bi = bidx(x, y, z);
            uint8_t m = 0;
            if (inside(I0 + x, J0 + y, K0 + z)) {
                const long long c = cid(I0 + x, J0 + y, K0 + z);
                if (S.flags[c] == ARIEL_FLUID) {
                    m = (uint8_t)(A.mask[c] | 64);
                    if (KIND == kBuild) {
                        din[li] = A.diag[c];
                    } else {
                        pbox[bi] = pcv[c];
                        if (KIND == kFwd) vin[li] = in[c];
                    }
                }
            }
            B.mbox[bi] = m;
        }
        for (int h = threadIdx.x; h < nh; h += blockDim.x) {
            int x, y, z;
            const bool ok = halo_cell(h, x, y, z);
            const int bi = bidx(x, y, z);
            uint8_t m = 0;
            if (ok) {
                const long long c = cid(I0 + x, J0 + y, K0 + z);
                if (S.flags[c] == ARIEL_FLUID) {
                    m = (uint8_t)(A.mask[c] | 64);
                    if (KIND == kFwd) pbox[bi] = pcv[c];
                }
            }
            B.mbox[bi] = m;
        }
        // 2. upstream bricks (and, backward, this brick's forward sweep)
        if (threadIdx.x == 0) {
            bool ok = true;
            if (KIND == kBwd) {
                ok = brick_wait(flag_of(br.y, br.z, br.w), val - 1, A.bar, S.dev_error, tmo);
                if (ok && br.y + 1 < nbI) ok = brick_wait(flag_of(br.y + 1, br.z, br.w), val, A.bar, S.dev_error, tmo);
                if (ok && br.z + 1 < nbJ) ok = brick_wait(flag_of(br.y, br.z + 1, br.w), val, A.bar, S.dev_error, tmo);
                if (ok && br.w + 1 < nbK) ok = brick_wait(flag_of(br.y, br.z, br.w + 1), val, A.bar, S.dev_error, tmo);
            } else {
                if (br.y > 0) ok = brick_wait(flag_of(br.y - 1, br.z, br.w), val, A.bar, S.dev_error, tmo);
                if (ok && br.z > 0) ok = brick_wait(flag_of(br.y, br.z - 1, br.w), val, A.bar, S.dev_error, tmo);
                if (ok && br.w > 0) ok = brick_wait(flag_of(br.y, br.z, br.w - 1), val, A.bar, S.dev_error, tmo);
            }
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) return false;
        // 3. what the upstream bricks produced, read through L2
        if (KIND == kBwd)
            for (int li = threadIdx.x; li < ncell; li += blockDim.x) {
                const int x = li / (by * bz), y = (li / bz) % by, z = li % bz;
                if (B.mbox[bidx(x, y, z)] & 64) vin[li] = __ldcg(in + cid(I0 + x, J0 + y, K0 + z));
            }
        for (int h = threadIdx.x; h < nh; h += blockDim.x) {
            int x, y, z;
            if (!halo_cell(h, x, y, z)) continue;
            const int bi = bidx(x, y, z);
            if (!(B.mbox[bi] & 64)) continue;
            const long long c = cid(I0 + x, J0 + y, K0 + z);
            if (KIND == kBuild)
                cbox[bi] = ref32 ? (double)__ldcg(A.pc32 + c) : __ldcg(A.pc64 + c);
            else
                vbox[bi] = __ldcg(out + c);
        }
        __syncthreads();
        // 4. the brick's own levels (highest first for the backward sweep)
        for (int lv = 0; lv < nl; ++lv) {
            const int l = KIND == kBwd ? nl - 1 - lv : lv;
            for (int e = B.lstart[l] + threadIdx.x; e < B.lstart[l + 1]; e += blockDim.x) {
                const unsigned pk = B.ltab[e];
                const int x = (int)(pk >> 11), y = (int)((pk >> 6) & 31u), z = (int)(pk & 63u);
                const int bi = bidx(x, y, z);
                const unsigned m = B.mbox[bi];
                if (!(m & 64u)) continue;
                const int li = (x * by + y) * bz + z;
                if (KIND == kFwd) {
                    // q = (r - sum_lower a pc_q q_q) pc
                    T t = vin[li];
                    const int offs[3] = {-sx, -sy, -1};
                    const unsigned bits[3] = {1u, 4u, 16u};
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        if (!(m & bits[d])) continue;
                        const T pq = pbox[bi + offs[d]], qq = vbox[bi + offs[d]];
                        if (mic)
                            t -= (T)-1.0 * pq * qq;
                        else if (pq == (T)1.0 && qq == (T)1.0)
                            t -= (T)-1.0;  // ARef*PRef(P)*PRef(Q) = -1
                    }
                    vbox[bi] = t * pbox[bi];
                } else if (KIND == kBwd) {
                    // z = (q - sum_upper a pc z_q) pc
                    const T pcc = pbox[bi];
                    T t = vin[li];
                    const int offs[3] = {sx, sy, 1};
                    const unsigned bits[3] = {2u, 8u, 32u};
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        if (!(m & bits[d])) continue;
                        const T zq = vbox[bi + offs[d]];
                        if (mic)
                            t -= (T)-1.0 * pcc * zq;
                        else if (pcc == (T)1.0 && zq == (T)1.0)
                            t -= (T)-1.0;
                    }
                    vbox[bi] = t * pcc;
                } else if (mic) {
                    // MIC(0) (Bridson): e = diag - sum_lower [(a p)^2 + tau a (sum of the lower
                    // neighbour's other upper couplings) p^2], safety sigma
                    const double tau = A.tau, sigma = A.sigma, ap = -1.0;
                    const double dg = din[li];
                    double e = dg;
                    const int offs[3] = {-sx, -sy, -1};
                    const unsigned bits[3] = {1u, 4u, 16u};
                    const unsigned oa[3] = {8u, 2u, 2u}, ob[3] = {32u, 32u, 8u};
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        if (!(m & bits[d])) continue;
                        const double pq = cbox[bi + offs[d]];
                        const unsigned mq = B.mbox[bi + offs[d]];
                        const double oth = ((mq & oa[d]) ? -1.0 : 0.0) + ((mq & ob[d]) ? -1.0 : 0.0);
                        e -= (ap * pq) * (ap * pq) + tau * (ap * oth * pq * pq);
                    }
                    if (e < sigma * dg) e = dg;
                    cbox[bi] = e > 0 ? 1.0 / sqrt(e) : 0.0;
                } else if (ref32) {
                    // BuildPreconditioner in fp32 (solver.inl:104-135)
                    auto term = [&](unsigned bit, int off) -> float {
                        return ((m & bit) && (float)cbox[bi + off] == 1.0f) ? -1.0f : 0.0f;
                    };
                    const float left = term(1u, -sx), bottom = term(4u, -sy), back = term(16u, -1);
                    const float diag = (float)din[li];
                    float e = diag - (left * left) - (bottom * bottom) - (back * back);
                    float pc = 0.0f;
                    if (diag > 0) {
                        if (e < 0.25f * diag) e = diag;
                        pc = 1.0f / sqrtf(e);
                    }
                    cbox[bi] = (double)pc;
                } else {
                    auto term = [&](unsigned bit, int off) -> double {
                        return ((m & bit) && cbox[bi + off] == 1.0) ? -1.0 : 0.0;
                    };
                    const double left = term(1u, -sx), bottom = term(4u, -sy), back = term(16u, -1);
                    const double dg = din[li];
                    double e = dg - left * left - bottom * bottom - back * back;
                    double pc = 0.0;
                    if (dg > 0) {
                        if (e < 0.25 * dg) e = dg;
                        pc = 1.0 / sqrt(e);
                    }
                    cbox[bi] = pc;
                }
            }
            __syncthreads();
        }
        // 5. results out, then publish the brick
        for (int li = threadIdx.x; li < ncell; li += blockDim.x) {
            const int x = li / (by * bz), y = (li / bz) % by, z = li % bz;
            const int bi = bidx(x, y, z);
            if (!(B.mbox[bi] & 64)) continue;
            const long long c = cid(I0 + x, J0 + y, K0 + z);
            if (KIND == kBuild) {
                const double pc = cbox[bi];
                A.pc64[c] = pc;
                A.pc32[c] = (float)pc;
            } else {
                out[c] = vbox[bi];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            st_release_u32(flag_of(br.y, br.z, br.w), val);
        }
    }
    return true;
}

// ------------------------------------------------------------------------------------------
// Operators.
// ------------------------------------------------------------------------------------------
// ComputeAx for one FLUID cell with the reference's exact expression (solver.inl:196-230).
// `sv(q)` yields the vector value at FLUID cell q; xc is the value at c.
template <class SV>
__device__ __forceinline__ float ax_ref32(const DevState& S, const SceneDev& D, long long c, float xc, SV&& sv) {
    const int n = D.n;
    int i, j, k;
    cell_ijk(D, c - D.c_begin, i, j, k);
    const float Lc = S.L[c];
    auto xref = [&](int pi, int pj, int pk) -> float {
        int a = min(max(0, pi), n - 1), b = min(max(0, pj), n - 1), cc = min(max(0, pk), n - 1);
        long long q = D.c_begin + ((long long)a * n + b) * n + cc;
        uint8_t t = S.flags[q];
        if (t == ARIEL_FLUID) return q == c ? xc : sv(q);
        if (t == ARIEL_SOLID) return xc;
        if (D.subcell) return S.L[q] / gmin(1.0e-6f, Lc) * xc;
        return 0.0f;
    };
    float result = (6.0f * xc - xref(i + 1, j, k) - xref(i - 1, j, k) - xref(i, j + 1, k) - xref(i, j - 1, k) -
                    xref(i, j, k + 1) - xref(i, j, k - 1)) /
                   D.ax_h;
    return result;
}

__device__ __forceinline__ long long nb_off(int d, int n) {
    const long long nn = (long long)n * n;
    switch (d) {
        case 0: return -nn;
        case 1: return nn;
        case 2: return -(long long)n;
        case 3: return (long long)n;
        case 4: return -1;
        default: return 1;
    }
}

// Diagonal form (FP64 and the MIXED fp32 inner operator): (diag*x_c - sum_FLUID x_q) / h.
template <class T, class SV>
__device__ __forceinline__ T ax_diag(const PcgArgs& A, const SceneDev& D, long long c, T xc, SV&& sv) {
    const uint8_t m = A.mask[c];
    T acc = (T)A.diag[c] * xc;
#pragma unroll
    for (int d = 0; d < 6; ++d)
        if (m & (1u << d)) acc -= sv(c + nb_off(d, D.n));
    const T scale = (T)(1.0 / (double)D.ax_h);
    return acc * scale;
}

// ------------------------------------------------------------------------------------------
// The persistent solve.
// ------------------------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(kPcgThreads, 2) k_pcg(PcgArgs A) {
    using T = typename VT<MODE>::T;
    const DevState& S = A.S;
    const int k = S.k;
    __shared__ long long fl_s[kMaxScenes + 1], ch_s[kMaxScenes + 1];
    __shared__ uint16_t csz_s[kMaxScenes];
    for (int i = threadIdx.x; i <= k; i += blockDim.x) {
        fl_s[i] = A.fl_pref[i];
        ch_s[i] = A.ch_pref[i];
        if (i < k) csz_s[i] = (uint16_t)A.sc[i].csize;
    }
    __syncthreads();
    const long long nch = ch_s[k];
    const long long MC = A.max_chunks;
    double* part0 = A.partial;
    double* part1 = A.partial + MC;
    PcgScene* SC = A.sc;
    T* r = (T*)A.r;
    T* z = (T*)A.z;
    T* q = (T*)A.q;
    T* const sb0 = (T*)A.s0;
    T* const sb1 = (T*)A.s1;
    T* ordq = (T*)A.ordq;
    const T* pcv = MODE == kFp64 ? (const T*)(const void*)A.pc64 : (const T*)(const void*)A.pc32;
    // x of the working solve: P (REF32), P64 (FP64), d32 (MIXED inner correction)
    T* x = MODE == kRef32 ? (T*)(void*)S.P : (MODE == kFp64 ? (T*)(void*)S.P64 : (T*)(void*)A.d32);
    const bool any_ordered = ldv(&A.ctl->any_ordered) != 0;
    if (A.fast && !any_ordered) return;  // solved by k_pcg_fast
    const unsigned long long tmo = A.timeout_ns;
    __shared__ int s_active;

    auto chunk_range = [&](long long ch, int& s, long long& t0, long long& t1) {
        s = find_scene(ch_s, k, ch);
        const long long cs = csz_s[s];
        t0 = fl_s[s] + (ch - ch_s[s]) * cs;
        t1 = min(t0 + cs, fl_s[s + 1]);
    };
    auto write_part = [&](long long ch, double a, double b) {
        block_sum2(a, b);
        if (threadIdx.x == 0) {
            part0[ch] = a;
            part1[ch] = b;
        }
    };
    // elementwise preconditioner of the reference ((r*pc)*pc) for non-ordered scenes
    auto precond_elem = [&](long long c, T rv) -> T { return (rv * ldv(pcv + c)) * ldv(pcv + c); };

    // ---- Phase 0: ordered preconditioner build (brick wavefront) ---------------------------
    extern __shared__ __align__(16) unsigned char kdyn[];
    BrickSmem BS = brick_smem(kdyn);
    unsigned bseq = 0;  // progress-flag value of the latest sweep (same in every block)
    if (any_ordered) {
        brick_levels(A, BS);
        if (!brick_sweep<kBuild, double>(A, BS, ++bseq, nullptr, nullptr, nullptr, tmo)) return;
        if (!grid_barrier(A.bar, S.dev_error, tmo, NoLeader{})) return;
    }

    int outer = 0;
    while (true) {
        // ---- Phase R: residual r = b - A x and |b|^2 ----------------------------------------
        for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
            int s;
            long long t0, t1;
            chunk_range(ch, s, t0, t1);
            const SceneDev& D = S.scenes[s];
            double a0 = 0.0, a1 = 0.0;
            if (!ldv(&SC[s].done)) {
                for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                    long long c = A.fl[t];
                    double bv = (double)S.D[c];
                    if (MODE == kRef32) {
                        float xc = ldv(S.P + c);
                        float ax = ax_ref32(S, D, c, xc, [&](long long qq) { return ldv(S.P + qq); });
                        float rv = S.D[c] + (-1.0f) * ax;  // Op(A, D, Z, R, -1)
                        r[c] = (T)rv;
                        a0 += (double)rv * (double)rv;
                    } else {
                        double xc = ldv(S.P64 + c);
                        double ax = ax_diag<double>(A, D, c, xc, [&](long long qq) { return ldv(S.P64 + qq); });
                        double rv = bv - ax;
                        if (MODE == kMixed)
                            A.r64[c] = rv;
                        else
                            r[c] = (T)rv;
                        a0 += rv * rv;
                    }
                    a1 += bv * bv;
                }
            }
            write_part(ch, a0, a1);
        }
        bool ok = grid_barrier(A.bar, S.dev_error, tmo, [&]() {
            if (threadIdx.x == 0) s_active = 0;
            __syncthreads();
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            for (int s = wid; s < k; s += blockDim.x / 32) {
                double rr = scene_sum(part0, ch_s[s], ch_s[s + 1]);
                double bb = scene_sum(part1, ch_s[s], ch_s[s + 1]);
                if (lane == 0) {
                    PcgScene P = load_sc(SC + s);
                    if (!P.done) {
                        const int n = S.scenes[s].n;
                        if (outer == 0) P.bb = bb;
                        P.rr_out = rr;
                        if (MODE == kMixed) P.outer += 1;
                        double lim2 = A.tol * A.tol * P.bb;
                        double abs_eps = (double)(1.0e-2f * (float)(n * n * n));
                        bool conv = false;
                        if (A.stop_rule == ARIEL_STOP_REL)
                            conv = rr <= lim2;
                        else if (MODE == kMixed)
                            conv = outer > 0 && rr <= abs_eps;
                        if (P.nf == 0) conv = true;
                        int cap = A.max_iters > 0 ? A.max_iters : n * n * n;
                        if (conv) {
                            P.done = 1;
                            P.converged = 1;
                        } else if (MODE == kMixed && (P.outer > A.max_outer || P.iters >= cap)) {
                            P.done = 1;
                            P.converged = 0;
                        }
                        if (!P.done) {
                            P.inner_done = 0;
                            P.rr = rr;
                            if (MODE == kMixed) {
                                // the correction solve stops at the final tolerance itself (its
                                // fp32 residual); the true fp64 residual then decides whether
                                // another sweep is needed
                                double t1 = A.inner_tol * A.inner_tol * rr;
                                double t2 = A.stop_rule == ARIEL_STOP_REL ? lim2 : 0.0;
                                P.target = t1 > t2 ? t1 : t2;
                            } else {
                                P.target = A.stop_rule == ARIEL_STOP_REL ? lim2 : abs_eps;
                            }
                            atomicAdd(&s_active, 1);
                        } else {
                            P.inner_done = 1;
                        }
                        SC[s] = P;
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                A.ctl->all_done = s_active == 0;
                A.ctl->all_inner_done = s_active == 0;
            }
        });
        if (!ok) return;
        if (ldv(&A.ctl->all_done)) break;

        if (MODE != kRef32 && !any_ordered) {
            // ---- single-reduction PCG (Chronopoulos & Gear, 1989): one grid barrier per
            // iteration.  Iteration i reads r_i = rb[i&1], w_i = wb[i&1], s_{i-1} = sb[(i+1)&1],
            // u_i, p_{i-1}, x_i and writes s_i = w_i + beta s_{i-1} (sb[i&1]), p_i = u_i + beta
            // p_{i-1}, x_{i+1} = x_i + alpha p_i, r_{i+1} = r_i - alpha s_i (rb[(i+1)&1]),
            // u_{i+1} = M r_{i+1}, w_{i+1} = A u_{i+1} (wb[(i+1)&1]).  The neighbour values of
            // u_{i+1} that A needs are recomputed from the same old arrays, bit-identically to
            // what their owners write.
            T* const rb0 = r;
            T* const rb1 = ordq;
            T* const wb0 = z;
            T* const wb1 = q;
            T* u = (T*)A.u;
            T* pv = (T*)A.p;
            double* part2 = A.partial + 2 * MC;
            auto precond = [&](long long c, T rv) -> T { return (rv * ldv(pcv + c)) * ldv(pcv + c); };
            auto write_part3 = [&](long long ch, double a, double b, double c3) {
                double z3 = 0.0;
                block_sum2(a, b);
                block_sum2(c3, z3);
                if (threadIdx.x == 0) {
                    part0[ch] = a;
                    part1[ch] = b;
                    part2[ch] = c3;
                }
            };
            // Phase I1: r_0 (MIXED: from r64), u_0 = M r_0, w_0 = A u_0, (r,u), (w,u), (r,r)
            for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
                int s;
                long long t0, t1;
                chunk_range(ch, s, t0, t1);
                const SceneDev& D = S.scenes[s];
                double g0 = 0.0, d0 = 0.0, q0 = 0.0;
                if (!ldv(&SC[s].inner_done)) {
                    auto r0 = [&](long long qq) -> T { return MODE == kMixed ? (T)A.r64[qq] : ldv(r + qq); };
                    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                        long long c = A.fl[t];
                        T rv = r0(c);
                        T uv = precond(c, rv);
                        T wv = ax_diag<T>(A, D, c, uv, [&](long long qq) { return precond(qq, r0(qq)); });
                        if (MODE == kMixed) {
                            rb0[c] = rv;
                            x[c] = (T)0;
                        }
                        u[c] = uv;
                        wb0[c] = wv;
                        g0 += (double)rv * (double)uv;
                        d0 += (double)wv * (double)uv;
                        q0 += (double)rv * (double)rv;
                    }
                }
                write_part3(ch, g0, d0, q0);
            }
            ok = grid_barrier(A.bar, S.dev_error, tmo, [&]() {
                const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
                for (int s = wid; s < k; s += blockDim.x / 32) {
                    double g = scene_sum(part0, ch_s[s], ch_s[s + 1]);
                    double d = scene_sum(part1, ch_s[s], ch_s[s + 1]);
                    if (lane == 0) {
                        PcgScene P = load_sc(SC + s);
                        if (!P.inner_done) {
                            P.rho = g;
                            P.alpha = d != 0.0 ? g / d : 0.0;
                            P.beta = 0.0;
                            SC[s] = P;
                        }
                    }
                }
            });
            if (!ok) return;
            for (int it = 0;; ++it) {
                const int cur = it & 1, nxt = cur ^ 1;
                for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
                    int s;
                    long long t0, t1;
                    chunk_range(ch, s, t0, t1);
                    const SceneDev& D = S.scenes[s];
                    double g1 = 0.0, d1 = 0.0, q1 = 0.0;
                    if (!ldv(&SC[s].inner_done)) {
                        const T al = (T)ldv(&SC[s].alpha);
                        const T bt = (T)ldv(&SC[s].beta);
                        const T* rc = cur ? rb1 : rb0;
                        const T* wc = cur ? wb1 : wb0;
                        const T* sp = nxt ? sb1 : sb0;
                        T* sw = cur ? sb1 : sb0;
                        T* rw = nxt ? rb1 : rb0;
                        T* ww = nxt ? wb1 : wb0;
                        // s_i at any FLUID cell, and u_{i+1} = M (r_i - alpha s_i) there
                        auto s_i = [&](long long qq) -> T { return it == 0 ? ldv(wc + qq) : ldv(wc + qq) + bt * ldv(sp + qq); };
                        auto u_n = [&](long long qq) -> T { return precond(qq, ldv(rc + qq) - al * s_i(qq)); };
                        for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                            long long c = A.fl[t];
                            T sv = s_i(c);
                            T pvv = it == 0 ? ldv(u + c) : ldv(u + c) + bt * ldv(pv + c);
                            T xv = ldv(x + c) + al * pvv;
                            T rn = ldv(rc + c) - al * sv;
                            T un = precond(c, rn);
                            T wn = ax_diag<T>(A, D, c, un, u_n);
                            sw[c] = sv;
                            pv[c] = pvv;
                            x[c] = xv;
                            rw[c] = rn;
                            u[c] = un;
                            ww[c] = wn;
                            g1 += (double)rn * (double)un;
                            d1 += (double)wn * (double)un;
                            q1 += (double)rn * (double)rn;
                        }
                    }
                    write_part3(ch, g1, d1, q1);
                }
                ok = grid_barrier(A.bar, S.dev_error, tmo, [&]() {
                    if (threadIdx.x == 0) s_active = 0;
                    __syncthreads();
                    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
                    for (int s = wid; s < k; s += blockDim.x / 32) {
                        double g = scene_sum(part0, ch_s[s], ch_s[s + 1]);
                        double d = scene_sum(part1, ch_s[s], ch_s[s + 1]);
                        double rr = scene_sum(part2, ch_s[s], ch_s[s + 1]);
                        if (lane == 0) {
                            PcgScene P = load_sc(SC + s);
                            if (!P.inner_done) {
                                const int n = S.scenes[s].n;
                                P.iters += 1;
                                P.rr = rr;
                                const int cap = A.max_iters > 0 ? A.max_iters : n * n * n;
                                bool conv = rr <= P.target;
                                if (conv || P.iters >= cap) {
                                    P.inner_done = 1;
                                    if (MODE != kMixed) {
                                        P.done = 1;
                                        P.converged = conv;
                                    }
                                } else {
                                    double beta = P.rho != 0.0 ? g / P.rho : 0.0;
                                    double den = d - (P.alpha != 0.0 ? beta * g / P.alpha : 0.0);
                                    P.beta = beta;
                                    P.alpha = den != 0.0 ? g / den : 0.0;
                                    P.rho = g;
                                    atomicAdd(&s_active, 1);
                                }
                                SC[s] = P;
                            }
                        }
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) A.ctl->all_inner_done = s_active == 0;
                });
                if (!ok) return;
                if (ldv(&A.ctl->all_inner_done)) break;
            }
            // the solution of this (inner) solve is x; MIXED folds it into x64 below
            if (MODE != kMixed) break;
            for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
                int s;
                long long t0, t1;
                chunk_range(ch, s, t0, t1);
                if (ldv(&SC[s].done)) continue;
                for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                    long long c = A.fl[t];
                    S.P64[c] = ldv(S.P64 + c) + (double)ldv(x + c);
                }
            }
            if (!grid_barrier(A.bar, S.dev_error, tmo, NoLeader{})) return;
            ++outer;
            continue;
        }

        // ---- Phase I: z = M r, s = z, rho = z.r (MIXED: r32 = r64, d = 0) ------------------
        for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
            int s;
            long long t0, t1;
            chunk_range(ch, s, t0, t1);
            const bool active = !ldv(&SC[s].inner_done);
            const bool ord = ldv(&SC[s].ordered) != 0;
            double a0 = 0.0;
            if (active) {
                for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                    long long c = A.fl[t];
                    T rv;
                    if (MODE == kMixed) {
                        rv = (T)A.r64[c];
                        r[c] = rv;
                        x[c] = (T)0;
                    } else {
                        rv = ldv(r + c);
                    }
                    if (!ord) {
                        T zv = precond_elem(c, rv);
                        z[c] = zv;
                        sb0[c] = zv;
                        a0 += (double)zv * (double)rv;
                    }
                }
            }
            if (!ord) write_part(ch, a0, 0.0);
        }
        if (any_ordered) {
            // z = M^-1 r for the ordered scenes: forward then backward brick sweeps, then z.r
            // per chunk like every other scene
            if (!grid_barrier(A.bar, S.dev_error, tmo, NoLeader{})) return;
            ++bseq;
            if (!brick_sweep<kFwd, T>(A, BS, bseq, r, ordq, pcv, tmo)) return;
            ++bseq;
            if (!brick_sweep<kBwd, T>(A, BS, bseq, ordq, z, pcv, tmo)) return;
            if (!grid_barrier(A.bar, S.dev_error, tmo, NoLeader{})) return;
            for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
                int s;
                long long t0, t1;
                chunk_range(ch, s, t0, t1);
                if (!ldv(&SC[s].ordered)) continue;
                double a0 = 0.0;
                if (!ldv(&SC[s].inner_done)) {
                    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                        long long c = A.fl[t];
                        T zv = ldv(z + c);
                        sb0[c] = zv;
                        a0 += (double)zv * (double)ldv(r + c);
                    }
                }
                write_part(ch, a0, 0.0);
            }
        }
        ok = grid_barrier(A.bar, S.dev_error, tmo, [&]() {
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            for (int s = wid; s < k; s += blockDim.x / 32) {
                double rho = scene_sum(part0, ch_s[s], ch_s[s + 1]);
                if (lane == 0) {
                    PcgScene P = load_sc(SC + s);
                    if (!P.inner_done) {
                        P.rho = rho;
                        P.rho32 = (float)rho;
                        SC[s] = P;
                    }
                }
            }
        });
        if (!ok) return;

        // ---- CG iterations -------------------------------------------------------------------
        for (int it = 0;; ++it) {
            T* s_cur = (it & 1) ? sb1 : sb0;
            T* s_prev = (it & 1) ? sb0 : sb1;
            // Phase A: s = z + beta s (it > 0), q = A s, s.q
            for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
                int s;
                long long t0, t1;
                chunk_range(ch, s, t0, t1);
                const SceneDev& D = S.scenes[s];
                double a0 = 0.0;
                if (!ldv(&SC[s].inner_done)) {
                    const double beta = ldv(&SC[s].beta);
                    const float beta32 = ldv(&SC[s].beta32);
                    const T bt = MODE == kRef32 ? (T)beta32 : (T)beta;
                    auto sval = [&](long long qq) -> T {
                        if (it == 0) return ldv(s_cur + qq);
                        return ldv(z + qq) + bt * ldv(s_prev + qq);  // Op(A, Z, S, S, beta)
                    };
                    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                        long long c = A.fl[t];
                        T sc_ = sval(c);
                        if (it > 0) s_cur[c] = sc_;
                        T qv;
                        if (MODE == kRef32)
                            qv = ax_ref32(S, D, c, sc_, sval);
                        else
                            qv = ax_diag<T>(A, D, c, sc_, sval);
                        q[c] = qv;
                        a0 += (double)sc_ * (double)qv;
                    }
                }
                write_part(ch, a0, 0.0);
            }
            ok = grid_barrier(A.bar, S.dev_error, tmo, [&]() {
                const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
                for (int s = wid; s < k; s += blockDim.x / 32) {
                    double sq = scene_sum(part0, ch_s[s], ch_s[s + 1]);
                    if (lane == 0) {
                        PcgScene P = load_sc(SC + s);
                        if (!P.inner_done) {
                            P.alpha = sq != 0.0 ? P.rho / sq : 0.0;
                            float sq32 = (float)sq;
                            P.alpha32 = sq32 != 0.0f ? P.rho32 / sq32 : 0.0f;
                            SC[s] = P;
                        }
                    }
                }
            });
            if (!ok) return;
            // Phase B: x += alpha s, r -= alpha q, r.r; z = M r, z.r (fused when no scene is
            // ordered)
            for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
                int s;
                long long t0, t1;
                chunk_range(ch, s, t0, t1);
                double a0 = 0.0, a1 = 0.0;
                if (!ldv(&SC[s].inner_done)) {
                    const T al = MODE == kRef32 ? (T)ldv(&SC[s].alpha32) : (T)ldv(&SC[s].alpha);
                    const bool fuse = !any_ordered;
                    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                        long long c = A.fl[t];
                        T sv = ldv(s_cur + c);
                        T xv = ldv(x + c) + al * sv;
                        T rv = ldv(r + c) + (-al) * ldv(q + c);
                        x[c] = xv;
                        r[c] = rv;
                        a0 += (double)rv * (double)rv;
                        if (fuse) {
                            T zv = precond_elem(c, rv);
                            z[c] = zv;
                            a1 += (double)zv * (double)rv;
                        }
                    }
                }
                write_part(ch, a0, a1);
            }
            if (any_ordered) {
                ok = grid_barrier(A.bar, S.dev_error, tmo, NoLeader{});
                if (!ok) return;
                for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
                    int s;
                    long long t0, t1;
                    chunk_range(ch, s, t0, t1);
                    if (ldv(&SC[s].ordered)) continue;
                    double a1 = 0.0;
                    if (!ldv(&SC[s].inner_done)) {
                        for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                            long long c = A.fl[t];
                            T rv = ldv(r + c);
                            T zv = precond_elem(c, rv);
                            z[c] = zv;
                            a1 += (double)zv * (double)rv;
                        }
                    }
                    double b0 = 0.0;
                    block_sum2(a1, b0);
                    if (threadIdx.x == 0) part1[ch] = a1;
                }
                ++bseq;
                if (!brick_sweep<kFwd, T>(A, BS, bseq, r, ordq, pcv, tmo)) return;
                ++bseq;
                if (!brick_sweep<kBwd, T>(A, BS, bseq, ordq, z, pcv, tmo)) return;
                ok = grid_barrier(A.bar, S.dev_error, tmo, NoLeader{});
                if (!ok) return;
                for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
                    int s;
                    long long t0, t1;
                    chunk_range(ch, s, t0, t1);
                    if (!ldv(&SC[s].ordered)) continue;
                    double a1 = 0.0;
                    if (!ldv(&SC[s].inner_done))
                        for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                            long long c = A.fl[t];
                            a1 += (double)ldv(z + c) * (double)ldv(r + c);
                        }
                    double b0 = 0.0;
                    block_sum2(a1, b0);
                    if (threadIdx.x == 0) part1[ch] = a1;
                }
            }
            ok = grid_barrier(A.bar, S.dev_error, tmo, [&]() {
                if (threadIdx.x == 0) s_active = 0;
                __syncthreads();
                const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
                for (int s = wid; s < k; s += blockDim.x / 32) {
                    double rr = scene_sum(part0, ch_s[s], ch_s[s + 1]);
                    double rho2 = scene_sum(part1, ch_s[s], ch_s[s + 1]);
                    if (lane == 0) {
                        PcgScene P = load_sc(SC + s);
                        if (!P.inner_done) {
                            const int n = S.scenes[s].n;
                            P.iters += 1;
                            P.rr = rr;
                            const int cap = A.max_iters > 0 ? A.max_iters : n * n * n;
                            bool conv = MODE == kRef32 ? ((float)rr <= (float)P.target) : (rr <= P.target);
                            if (conv || P.iters >= cap) {
                                P.inner_done = 1;
                                if (MODE != kMixed) {
                                    P.done = 1;
                                    P.converged = conv;
                                }
                            } else {
                                P.beta = P.rho != 0.0 ? rho2 / P.rho : 0.0;
                                P.rho = rho2;
                                float r32 = (float)rho2;
                                P.beta32 = P.rho32 != 0.0f ? r32 / P.rho32 : 0.0f;
                                P.rho32 = r32;
                                atomicAdd(&s_active, 1);
                            }
                            SC[s] = P;
                        }
                    }
                }
                __syncthreads();
                if (threadIdx.x == 0) A.ctl->all_inner_done = s_active == 0;
            });
            if (!ok) return;
            if (ldv(&A.ctl->all_inner_done)) break;
        }

        if (MODE != kMixed) break;
        // ---- MIXED: x64 += d ------------------------------------------------------------------
        for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
            int s;
            long long t0, t1;
            chunk_range(ch, s, t0, t1);
            if (ldv(&SC[s].done)) continue;
            for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                long long c = A.fl[t];
                S.P64[c] = ldv(S.P64 + c) + (double)ldv(x + c);
            }
        }
        if (!grid_barrier(A.bar, S.dev_error, tmo, NoLeader{})) return;
        ++outer;
    }

    // ---- totals (block 0; every scene is done here) ---------------------------------------
    if (blockIdx.x == 0) {
        for (int s = threadIdx.x; s < k; s += blockDim.x) {
            PcgScene P = load_sc(SC + s);
            PcgTotals& T = A.totals[s];
            T.solves += 1;
            T.iterations += P.iters;
            T.outer += MODE == kMixed ? P.outer : 1;
            T.cell_iterations += (double)P.nf * (double)P.iters;
            T.cell_outer += (double)P.nf * (double)(MODE == kMixed ? P.outer : 1);
            T.not_converged += P.converged ? 0 : 1;
        }
    }
    // ---- output: fp32 pressure from the fp64 solution ---------------------------------------
    if (MODE != kRef32) {
        for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
            int s;
            long long t0, t1;
            chunk_range(ch, s, t0, t1);
            for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                long long c = A.fl[t];
                S.P[c] = (float)ldv(S.P64 + c);
            }
        }
    }
}

__global__ void k_barrier_selftest(Barrier* bar, int* err, unsigned long long tmo) {
    // Nobody releases this barrier, so every block must give up when its budget runs out.
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned g = ld_acquire_u32(&bar->gen);
        atomicAdd(&bar->count, 1u);
        unsigned long long t0 = gtimer();
        while (ld_acquire_u32(&bar->gen) == g) {
            if (gtimer() - t0 > tmo) {
                atomicExch(&bar->error, 1);
                atomicExch(err, 1);
                break;
            }
            __nanosleep(1000);
        }
    }
    __syncthreads();
}

}  // namespace

cudaError_t launch_pcg_prepare(const PcgArgs& A, uint32_t* pred, uint32_t* scan, void* scan_tmp, cudaStream_t st) {
    const DevState& S = A.S;
    cudaMemsetAsync(A.sc, 0, sizeof(PcgScene) * (size_t)S.k, st);
    cudaMemsetAsync(A.ctl, 0, sizeof(PcgCtl), st);
    cudaMemsetAsync(A.bar, 0, sizeof(Barrier), st);
    if (A.nbricks > 0) cudaMemsetAsync(A.bflag, 0, sizeof(unsigned) * (size_t)A.nbricks, st);
    if (S.nc > 0) {
        k_prep_cells<<<grid_for(S.nc), kBlock, 0, st>>>(A, pred);
        count_launch();
    }
    cudaError_t e = launch_scan_u32(pred, scan, S.nc, scan_tmp, st);
    if (e != cudaSuccess) return e;
    if (S.nc > 0) {
        k_fl_write<<<grid_for(S.nc), kBlock, 0, st>>>(A, pred, scan);
        count_launch();
    }
    k_pcg_tables<<<1, 32, 0, st>>>(A, scan);
    count_launch();
    return cudaGetLastError();
}

// ==========================================================================================
// Fast path (elementwise reference preconditioner, up to kFastMaxScenes scenes per launch).
//
// No leader block: a grid barrier is a monotonic arrival counter (barrier e completes when it
// reaches e * gridDim.x), after which every block reads all chunk partials and reduces each
// scene's range in the same fixed tree.  Every block therefore holds bit-identical copies of
// every scene's alpha/beta/stop state in shared memory, and a barrier costs one arrival plus
// one partial read on the critical path.  Each block also keeps the FLUID-list records of its
// first chunk in shared memory for the whole solve and streams the others' through per-thread
// prefetch slots.
// ==========================================================================================
constexpr int kFastMaxScenes = 128;
constexpr int kChunkCells = kChunkMax;  // the largest chunk (cache slot size)
// Records of each block's first chunk stay in shared memory for the whole solve (at 128^3 that
// is every chunk); later chunks stream theirs through the prefetch slots.  A second cached chunk
// measured slower: the shared memory it takes comes out of the L1 the neighbour loads hit.
constexpr int kFlCacheChunks = 1;

struct SceneLocal {
    double bb, rr, rho, alpha, beta, target, rr_out;
    float alpha32, beta32, rho32;
    int iters, outer, done, inner_done, converged, nf;
};

// Asynchronous 16-byte global -> shared copies (L1 bypassed), completed per thread.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(__cvta_generic_to_global(gmem))
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(__cvta_generic_to_global(gmem))
                 : "memory");
}
__device__ __forceinline__ void cp_async_el(float4* smem, const float4* gmem) { cp_async16(smem, gmem); }
__device__ __forceinline__ void cp_async_el(double4* smem, const double4* gmem) {
    cp_async16(smem, gmem);
    cp_async16(reinterpret_cast<char*>(smem) + 16, reinterpret_cast<const char*>(gmem) + 16);
}
__device__ __forceinline__ void cp_async_el(float2* smem, const float2* gmem) { cp_async8(smem, gmem); }
__device__ __forceinline__ void cp_async_el(double2* smem, const double2* gmem) { cp_async16(smem, gmem); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ unsigned ld_acquire_cnt(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Barrier number `epoch` (1, 2, ...) of this launch.  The block's writes are ordered before its
// arrival by __syncthreads and thread 0's release reduction (cumulative over what the block's
// barrier made visible to it); thread 0's acquire load that sees the count complete, followed by
// __syncthreads, orders every thread's later loads after all blocks' arrivals -- the pattern of
// grid_barrier with the release and acquire carried by the counter operations themselves.
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ bool count_barrier(Barrier* bar, int* dev_error, unsigned epoch, unsigned long long timeout_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        red_release_add(&bar->count, 1u);
        const unsigned target = epoch * gridDim.x;
        const unsigned long long t0 = gtimer();
        while (ld_acquire_cnt(&bar->count) < target) {
            if (*(volatile int*)&bar->error) {
                s_ok = 0;
                break;
            }
            if (gtimer() - t0 > timeout_ns) {
                atomicExch(&bar->error, 1);
                if (dev_error) atomicExch(dev_error, 1);
                s_ok = 0;
                break;
            }
            __nanosleep(16);
        }
    }
    __syncthreads();
    return s_ok != 0;
}

// Sums of three partial arrays over [b, e) by one warp (fixed tree depending only on e - b).
__device__ __forceinline__ void scene_sum3(const double* p0, const double* p1, const double* p2, int nsum,
                                           long long b, long long e, double& o0, double& o1, double& o2) {
    const int lane = threadIdx.x & 31;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    for (long long base = b; base < e; base += 32 * 16) {
        double x0[16], x1[16], x2[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            long long c = base + (long long)u * 32 + lane;
            bool in = c < e;
            x0[u] = in ? p0[c] : 0.0;
            x1[u] = (in && nsum > 1) ? p1[c] : 0.0;
            x2[u] = (in && nsum > 2) ? p2[c] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            v0 += x0[u];
            v1 += x1[u];
            v2 += x2[u];
        }
    }
    v0 = warp_sum(v0);
    v1 = warp_sum(v1);
    v2 = warp_sum(v2);
    o0 = __shfl_sync(0xffffffffu, v0, 0);
    o1 = __shfl_sync(0xffffffffu, v1, 0);
    o2 = __shfl_sync(0xffffffffu, v2, 0);
}

// Packed per-cell state of the single-reduction path (T = float for MIXED, double for FP64):
//   Av[parity][c] = (r_i, w_i, s_{i-1}, pc)  -- read at c and its six neighbours, so
//                                              double-buffered by iteration parity;
//   Bv[c]         = (p_{i-1}, x_i)           -- read and written only by c's owner.
// u_i = M r_i is not stored: its owner recomputes it as (r_i * pc) * pc from Av, the same
// expression on the same values as in the iteration that produced r_i, so the same bits.
template <class T>
struct V2;
template <>
struct V2<float> {
    using type = float2;
};
template <>
struct V2<double> {
    using type = double2;
};
template <class T>
__device__ __forceinline__ typename V2<T>::type mk2(T a, T b);
template <>
__device__ __forceinline__ float2 mk2<float>(float a, float b) {
    return make_float2(a, b);
}
template <>
__device__ __forceinline__ double2 mk2<double>(double a, double b) {
    return make_double2(a, b);
}
template <class T>
struct V4;
template <>
struct V4<float> {
    using type = float4;
};
template <>
struct V4<double> {
    using type = double4;
};
__device__ __forceinline__ double4 ld4(const double4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = q[0], b = q[1];
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ld4(const float4* p) { return *p; }
__device__ __forceinline__ void st4(double4* p, double4 v) {
    double2* q = reinterpret_cast<double2*>(p);
    q[0] = make_double2(v.x, v.y);
    q[1] = make_double2(v.z, v.w);
}
__device__ __forceinline__ void st4(float4* p, float4 v) { *p = v; }
template <class T>
__device__ __forceinline__ typename V4<T>::type mk4(T a, T b, T c, T d);
template <>
__device__ __forceinline__ float4 mk4<float>(float a, float b, float c, float d) {
    return make_float4(a, b, c, d);
}
template <>
__device__ __forceinline__ double4 mk4<double>(double a, double b, double c, double d) {
    return make_double4(a, b, c, d);
}

__device__ __forceinline__ void dec_diag(const uint4& r, float& d) { d = __uint_as_float(r.z); }
__device__ __forceinline__ void dec_diag(const uint4& r, double& d) {
    d = __longlong_as_double((long long)(((unsigned long long)r.w << 32) | (unsigned long long)r.z));
}

// Dynamic shared memory of k_pcg_fast: the per-solve caches of the block's first chunks
// (diagonal, cell index, mask), then the single-reduction path's per-thread prefetch slots,
// [kIlp][threads] each: records for 3 rounds, packed Av and packed Bv for 2 rounds.
__host__ __device__ constexpr int fast_ilp(int mode) { return mode == kFp64 ? 1 : 2; }
size_t fast_slot_bytes(int mode) {
    if (mode == kRef32) return 0;
    const size_t tb = mode == kFp64 ? 8 : 4;
    return (size_t)fast_ilp(mode) * kPcgThreads * (3 * 16 + 2 * (4 * tb + 2 * tb));
}
size_t fast_cache_bytes(int mode) {
    const size_t tb = mode == kFp64 ? 8 : 4;
    return (size_t)kFlCacheChunks * kChunkCells * (4 + 1 + tb);
}
size_t fast_dyn_smem(int mode) { return fast_cache_bytes(mode) + fast_slot_bytes(mode); }

template <int MODE>
__global__ void __launch_bounds__(kPcgThreads, 2) k_pcg_fast(PcgArgs A) {
    using T = typename VT<MODE>::T;
    using T4 = typename V4<T>::type;
    if (A.ctl->any_ordered) return;  // the ordered preconditioner runs in k_pcg
    const DevState& S = A.S;
    const int k = S.k;
    __shared__ long long fl_s[kFastMaxScenes + 1], ch_s[kFastMaxScenes + 1];
    __shared__ int csz_s[kFastMaxScenes];
    __shared__ SceneLocal L[kFastMaxScenes];
    __shared__ int s_active;
    // per-solve caches of this block's first kFlCacheChunks chunks: FLUID cell index,
    // neighbour mask, diagonal
    extern __shared__ __align__(16) unsigned char dyn[];
    T* dgc = reinterpret_cast<T*>(dyn);
    uint32_t* flc = reinterpret_cast<uint32_t*>(dyn + sizeof(T) * kFlCacheChunks * kChunkCells);
    uint8_t* mkc = reinterpret_cast<uint8_t*>(flc + kFlCacheChunks * kChunkCells);
    // prefetch slots of the single-reduction path, [buffer][ILP lane][thread]: records in 3
    // buffers (round mod 3), own state in 2 (round parity)
    using T2 = typename V2<T>::type;
    constexpr int kIlp = fast_ilp(MODE);
    uint4* const recbuf = reinterpret_cast<uint4*>(dyn + (size_t)kFlCacheChunks * kChunkCells * (sizeof(T) + 5));
    T4* const ownA = reinterpret_cast<T4*>(recbuf + 3 * kIlp * kPcgThreads);
    T2* const ownB = reinterpret_cast<T2*>(ownA + 2 * kIlp * kPcgThreads);
    auto slot = [&](int buf, int u) { return (buf * kIlp + u) * kPcgThreads + (int)threadIdx.x; };
    for (int i = threadIdx.x; i <= k; i += blockDim.x) {
        fl_s[i] = A.fl_pref[i];
        ch_s[i] = A.ch_pref[i];
    }
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        SceneLocal z{};
        z.nf = A.sc[i].nf;
        L[i] = z;
        csz_s[i] = A.sc[i].csize;
    }
    __syncthreads();
    const long long nch = ch_s[k];
    const long long MC = A.max_chunks;
    double* part0 = A.partial;
    double* part1 = A.partial + MC;
    double* part2 = A.partial + 2 * MC;
    const unsigned long long tmo = A.timeout_ns;
    unsigned epoch = 0;
    // Chunk sums are reduced per warp at once but combined across warps only every kDefer
    // chunks (and at the end of each pass), so warps never wait for one another inside a pass.
    // The combination is the same fixed tree as block_sum2: lane-0 warp sums, then one warp
    // over the warp sums with zero padding.
    constexpr int kDefer = 16;
    constexpr int kWarps = kPcgThreads / 32;
    __shared__ double dsum[kDefer][3][kWarps];
    int npend = 0, jpend0 = 0;
    auto flush = [&]() {
        if (npend == 0) return;
        __syncthreads();
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int jj = wid; jj < npend; jj += kWarps) {
            double v0 = lane < kWarps ? dsum[jj][0][lane] : 0.0;
            double v1 = lane < kWarps ? dsum[jj][1][lane] : 0.0;
            double v2 = lane < kWarps ? dsum[jj][2][lane] : 0.0;
            v0 = warp_sum(v0);
            v1 = warp_sum(v1);
            v2 = warp_sum(v2);
            if (lane == 0) {
                const long long ch = blockIdx.x + (long long)(jpend0 + jj) * gridDim.x;
                part0[ch] = v0;
                part1[ch] = v1;
                part2[ch] = v2;
            }
        }
        __syncthreads();
        npend = 0;
    };
    auto chunk_of = [&](int j, int& s, long long& t0, long long& t1) -> bool {
        long long ch = blockIdx.x + (long long)j * gridDim.x;
        if (ch >= nch) {
            flush();  // every chunk pass ends here
            return false;
        }
        s = find_scene(ch_s, k, ch);
        const long long cs = csz_s[s];
        t0 = fl_s[s] + (ch - ch_s[s]) * cs;
        t1 = min(t0 + cs, fl_s[s + 1]);
        return true;
    };
    for (int j = 0; j < kFlCacheChunks; ++j) {
        int s;
        long long t0, t1;
        if (!chunk_of(j, s, t0, t1)) break;
        for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
            const uint4 rc = A.rec[t];
            int o = j * kChunkCells + (int)(t - t0);
            flc[o] = rc.x;
            mkc[o] = (uint8_t)rc.y;
            T dg;
            dec_diag(rc, dg);
            dgc[o] = dg;
        }
    }
    __syncthreads();
    auto cell_at = [&](int j, long long t, long long t0) -> long long {
        return j < kFlCacheChunks ? (long long)flc[j * kChunkCells + (int)(t - t0)] : (long long)A.fl[t];
    };
    auto mask_at = [&](int j, long long t, long long t0, long long c) -> uint32_t {
        return j < kFlCacheChunks ? (uint32_t)mkc[j * kChunkCells + (int)(t - t0)] : (uint32_t)A.mask[c];
    };
    auto diag_at = [&](int j, long long t, long long t0, long long c) -> T {
        return j < kFlCacheChunks ? dgc[j * kChunkCells + (int)(t - t0)] : (T)A.diag[c];
    };
    // cell, mask and diagonal of list entry t from one shared-memory or one 16-byte global read
    auto cell_rec = [&](int j, long long t, long long t0, long long& c, uint32_t& m, T& dg) {
        if (j < kFlCacheChunks) {
            const int o = j * kChunkCells + (int)(t - t0);
            c = (long long)flc[o];
            m = (uint32_t)mkc[o];
            dg = dgc[o];
        } else {
            const uint4 rc = A.rec[t];
            c = (long long)rc.x;
            m = rc.y;
            dec_diag(rc, dg);
        }
    };
    auto put3 = [&](int j, double a, double b, double c) {
        a = warp_sum(a);
        b = warp_sum(b);
        c = warp_sum(c);
        if (npend == 0) jpend0 = j;
        if ((threadIdx.x & 31) == 0) {
            const int wid = threadIdx.x >> 5;
            dsum[npend][0][wid] = a;
            dsum[npend][1][wid] = b;
            dsum[npend][2][wid] = c;
        }
        if (++npend == kDefer) flush();
    };
    auto reduce = [&](int nsum, auto&& f) {
        if (threadIdx.x == 0) s_active = 0;
        __syncthreads();
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int s = wid; s < k; s += blockDim.x / 32) {
            if (L[s].inner_done && L[s].done) continue;
            double v0, v1, v2;
            scene_sum3(part0, part1, part2, nsum, ch_s[s], ch_s[s + 1], v0, v1, v2);
            if (lane == 0) {
                if (f(s, L[s], v0, v1, v2)) atomicAdd(&s_active, 1);
            }
        }
        __syncthreads();
        return s_active;
    };

    T* r = (T*)A.r;
    T* z = (T*)A.z;
    T* q = (T*)A.q;
    T* const sb0 = (T*)A.s0;
    T* const sb1 = (T*)A.s1;
    const T* pcv = MODE == kFp64 ? (const T*)(const void*)A.pc64 : (const T*)(const void*)A.pc32;
    T* x = MODE == kRef32 ? (T*)(void*)S.P : (MODE == kFp64 ? (T*)(void*)S.P64 : (T*)(void*)A.d32);
    auto precond = [&](long long c, T rv) -> T { return (rv * pcv[c]) * pcv[c]; };
    T4* const Av0 = (T4*)A.va0;
    T4* const Av1 = (T4*)A.va1;
    T2* const Bv = (T2*)A.vb;

    int outer = 0;
    while (true) {
        // ---- residual r = b - A x, |b|^2 --------------------------------------------------
        for (int j = 0;; ++j) {
            int s;
            long long t0, t1;
            if (!chunk_of(j, s, t0, t1)) break;
            const SceneDev& D = S.scenes[s];
            double a0 = 0.0, a1 = 0.0;
            if (!L[s].done) {
                for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                    long long c = cell_at(j, t, t0);
                    double bv = (double)S.D[c];
                    if (MODE == kRef32) {
                        float xc = S.P[c];
                        float ax = ax_ref32(S, D, c, xc, [&](long long qq) { return S.P[qq]; });
                        float rv = S.D[c] + (-1.0f) * ax;
                        r[c] = (T)rv;
                        a0 += (double)rv * (double)rv;
                    } else {
                        double xc = S.P64[c];
                        double ax = ax_diag<double>(A, D, c, xc, [&](long long qq) { return S.P64[qq]; });
                        double rv = bv - ax;
                        if (MODE == kMixed)
                            A.r64[c] = rv;
                        else
                            r[c] = (T)rv;
                        a0 += rv * rv;
                    }
                    a1 += bv * bv;
                }
            }
            put3(j, a0, a1, 0.0);
        }
        if (!count_barrier(A.bar, S.dev_error, ++epoch, tmo)) return;
        int active = reduce(2, [&](int s, SceneLocal& P, double rr, double bb, double) -> bool {
            if (P.done) return false;
            const int n = S.scenes[s].n;
            if (outer == 0) P.bb = bb;
            P.rr_out = rr;
            if (MODE == kMixed) P.outer += 1;
            double lim2 = A.tol * A.tol * P.bb;
            double abs_eps = (double)(1.0e-2f * (float)(n * n * n));
            bool conv = false;
            if (A.stop_rule == ARIEL_STOP_REL)
                conv = rr <= lim2;
            else if (MODE == kMixed)
                conv = outer > 0 && rr <= abs_eps;
            if (P.nf == 0) conv = true;
            int cap = A.max_iters > 0 ? A.max_iters : n * n * n;
            if (conv) {
                P.done = 1;
                P.converged = 1;
            } else if (MODE == kMixed && (P.outer > A.max_outer || P.iters >= cap)) {
                P.done = 1;
                P.converged = 0;
            }
            if (P.done) {
                P.inner_done = 1;
                return false;
            }
            P.inner_done = 0;
            P.rr = rr;
            if (MODE == kMixed) {
                // the correction solve stops at the final tolerance itself (its fp32 residual);
                // the true fp64 residual then decides whether another sweep is needed
                double a = A.inner_tol * A.inner_tol * rr;
                double b = A.stop_rule == ARIEL_STOP_REL ? lim2 : 0.0;
                P.target = a > b ? a : b;
            } else {
                P.target = A.stop_rule == ARIEL_STOP_REL ? lim2 : abs_eps;
            }
            return true;
        });
        if (active == 0) break;

        if (MODE != kRef32) {
            // ---- single-reduction PCG (Chronopoulos & Gear, 1989), one barrier per
            // iteration.  Iteration i reads Av[i&1] = (r_i, w_i, s_{i-1}, pc) at c and its
            // neighbours and Bv = (p_{i-1}, x_i) at c, and writes s_i = w_i + beta s_{i-1},
            // p_i = u_i + beta p_{i-1}, x_{i+1} = x_i + alpha p_i, r_{i+1} = r_i - alpha s_i,
            // u_{i+1} = M r_{i+1} and w_{i+1} = A u_{i+1}; the neighbour values of u_{i+1} are
            // recomputed from the same old state, bit-identically to what their owners write.
            for (int j = 0;; ++j) {
                int s;
                long long t0, t1;
                if (!chunk_of(j, s, t0, t1)) break;
                const SceneDev& D = S.scenes[s];
                double g0 = 0.0, d0 = 0.0, q0 = 0.0;
                if (!L[s].inner_done) {
                    auto r0 = [&](long long qq) -> T { return MODE == kMixed ? (T)A.r64[qq] : r[qq]; };
                    const T scale = (T)(1.0 / (double)D.ax_h);
                    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                        long long c = cell_at(j, t, t0);
                        const uint32_t m = mask_at(j, t, t0, c);
                        T rv = r0(c);
                        T pcc = pcv[c];
                        T uv = (rv * pcc) * pcc;
                        T acc = diag_at(j, t, t0, c) * uv;
#pragma unroll
                        for (int d = 0; d < 6; ++d)
                            if (m & (1u << d)) {
                                long long qq = c + nb_off(d, D.n);
                                acc -= precond(qq, r0(qq));
                            }
                        T wv = acc * scale;
                        T xv = MODE == kMixed ? (T)0 : S.P64[c];
                        st4(Av0 + c, mk4<T>(rv, wv, (T)0, pcc));
                        Bv[c] = mk2<T>((T)0, xv);
                        g0 += (double)rv * (double)uv;
                        d0 += (double)wv * (double)uv;
                        q0 += (double)rv * (double)rv;
                    }
                }
                put3(j, g0, d0, q0);
            }
            if (!count_barrier(A.bar, S.dev_error, ++epoch, tmo)) return;
            reduce(2, [&](int, SceneLocal& P, double g, double d, double) -> bool {
                if (P.inner_done) return false;
                P.rho = g;
                P.alpha = d != 0.0 ? g / d : 0.0;
                P.beta = 0.0;
                return true;
            });
            for (int it = 0;; ++it) {
                const T4* Ac = (it & 1) ? Av1 : Av0;
                T4* An = (it & 1) ? Av0 : Av1;
                const int step = kIlp * (int)blockDim.x;
                // This thread's rounds in the streamed chunks (those past the cached ones) form one
                // pipeline across chunk boundaries: a round's records and own state are copied
                // into this thread's slots ahead of use (own state one round, records two), and no
                // copy targets a slot read in the same round, so a round waits only for its
                // neighbours' loads.  A position is (chunk j, chunk end t1, round start tb); list
                // indices fit 32 bits (fewer than 2^31 cells).
                struct Pos {
                    int j, t1, tb;
                };
                // to this thread's next round in an active streamed chunk; false past the last
                auto advance = [&](Pos& p) -> bool {
                    if (p.tb + step < p.t1) {
                        p.tb += step;
                        return true;
                    }
                    for (int jj = p.j + 1;; ++jj) {
                        const long long ch = blockIdx.x + (long long)jj * gridDim.x;
                        if (ch >= nch) return false;
                        const int s2 = find_scene(ch_s, k, ch);
                        const long long cs = csz_s[s2];
                        const long long a0 = fl_s[s2] + (ch - ch_s[s2]) * cs;
                        const long long a1 = min(a0 + cs, fl_s[s2 + 1]);
                        if (L[s2].inner_done || a0 + (long long)threadIdx.x >= a1) continue;
                        p.j = jj;
                        p.t1 = (int)a1;
                        p.tb = (int)a0 + (int)threadIdx.x;
                        return true;
                    }
                };
                auto issue_rec = [&](const Pos& p, int par) {
#pragma unroll
                    for (int u = 0; u < kIlp; ++u) {
                        const int t = p.tb + u * (int)blockDim.x;
                        if (t < p.t1) cp_async16(recbuf + slot(par, u), A.rec + t);
                    }
                };
                auto read_rec = [&](const Pos& p, int par, long long* c, uint32_t* m, T* dg, bool* on) {
#pragma unroll
                    for (int u = 0; u < kIlp; ++u) {
                        on[u] = p.tb + u * (int)blockDim.x < p.t1;
                        if (on[u]) {
                            const uint4 rc = recbuf[slot(par, u)];
                            c[u] = (long long)rc.x;
                            m[u] = rc.y;
                            dec_diag(rc, dg[u]);
                        } else {
                            c[u] = c[0];
                            m[u] = 0u;
                            dg[u] = (T)0;
                        }
                    }
                };
                auto issue_own = [&](const long long* c, const bool* on, int par) {
#pragma unroll
                    for (int u = 0; u < kIlp; ++u)
                        if (on[u]) {
                            cp_async_el(ownA + slot(par, u), Ac + c[u]);
                            cp_async_el(ownB + slot(par, u), Bv + c[u]);
                        }
                };
                // pipeline state: the current position p0 and the next p1; round R keeps its
                // records in buffer R mod 3 (rb) and its own state in buffer R mod 2
                Pos p0{kFlCacheChunks - 1, 0, 0}, p1{0, 0, 0};
                bool v0 = advance(p0), v1 = false;
                int R = 0, rb = 0;
                if (v0) {
                    issue_rec(p0, 0);
                    cp_async_commit();
                    cp_async_wait_all();
                    long long c[kIlp];
                    uint32_t m[kIlp];
                    T dg[kIlp];
                    bool on[kIlp];
                    read_rec(p0, 0, c, m, dg, on);
                    issue_own(c, on, 0);
                    p1 = p0;
                    v1 = advance(p1);
                    if (v1) issue_rec(p1, 1);
                    cp_async_commit();
                }
                for (int j = 0;; ++j) {
                    int s;
                    long long t0, t1;
                    if (!chunk_of(j, s, t0, t1)) break;
                    const SceneDev& D = S.scenes[s];
                    double g1 = 0.0, d1 = 0.0, q1 = 0.0;
                    if (!L[s].inner_done) {
                        const T al = (T)L[s].alpha;
                        const T bt = (T)L[s].beta;
                        const T scale = (T)(1.0 / (double)D.ax_h);
                        const long long nn = (long long)D.n * D.n, n1 = D.n;
                        // kIlp list entries per thread at once (t, t + blockDim.x, ...): their
                        // loads overlap; the sums still accumulate in ascending t per thread.
                        auto off = [&](int d) -> long long {
                            return d == 0 ? -nn : d == 1 ? nn : d == 2 ? -n1 : d == 3 ? n1 : d == 4 ? -1ll : 1ll;
                        };
                        // One round: the six neighbours' (r, w, s, pc), then the update of the
                        // round's cells from their own state (a, b).
                        auto round = [&](const long long* c, const uint32_t* m, const T* dg, const bool* on,
                                         const T4* a, const T2* b) {
                            T4 nb[kIlp][6];
#pragma unroll
                            for (int u = 0; u < kIlp; ++u)
#pragma unroll
                                for (int d = 0; d < 6; ++d)
                                    nb[u][d] = ld4(Ac + ((m[u] >> d) & 1u ? c[u] + off(d) : c[u]));
#pragma unroll
                            for (int u = 0; u < kIlp; ++u) {
                                if (!on[u]) continue;
                                const T sv = it == 0 ? a[u].y : a[u].y + bt * a[u].z;
                                const T ui = (a[u].x * a[u].w) * a[u].w;
                                const T pvv = it == 0 ? ui : ui + bt * b[u].x;
                                const T xv = b[u].y + al * pvv;
                                const T rn = a[u].x - al * sv;
                                const T un = (rn * a[u].w) * a[u].w;
                                T acc = dg[u] * un;
#pragma unroll
                                for (int d = 0; d < 6; ++d) {
                                    if ((m[u] >> d) & 1u) {
                                        const T4 e = nb[u][d];
                                        const T sq = it == 0 ? e.y : e.y + bt * e.z;
                                        const T rq = e.x - al * sq;
                                        acc -= (rq * e.w) * e.w;
                                    }
                                }
                                const T wn = acc * scale;
                                st4(An + c[u], mk4<T>(rn, wn, sv, a[u].w));
                                Bv[c[u]] = mk2<T>(pvv, xv);
                                g1 += (double)rn * (double)un;
                                d1 += (double)wn * (double)un;
                                q1 += (double)rn * (double)rn;
                            }
                        };
                        if (j >= kFlCacheChunks) {
                            while (v0 && p0.j == j) {
                                const int rb1 = rb == 2 ? 0 : rb + 1, rb2 = rb1 == 2 ? 0 : rb1 + 1;
                                cp_async_wait_all();  // own state of this round, records of the next
                                Pos p2 = p1;
                                bool v2 = false;
                                if (v1) {
                                    long long cn[kIlp];
                                    uint32_t mn[kIlp];
                                    T dn[kIlp];
                                    bool onn[kIlp];
                                    read_rec(p1, rb1, cn, mn, dn, onn);
                                    issue_own(cn, onn, (R + 1) & 1);
                                    v2 = advance(p2);
                                    if (v2) issue_rec(p2, rb2);
                                }
                                cp_async_commit();
                                long long c[kIlp];
                                uint32_t m[kIlp];
                                T dg[kIlp];
                                bool on[kIlp];
                                read_rec(p0, rb, c, m, dg, on);
                                T4 a[kIlp];
                                T2 b[kIlp];
#pragma unroll
                                for (int u = 0; u < kIlp; ++u) {
                                    a[u] = ld4(ownA + slot(R & 1, u));
                                    b[u] = ownB[slot(R & 1, u)];
                                }
                                round(c, m, dg, on, a, b);
                                p0 = p1;
                                v0 = v1;
                                p1 = p2;
                                v1 = v2;
                                ++R;
                                rb = rb1;
                            }
                        } else {
                            for (long long tb = t0 + threadIdx.x; tb < t1; tb += step) {
                                long long c[kIlp];
                                uint32_t m[kIlp];
                                T dg[kIlp];
                                bool on[kIlp];
#pragma unroll
                                for (int u = 0; u < kIlp; ++u) {
                                    const long long t = tb + (long long)u * blockDim.x;
                                    on[u] = t < t1;
                                    if (on[u]) {
                                        cell_rec(j, t, t0, c[u], m[u], dg[u]);
                                    } else {
                                        c[u] = c[0];
                                        m[u] = 0u;
                                        dg[u] = (T)0;
                                    }
                                }
                                T4 a[kIlp];
                                T2 b[kIlp];
#pragma unroll
                                for (int u = 0; u < kIlp; ++u) {
                                    a[u] = ld4(Ac + c[u]);
                                    b[u] = Bv[c[u]];
                                }
                                round(c, m, dg, on, a, b);
                            }
                        }
                    }
                    put3(j, g1, d1, q1);
                }
                if (!count_barrier(A.bar, S.dev_error, ++epoch, tmo)) return;
                int act = reduce(3, [&](int s, SceneLocal& P, double g, double d, double rr) -> bool {
                    if (P.inner_done) return false;
                    const int n = S.scenes[s].n;
                    P.iters += 1;
                    P.rr = rr;
                    const int cap = A.max_iters > 0 ? A.max_iters : n * n * n;
                    bool conv = rr <= P.target;
                    if (conv || P.iters >= cap) {
                        P.inner_done = 1;
                        if (MODE != kMixed) {
                            P.done = 1;
                            P.converged = conv;
                        }
                        return false;
                    }
                    double beta = P.rho != 0.0 ? g / P.rho : 0.0;
                    double den = d - (P.alpha != 0.0 ? beta * g / P.alpha : 0.0);
                    P.beta = beta;
                    P.alpha = den != 0.0 ? g / den : 0.0;
                    P.rho = g;
                    return true;
                });
                if (act == 0) break;
            }
            // fold the solve's x back: MIXED adds the correction to x64, FP64 stores x64
            for (int j = 0;; ++j) {
                int s;
                long long t0, t1;
                if (!chunk_of(j, s, t0, t1)) break;
                if (MODE == kMixed && L[s].done) continue;
                for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                    long long c = cell_at(j, t, t0);
                    const T2 b = Bv[c];
                    S.P64[c] = MODE == kMixed ? S.P64[c] + (double)b.y : (double)b.y;
                }
            }
            if (MODE != kMixed) break;
            if (!count_barrier(A.bar, S.dev_error, ++epoch, tmo)) return;
            ++outer;
            continue;
        }

        // ---- REF32: the reference's two-reduction PCG (solver.inl:289-354) ------------------
        for (int j = 0;; ++j) {
            int s;
            long long t0, t1;
            if (!chunk_of(j, s, t0, t1)) break;
            double a0 = 0.0;
            if (!L[s].inner_done) {
                for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                    long long c = cell_at(j, t, t0);
                    T rv = r[c];
                    T zv = precond(c, rv);
                    z[c] = zv;
                    sb0[c] = zv;
                    a0 += (double)zv * (double)rv;
                }
            }
            put3(j, a0, 0.0, 0.0);
        }
        if (!count_barrier(A.bar, S.dev_error, ++epoch, tmo)) return;
        reduce(1, [&](int, SceneLocal& P, double rho, double, double) -> bool {
            if (P.inner_done) return false;
            P.rho = rho;
            P.rho32 = (float)rho;
            return true;
        });
        for (int it = 0;; ++it) {
            T* s_cur = (it & 1) ? sb1 : sb0;
            T* s_prev = (it & 1) ? sb0 : sb1;
            for (int j = 0;; ++j) {
                int s;
                long long t0, t1;
                if (!chunk_of(j, s, t0, t1)) break;
                const SceneDev& D = S.scenes[s];
                double a0 = 0.0;
                if (!L[s].inner_done) {
                    const T bt = (T)L[s].beta32;
                    auto sval = [&](long long qq) -> T { return it == 0 ? s_cur[qq] : z[qq] + bt * s_prev[qq]; };
                    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                        long long c = cell_at(j, t, t0);
                        T sc_ = sval(c);
                        if (it > 0) s_cur[c] = sc_;
                        T qv = ax_ref32(S, D, c, sc_, sval);
                        q[c] = qv;
                        a0 += (double)sc_ * (double)qv;
                    }
                }
                put3(j, a0, 0.0, 0.0);
            }
            if (!count_barrier(A.bar, S.dev_error, ++epoch, tmo)) return;
            reduce(1, [&](int, SceneLocal& P, double sq, double, double) -> bool {
                if (P.inner_done) return false;
                P.alpha = sq != 0.0 ? P.rho / sq : 0.0;
                float sq32 = (float)sq;
                P.alpha32 = sq32 != 0.0f ? P.rho32 / sq32 : 0.0f;
                return true;
            });
            for (int j = 0;; ++j) {
                int s;
                long long t0, t1;
                if (!chunk_of(j, s, t0, t1)) break;
                double a0 = 0.0, a1 = 0.0;
                if (!L[s].inner_done) {
                    const T al = (T)L[s].alpha32;
                    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                        long long c = cell_at(j, t, t0);
                        T sv = s_cur[c];
                        T xv = x[c] + al * sv;
                        T rv = r[c] + (-al) * q[c];
                        x[c] = xv;
                        r[c] = rv;
                        a0 += (double)rv * (double)rv;
                        T zv = precond(c, rv);
                        z[c] = zv;
                        a1 += (double)zv * (double)rv;
                    }
                }
                put3(j, a0, a1, 0.0);
            }
            if (!count_barrier(A.bar, S.dev_error, ++epoch, tmo)) return;
            int act = reduce(2, [&](int s, SceneLocal& P, double rr, double rho2, double) -> bool {
                if (P.inner_done) return false;
                const int n = S.scenes[s].n;
                P.iters += 1;
                P.rr = rr;
                const int cap = A.max_iters > 0 ? A.max_iters : n * n * n;
                bool conv = (float)rr <= (float)P.target;
                if (conv || P.iters >= cap) {
                    P.inner_done = 1;
                    P.done = 1;
                    P.converged = conv;
                    return false;
                }
                P.beta = P.rho != 0.0 ? rho2 / P.rho : 0.0;
                P.rho = rho2;
                float r32 = (float)rho2;
                P.beta32 = P.rho32 != 0.0f ? r32 / P.rho32 : 0.0f;
                P.rho32 = r32;
                return true;
            });
            if (act == 0) break;
        }
        break;
    }

    // ---- results: final per-scene state and totals (block 0), fp32 pressure ---------------
    if (blockIdx.x == 0) {
        for (int s = threadIdx.x; s < k; s += blockDim.x) {
            const SceneLocal& P = L[s];
            PcgScene o = load_sc(A.sc + s);
            o.bb = P.bb;
            o.rr = P.rr;
            o.rho = P.rho;
            o.alpha = P.alpha;
            o.beta = P.beta;
            o.rr_out = P.rr_out;
            o.target = P.target;
            o.iters = P.iters;
            o.outer = P.outer;
            o.done = P.done;
            o.inner_done = P.inner_done;
            o.converged = P.converged;
            A.sc[s] = o;
            PcgTotals& Tt = A.totals[s];
            Tt.solves += 1;
            Tt.iterations += P.iters;
            Tt.outer += MODE == kMixed ? P.outer : 1;
            Tt.cell_iterations += (double)P.nf * (double)P.iters;
            Tt.cell_outer += (double)P.nf * (double)(MODE == kMixed ? P.outer : 1);
            Tt.not_converged += P.converged ? 0 : 1;
        }
    }
    if (MODE != kRef32) {
        // P64 of this block's cells was written by this block above (no barrier needed)
        for (int j = 0;; ++j) {
            int s;
            long long t0, t1;
            if (!chunk_of(j, s, t0, t1)) break;
            for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                long long c = cell_at(j, t, t0);
                S.P[c] = (float)S.P64[c];
            }
        }
    }
}

template <int MODE>
static cudaError_t coop_launch(const PcgArgs& A, int nblocks, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)nblocks);
    cfg.blockDim = dim3(kPcgThreads);
    cfg.dynamicSmemBytes = brick_dyn_smem();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_pcg<MODE>, A);
    count_launch();
    return e;
}

template <int MODE>
static cudaError_t coop_launch_fast(const PcgArgs& A, int nblocks, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)nblocks);
    cfg.blockDim = dim3(kPcgThreads);
    cfg.dynamicSmemBytes = fast_dyn_smem(MODE);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_pcg_fast<MODE>, A);
    count_launch();
    return e;
}

// With the reference preconditioner and few enough scenes the fast kernel solves and the
// general kernel returns at once; with an ordered preconditioner it is the other way round
// (the choice is made on the device, from the preparation's FLUID-cell scan).
cudaError_t launch_pcg_solve(const PcgArgs& A, int nblocks, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    if (A.fast) {
        switch (A.mode) {
            case kRef32: e = coop_launch_fast<kRef32>(A, nblocks, st); break;
            case kFp64: e = coop_launch_fast<kFp64>(A, nblocks, st); break;
            default: e = coop_launch_fast<kMixed>(A, nblocks, st); break;
        }
        if (e != cudaSuccess) return e;
        if (A.precond != ARIEL_PRECOND_MIC0 && !A.may_be_ordered) return e;
    }
    switch (A.mode) {
        case kRef32: return coop_launch<kRef32>(A, nblocks, st);
        case kFp64: return coop_launch<kFp64>(A, nblocks, st);
        default: return coop_launch<kMixed>(A, nblocks, st);
    }
}

int pcg_max_blocks(int device, int mode, int per_sm_cap) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e;
    int per_fast = 0;
    const int dyn = (int)fast_dyn_smem(mode);
    const int bdyn = (int)brick_dyn_smem();
    if (mode == kRef32) {
        cudaFuncSetAttribute(k_pcg_fast<kRef32>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
        cudaFuncSetAttribute(k_pcg<kRef32>, cudaFuncAttributeMaxDynamicSharedMemorySize, bdyn);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg<kRef32>, kPcgThreads, bdyn);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_fast, k_pcg_fast<kRef32>, kPcgThreads, dyn);
    } else if (mode == kFp64) {
        cudaFuncSetAttribute(k_pcg_fast<kFp64>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
        cudaFuncSetAttribute(k_pcg<kFp64>, cudaFuncAttributeMaxDynamicSharedMemorySize, bdyn);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg<kFp64>, kPcgThreads, bdyn);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_fast, k_pcg_fast<kFp64>, kPcgThreads, dyn);
    } else {
        cudaFuncSetAttribute(k_pcg_fast<kMixed>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
        cudaFuncSetAttribute(k_pcg<kMixed>, cudaFuncAttributeMaxDynamicSharedMemorySize, bdyn);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg<kMixed>, kPcgThreads, bdyn);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_fast, k_pcg_fast<kMixed>, kPcgThreads, dyn);
    }
    if (per_fast < per) per = per_fast;  // one grid size serves both kernels
    if (e != cudaSuccess || per < 1) per = 1;
    // The default of two blocks per SM covers the FLUID chunks of the bench sizes; more blocks
    // add arrivals to every grid barrier.
    int cap = per_sm_cap > 0 ? per_sm_cap : 2;
    return sms * (per < cap ? per : cap);
}

cudaError_t launch_barrier_selftest(Barrier* bar, int* err, unsigned long long timeout_ns, cudaStream_t st) {
    cudaMemsetAsync(bar, 0, sizeof(Barrier), st);
    k_barrier_selftest<<<2, 32, 0, st>>>(bar, err, timeout_ns);
    count_launch();
    return cudaGetLastError();
}

size_t brick_dyn_smem() {
    return (size_t)2 * kBrickMaxExt * 8 + (size_t)kBrickMaxCells * 8 + (size_t)(kBrickMaxLevels + 1) * 4 +
           (size_t)kBrickMaxCells * 2 + (size_t)kBrickMaxExt;
}

bool brick_shape_ok(int bx, int by, int bz) {
    return bx >= 1 && by >= 1 && bz >= 1 && bx <= 31 && by <= 31 && bz <= 63 && bx * by * bz <= kBrickMaxCells &&
           (bx + 1) * (by + 1) * (bz + 1) <= kBrickMaxExt && bx + by + bz - 2 <= kBrickMaxLevels;
}

}  // namespace ariel
