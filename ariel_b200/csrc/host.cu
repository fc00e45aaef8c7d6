// host.cu -- host orchestration behind the C ABI (include/ariel.h).
//
// An `ariel_sim` owns k >= 1 scenes laid out over packed particle / cell / face index spaces
// (see common.cuh).  The FlipSim step order of the reference (src/sim/flip.cpp:92-128) is
// reproduced stage by stage; a whole step is captured once into a CUDA graph and replayed.
// Frame counters, the resampling schedule and the pressure solve's stopping decisions all live
// on the device, so a step needs no host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <zlib.h>

#include "sim.cuh"

using namespace ariel;

namespace {

thread_local char g_last_error[256] = "";

#define ARIEL_CUDA(call)                                                                    \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) return ::ariel::hostimpl::map_cuda_error(e_, #call);         \
    } while (0)

#define ARIEL_TRY(x)                          \
    do {                                      \
        ariel_status st_ = (x);               \
        if (st_ != ARIEL_OK) return st_;      \
    } while (0)

inline float hmin(float x, float y) { return (y < x) ? y : x; }  // glm::min
inline float hmax(float x, float y) { return (x < y) ? y : x; }  // glm::max

// FlipSim::Init's density normaliser (flip.cpp:42-70): density of a 10x10x10 lattice of
// unit-mass FLUID particles at spacing density/maxd, max over the lattice.  One block per
// scene; each particle gathers the lattice particles of its 27 cells in cell order, then in
// particle order inside a cell -- the order ParticleGrid::Sort gives them.
__global__ void k_max_density(SceneDev* scenes, int k) {
    const int s = blockIdx.x;
    if (s >= k) return;
    SceneDev& D = scenes[s];
    __shared__ float px[1000], py[1000], pz[1000];
    __shared__ int pc[1000];
    __shared__ float best[1024];
    const float maxd = D.maxd;
    const float h = D.density / maxd;
    const int n = D.n;
    for (int t = threadIdx.x; t < 1000; t += blockDim.x) {
        int i = t / 100, j = (t / 10) % 10, kk = t % 10;
        px[t] = ((float)i + 0.5f) * h;
        py[t] = ((float)j + 0.5f) * h;
        pz[t] = ((float)kk + 0.5f) * h;
        int ci = cell_coord(maxd, px[t]), cj = cell_coord(maxd, py[t]), ck = cell_coord(maxd, pz[t]);
        pc[t] = (ci * n + cj) * n + ck;
    }
    __syncthreads();
    float dens = 0.0f;
    const int t = threadIdx.x;
    if (t < 1000) {
        int ci = cell_coord(maxd, px[t]), cj = cell_coord(maxd, py[t]), ck = cell_coord(maxd, pz[t]);
        const float hk = D.dens_h;
        float weightsum = 0.0f;
        for (int sx = ci - 1; sx <= ci + 1; ++sx) {
            if (sx < 0 || sx > n - 1) continue;
            for (int sy = cj - 1; sy <= cj + 1; ++sy) {
                if (sy < 0 || sy > n - 1) continue;
                for (int sz = ck - 1; sz <= ck + 1; ++sz) {
                    if (sz < 0 || sz > n - 1) continue;
                    int cell = (sx * n + sy) * n + sz;
                    for (int m = 0; m < 1000; ++m) {
                        if (pc[m] != cell) continue;
                        float sqd = sqrlength(px[m], py[m], pz[m], px[t], py[t], pz[t]);
                        float weight = 1.0f * smooth_k(sqd, hk);
                        weightsum = weightsum + weight;
                    }
                }
            }
        }
        dens = weightsum / 1.0f;
    }
    best[t] = t < 1000 ? dens : 0.0f;
    __syncthreads();
    if (t == 0) {
        float m = 0.0f;
        for (int i = 0; i < 1000; ++i) m = gmax(m, best[i]);
        D.max_density = m;
    }
}

// dst[i] = (src ? src[i] : 0) + add: places a scene's solid bins at their packed offset.
__global__ void k_u32_offset(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, long long n, uint32_t add) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = (src ? src[i] : 0u) + add;
}

cudaError_t launch_u32_offset(uint32_t* dst, const uint32_t* src, long long n, uint32_t add, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_u32_offset<<<grid_for(n), kBlock, 0, st>>>(dst, src, n, add);
    count_launch();
    return cudaGetLastError();
}

template <class T>
ariel_status dalloc(ariel_sim* s, T** p, size_t count, bool keep = false) {
    *p = nullptr;
    if (count == 0) count = 1;
    void* q = nullptr;
    const size_t bytes = count * sizeof(T);
    cudaError_t e = s->pool ? cudaMallocFromPoolAsync(&q, bytes, s->pool, s->stream) : cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ARIEL_ERR_OOM;
    }
    s->bufs.push_back(DeviceBuf{q, bytes, keep, s->pool != nullptr});
    *p = (T*)q;
    return ARIEL_OK;
}

void destroy_graphs(ariel_sim* s) {
    for (int i = 0; i < 3; ++i) {
        if (s->graph[i]) cudaGraphExecDestroy(s->graph[i]);
        s->graph[i] = nullptr;
        s->graph_tried[i] = false;
    }
}

void free_bufs(ariel_sim* s, bool scratch_only) {
    destroy_graphs(s);
    std::vector<DeviceBuf> left;
    for (auto& b : s->bufs) {
        if (scratch_only && b.keep) {
            left.push_back(b);
            continue;
        }
        if (b.pooled)
            cudaFreeAsync(b.p, s->stream);
        else
            cudaFree(b.p);
    }
    s->bufs.swap(left);
}

void free_all(ariel_sim* s) { free_bufs(s, false); }

// Buffer sizes of one packed layout.
struct Layout {
    long long k = 0, np = 0, nc = 0, nf = 0, ns = 0, maxch = 0, nbricks = 0, mesh_nodes = 0, mesh_tris = 0;
    bool any_solid = false;
    bool any_reseed = false;
    int mode = kRef32;
};

// Brick of the ordered wavefront sweeps.
void sweep_brick(const AsimParams& p, int& bx, int& by, int& bz) {
    bx = p.sweep_brick[0];
    by = p.sweep_brick[1];
    bz = p.sweep_brick[2];
    if (bx == 0 && by == 0 && bz == 0) {
        // fastest of the autotuner's candidates at 128^3 (MIC(0), MIXED)
        bx = 12;
        by = 12;
        bz = 12;
    }
}

// Particle-count bounds of the reseeding pass (0 selects the defaults 6 and 10).
void reseed_bounds(const AsimParams& p, int& lo, int& hi) {
    lo = p.reseed_min > 0 ? p.reseed_min : 6;
    hi = p.reseed_max > 0 ? p.reseed_max : 10;
}

long long bricks_of(int n, int bx, int by, int bz) {
    return (long long)((n + bx - 1) / bx) * ((n + by - 1) / by) * ((n + bz - 1) / bz);
}

int mode_of(const AsimParams& p) {
    return p.precision == ARIEL_PREC_FP64 ? kFp64 : (p.precision == ARIEL_PREC_MIXED ? kMixed : kRef32);
}

// The allocation list of build_state, in bytes (each buffer rounded to 256 bytes as the
// allocators place them).  Kept next to build_state; a GPU test holds the two equal.
long long layout_bytes(const Layout& L) {
    long long total = 0;
    auto add = [&](long long count, long long esize) {
        long long b = std::max(1ll, count) * esize;
        total += (b + 255) / 256 * 256;
    };
    const long long k = L.k, np = L.np, nc = L.nc, nf = L.nf;
    add(k, sizeof(SceneDev));
    for (int i = 0; i < 3; ++i) add(k + 1, 8);
    add(np, 16);
    add(np, 16);
    if (L.any_solid) {
        add(np, 16);
        add(np, 16);
    }
    add(np, 4);  // key
    add(np, 4);  // off
    add(nc, 4);  // count
    add(nc + 1, 4);  // start
    add(np, 4);   // sid
    add(np, 16);  // spos4
    add(np, 16);  // svel4
    add(np, 16);  // gpos4
    add(np, 4);   // dens
    add(np, 4);   // dens by id
    add(6 * np, 4);  // host I/O staging
    add(nc + 1, 4);  // solid_start
    add(nc, 1);      // flags
    add(nc, 4);      // L
    add(nc, 4);      // D
    add(nc, 4);      // P
    add(nc, 8);      // P64
    add(nf, 4);      // u
    add(nf, 4);      // pu
    add(1, 4);       // dev_error
    add((long long)scan_tmp_bytes(nc), 1);
    if (L.any_reseed) {
        add(nc, 4);      // reseed: excess
        add(nc + 1, 4);  // its scan
        add(nc, 4);      // deficit
        add(nc + 1, 4);  // its scan
    }
    add(nc, 4);      // FLUID list
    add(nc, 16);     // FLUID-list records
    add(k + 1, 8);
    add(k + 1, 8);
    add(nc, 4);      // flpred
    add(nc + 1, 4);  // flscan
    add(nc, 1);      // mask
    add(nc, 8);      // diag
    add(nc, 8);      // pc64
    add(nc, 4);      // pc32
    const long long vb = L.mode == kFp64 ? 8 : 4;
    for (int i = 0; i < 8; ++i) add(nc, vb);
    for (int i = 0; i < 3; ++i) add((i < 2 ? 4 : 2) * nc, vb);
    if (L.mode == kMixed) {
        add(nc, 8);
        add(nc, 4);
    }
    add(3 * std::max(1ll, L.maxch), 8);
    add(L.nbricks, 16);  // brick list
    add(k + 1, 4);       // brick bases
    add(L.nbricks, 4);   // brick flags
    add(k, sizeof(PcgScene));
    add(k, sizeof(PcgTotals));
    add(1, sizeof(PcgCtl));
    add(1, sizeof(Barrier));
    add(L.ns, 16);  // solid_pos
    add(L.mesh_nodes, sizeof(MeshNode));
    add(L.mesh_tris, sizeof(MeshTri));
    return total;
}

}  // namespace

namespace ariel {
namespace hostimpl {

ariel_status map_cuda_error(cudaError_t e, const char* what) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return ARIEL_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return ARIEL_ERR_NO_DEVICE;
    return ARIEL_ERR_CUDA;
}

// Every copy goes through the handle's stream (non-blocking, so the legacy default stream would
// not be ordered with the kernels) and is waited for before returning.
cudaError_t copy_sync(cudaStream_t st, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

// Scene::GenerateParticles (src/scene/scene.cpp:257-360) for box liquids and analytic sphere
// solids, placed in lexicographic (i,j,k) lattice order: liquid particles first, then solids
// (scene.cpp:349-354).  Liquid particles may be jittered inside their lattice sub-cell by
// Philox4x32-10 keyed by (seed, particle index, box).
void generate_particles(const AsimSceneDesc& d, HostParticles& out) {
    const int n = d.dim;
    const float maxdim = (float)n;
    const float thickness = 1.0f / maxdim;
    const float density = d.density;
    const float w = density * thickness;
    const uint32_t k0 = (uint32_t)d.seed, k1 = (uint32_t)(d.seed >> 32);
    std::shared_ptr<SceneMeshes> M;
    if (scene_meshes(d, M) != ARIEL_OK) M = std::make_shared<SceneMeshes>();
    const MeshNode* mn = M->nodes.empty() ? nullptr : M->nodes.data();
    const MeshTri* mt = M->tris.empty() ? nullptr : M->tris.data();
    auto inside_solid = [&](float x, float y, float z) {
        for (int s = 0; s < d.n_solid; ++s) {
            float cx = d.solid[s].center[0] * maxdim, cy = d.solid[s].center[1] * maxdim,
                  cz = d.solid[s].center[2] * maxdim, r = d.solid[s].radius * maxdim;
            float dx = x - cx, dy = y - cy, dz = z - cz;
            float dd = (dx * dx + dy * dy) + dz * dz;
            if (dd < r * r) return true;
        }
        return mesh_inside_bits(mn, mt, make_float3(x, y, z)) != 0u;
    };
    out = HostParticles{};
    for (int l = 0; l < d.n_liquid; ++l) {
        const AsimBox& bx = d.liquid[l];
        float lminx = hmax(std::floor(bx.lo[0] * maxdim), 0.0f) / density;
        float lminy = hmax(std::floor(bx.lo[1] * maxdim), 0.0f) / density;
        float lminz = hmax(std::floor(bx.lo[2] * maxdim), 0.0f) / density;
        float lmaxx = hmin(std::ceil(bx.hi[0] * maxdim), maxdim + 1.0f) / density;
        float lmaxy = hmin(std::ceil(bx.hi[1] * maxdim), maxdim + 1.0f) / density;
        float lmaxz = hmin(std::ceil(bx.hi[2] * maxdim), maxdim + 1.0f) / density;
        for (unsigned i = (unsigned)lminx; i < (unsigned)lmaxx; ++i)
            for (unsigned j = (unsigned)lminy; (float)j < lmaxy; ++j)
                for (unsigned k = (unsigned)lminz; (float)k < lmaxz; ++k) {
                    float cx = (i * w) + (w / 2.0f), cy = (j * w) + (w / 2.0f), cz = (k * w) + (w / 2.0f);
                    float wx = cx * maxdim, wy = cy * maxdim, wz = cz * maxdim;
                    bool inside = wx > bx.lo[0] * maxdim && wx < bx.hi[0] * maxdim && wy > bx.lo[1] * maxdim &&
                                  wy < bx.hi[1] * maxdim && wz > bx.lo[2] * maxdim && wz < bx.hi[2] * maxdim;
                    if (!inside || inside_solid(wx, wy, wz)) continue;
                    float px = cx, py = cy, pz = cz;
                    if (d.jitter > 0.0f) {
                        uint32_t id = (uint32_t)out.pos4.size();
                        uint4 rv = philox4x32_10(make_uint4(id, (uint32_t)l, 0u, kTagSeed), k0, k1);
                        float ux = (float)(rv.x >> 8) * (1.0f / 16777216.0f);
                        float uy = (float)(rv.y >> 8) * (1.0f / 16777216.0f);
                        float uz = (float)(rv.z >> 8) * (1.0f / 16777216.0f);
                        px = (i * w) + (ux * w);
                        py = (j * w) + (uy * w);
                        pz = (k * w) + (uz * w);
                    }
                    out.pos4.push_back(make_float4(px, py, pz, 1.0f));
                    out.vel4.push_back(pack_vel(bx.vel[0], bx.vel[1], bx.vel[2], ARIEL_FLUID));
                }
    }
    for (int s = 0; s < d.n_solid; ++s) {
        float cx = d.solid[s].center[0] * maxdim, cy = d.solid[s].center[1] * maxdim,
              cz = d.solid[s].center[2] * maxdim, r = d.solid[s].radius * maxdim;
        float lminx = hmax(std::floor(cx - r), 0.0f) / density;
        float lminy = hmax(std::floor(cy - r), 0.0f) / density;
        float lminz = hmax(std::floor(cz - r), 0.0f) / density;
        float lmaxx = hmin(std::ceil(cx + r), maxdim + 1.0f) / density;
        float lmaxy = hmin(std::ceil(cy + r), maxdim + 1.0f) / density;
        float lmaxz = hmin(std::ceil(cz + r), maxdim + 1.0f) / density;
        for (unsigned i = (unsigned)lminx; i < (unsigned)lmaxx; ++i)
            for (unsigned j = (unsigned)lminy; (float)j < lmaxy; ++j)
                for (unsigned k = (unsigned)lminz; (float)k < lmaxz; ++k) {
                    float px = (i * w) + (w / 2.0f), py = (j * w) + (w / 2.0f), pz = (k * w) + (w / 2.0f);
                    float wx = px * maxdim - cx, wy = py * maxdim - cy, wz = pz * maxdim - cz;
                    float dd = (wx * wx + wy * wy) + wz * wz;
                    if (!(dd < r * r)) continue;
                    out.pos4.push_back(make_float4(px, py, pz, 10.0f));
                    out.vel4.push_back(pack_vel(0.0f, 0.0f, 0.0f, ARIEL_SOLID));
                }
    }
    // solid meshes after the spheres, each over the lattice of its world bounding box
    // (scene.cpp:307-332), keeping the points the mesh itself contains
    for (size_t m = 0; m < M->lo.size(); ++m) {
        const float3 lo = M->lo[m], hi = M->hi[m];
        float lminx = hmax(std::floor(lo.x), 0.0f) / density;
        float lminy = hmax(std::floor(lo.y), 0.0f) / density;
        float lminz = hmax(std::floor(lo.z), 0.0f) / density;
        float lmaxx = hmin(std::ceil(hi.x), maxdim + 1.0f) / density;
        float lmaxy = hmin(std::ceil(hi.y), maxdim + 1.0f) / density;
        float lmaxz = hmin(std::ceil(hi.z), maxdim + 1.0f) / density;
        for (unsigned i = (unsigned)lminx; i < (unsigned)lmaxx; ++i)
            for (unsigned j = (unsigned)lminy; (float)j < lmaxy; ++j)
                for (unsigned k = (unsigned)lminz; (float)k < lmaxz; ++k) {
                    float px = (i * w) + (w / 2.0f), py = (j * w) + (w / 2.0f), pz = (k * w) + (w / 2.0f);
                    const uint32_t bits = mesh_inside_bits(mn, mt, make_float3(px * maxdim, py * maxdim, pz * maxdim));
                    if (!((bits >> m) & 1u)) continue;
                    out.pos4.push_back(make_float4(px, py, pz, 10.0f));
                    out.vel4.push_back(pack_vel(0.0f, 0.0f, 0.0f, ARIEL_SOLID));
                }
    }
    bin_solids(d, out);
}

// Static SOLID particles binned by cell, id order inside a cell: their positions never change
// (only FLUID particles are moved by any stage of the step), so the bins are built once.
void bin_solids(const AsimSceneDesc& d, HostParticles& hp) {
    hp.solid_pos.clear();
    hp.solid_start.clear();
    hp.binned = true;
    const long long n = d.dim;
    const float maxd = (float)n;
    std::vector<std::pair<long long, float4>> sol;
    for (size_t p = 0; p < hp.pos4.size(); ++p) {
        if (type_bits(hp.vel4[p]) != ARIEL_SOLID) continue;
        const float4& q = hp.pos4[p];
        auto cc = [&](float x) { return (long long)(int)hmax(0.0f, hmin((float)(int)maxd - 1.0f, (float)(int)maxd * x)); };
        sol.push_back({(cc(q.x) * n + cc(q.y)) * n + cc(q.z), q});
    }
    if (sol.empty()) return;
    std::stable_sort(sol.begin(), sol.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    const long long ncell = n * n * n;
    hp.solid_start.assign(ncell + 1, 0);
    hp.solid_pos.resize(sol.size());
    for (size_t i = 0; i < sol.size(); ++i) {
        hp.solid_start[sol[i].first + 1]++;
        hp.solid_pos[i] = sol[i].second;
    }
    for (long long c = 0; c < ncell; ++c) hp.solid_start[c + 1] += hp.solid_start[c];
}

SceneDev make_scene(const AsimSceneDesc& d, const AsimParams& p) {
    SceneDev D{};
    D.n = d.dim;
    D.n_forces = d.n_forces;
    D.n_spheres = d.n_solid;
    D.n_meshes = d.n_mesh;
    D.frame = 0;
    D.maxd = (float)d.dim;
    D.density = d.density;
    D.dt = d.stepsize;
    D.picflip = p.picflip;
    D.max_density = 1.0f;
    D.dens_h = 4.0f * d.density / D.maxd;
    float n0 = 1.0f / (d.density * d.density * d.density);
    D.sdf0 = 0.2f * n0;
    D.h = 1.0f / D.maxd;
    float nn = (float)d.dim;
    D.ax_h = 1.0f / (nn * nn);
    D.resample_re = d.density / D.maxd;
    D.pushout_re = 1.5f * d.density / D.maxd;
    D.subcell = p.subcell;
    for (int j = 0; j < d.n_forces && j < ARIEL_MAX_FORCES; ++j)
        for (int a = 0; a < 3; ++a) D.fdt[j][a] = d.forces[j][a] * d.stepsize;
    for (int i = 0; i < d.n_solid && i < ARIEL_MAX_SPHERES; ++i)
        D.sphere[i] = make_float4(d.solid[i].center[0] * D.maxd, d.solid[i].center[1] * D.maxd,
                                  d.solid[i].center[2] * D.maxd, d.solid[i].radius * D.maxd);
    D.rng_seed = p.rng_seed;
    D.resample_every = p.resample_every;
    D.reseed_every = p.reseed_every;
    reseed_bounds(p, D.reseed_min, D.reseed_max);
    auto pow2 = [](float v, float* inv) {
        int e = 0;
        float m = std::frexp(v, &e);
        *inv = 1.0f / v;
        return (m == 0.5f && std::isfinite(*inv) && *inv * v == 1.0f) ? 1 : 0;
    };
    const double dn = (double)d.dim;
    D.inv_n = 1.0 / dn;
    D.inv_n1 = 1.0 / (dn + 1.0);
    D.inv_nn = 1.0 / (dn * dn);
    D.inv_nn1 = 1.0 / (dn * (dn + 1.0));
    D.dens_pow2 = pow2(D.dens_h * D.dens_h, &D.dens_inv_hh);
    D.re_pow2 = pow2(D.resample_re * D.resample_re, &D.re_inv_hh);
    return D;
}

ariel_status validate(const AsimSceneDesc& d) {
    if (d.dim < 2 || d.dim > 1024) return ARIEL_ERR_INVALID_ARG;
    if (!(d.density > 0.0f) || !(d.stepsize > 0.0f)) return ARIEL_ERR_INVALID_ARG;
    if (d.n_forces < 0 || d.n_forces > ARIEL_MAX_FORCES) return ARIEL_ERR_INVALID_ARG;
    if (d.n_liquid < 0 || d.n_liquid > ARIEL_MAX_BOXES) return ARIEL_ERR_INVALID_ARG;
    if (d.n_solid < 0 || d.n_solid > ARIEL_MAX_SPHERES) return ARIEL_ERR_INVALID_ARG;
    if (!meshes_valid(d)) return ARIEL_ERR_INVALID_ARG;
    if ((long long)d.dim * d.dim * d.dim > (1ll << 30)) return ARIEL_ERR_INVALID_ARG;
    return ARIEL_OK;
}

long long state_bytes(const std::vector<AsimSceneDesc>& descs, const std::vector<long long>& particles,
                      const std::vector<long long>& solids, const AsimParams& prm) {
    Layout L;
    L.k = (long long)descs.size();
    L.mode = mode_of(prm);
    L.any_reseed = prm.reseed_every > 0;
    int bx, by, bz;
    sweep_brick(prm, bx, by, bz);
    for (size_t i = 0; i < descs.size(); ++i) {
        const long long n = descs[i].dim;
        L.nbricks += bricks_of((int)n, bx, by, bz);
        L.np += particles[i];
        L.nc += n * n * n;
        L.nf += 3 * n * n * (n + 1);
        L.ns += solids[i];
        L.maxch += chunk_bound(n * n * n);
        if (descs[i].n_solid > 0 || descs[i].n_mesh > 0) L.any_solid = true;
        long long mn = 0, mt = 0;
        mesh_counts(descs[i], mn, mt);
        L.mesh_nodes += mn;
        L.mesh_tris += mt;
    }
    return layout_bytes(L);
}

void free_scratch(ariel_sim* s) { free_bufs(s, true); }

ariel_status build_state(ariel_sim* s, std::vector<HostParticles>& hp, const ariel_sim* src,
                         const std::vector<int>* src_idx, const std::vector<DeviceParticles>* staged) {
    free_all(s);
    const int k = s->k;
    auto from_src = [&](int i) { return src && src_idx && (*src_idx)[i] >= 0; };
    auto from_staged = [&](int i) { return !from_src(i) && staged && (*staged)[i].valid; };
    for (int i = 0; i < k; ++i)
        if (!from_src(i) && !from_staged(i) && !hp[i].binned) bin_solids(s->descs[i], hp[i]);
    s->ppref.assign(k + 1, 0);
    s->cpref.assign(k + 1, 0);
    s->fpref.assign(k + 1, 0);
    s->spref.assign(k + 1, 0);
    s->any_solid = false;
    long long maxch = 0;
    for (int i = 0; i < k; ++i) {
        long long n = s->descs[i].dim;
        long long cnt, scnt;
        if (from_src(i)) {
            const int j = (*src_idx)[i];
            cnt = src->ppref[j + 1] - src->ppref[j];
            scnt = src->spref[j + 1] - src->spref[j];
        } else if (from_staged(i)) {
            cnt = (*staged)[i].np;
            scnt = (*staged)[i].ns;
        } else {
            cnt = (long long)hp[i].pos4.size();
            scnt = (long long)hp[i].solid_pos.size();
        }
        s->ppref[i + 1] = s->ppref[i] + cnt;
        s->cpref[i + 1] = s->cpref[i] + n * n * n;
        s->fpref[i + 1] = s->fpref[i] + 3 * n * n * (n + 1);
        s->spref[i + 1] = s->spref[i] + scnt;
        s->sh[i].p_begin = s->ppref[i];
        s->sh[i].p_end = s->ppref[i + 1];
        s->sh[i].c_begin = s->cpref[i];
        s->sh[i].f_begin = s->fpref[i];
        if (s->descs[i].n_solid > 0 || s->descs[i].n_mesh > 0) s->any_solid = true;
        maxch += chunk_bound(n * n * n);
    }
    s->np = s->ppref[k];
    s->nc = s->cpref[k];
    s->nf = s->fpref[k];
    if (s->np >= (1ll << 31) || s->nc >= (1ll << 31) || s->spref[k] >= (1ll << 32)) return ARIEL_ERR_INVALID_ARG;
    const long long np = s->np, nc = s->nc, nf = s->nf;
    DevState& S = s->S;
    S = DevState{};
    S.k = k;
    S.any_solid = s->any_solid;
    S.np = np;
    S.nc = nc;
    S.nf = nf;
    // The order and sizes of these allocations are mirrored by layout_bytes.
    ARIEL_TRY(dalloc(s, &s->d_scenes, k, true));
    ARIEL_TRY(dalloc(s, &s->d_ppref, k + 1));
    ARIEL_TRY(dalloc(s, &s->d_cpref, k + 1));
    ARIEL_TRY(dalloc(s, &s->d_fpref, k + 1));
    S.scenes = s->d_scenes;
    S.p_pref = s->d_ppref;
    S.c_pref = s->d_cpref;
    S.f_pref = s->d_fpref;
    ARIEL_TRY(dalloc(s, &S.pos4, np, true));
    ARIEL_TRY(dalloc(s, &S.vel4, np, true));
    if (s->any_solid) {
        ARIEL_TRY(dalloc(s, &S.pt4, np));
        ARIEL_TRY(dalloc(s, &S.ut4, np));
    }
    ARIEL_TRY(dalloc(s, &S.key, np));
    ARIEL_TRY(dalloc(s, &S.off, np));
    ARIEL_TRY(dalloc(s, &S.count, nc));
    ARIEL_TRY(dalloc(s, &S.start, nc + 1));
    ARIEL_TRY(dalloc(s, &S.sid, np));
    ARIEL_TRY(dalloc(s, &S.spos4, np));
    ARIEL_TRY(dalloc(s, &S.svel4, np));
    ARIEL_TRY(dalloc(s, &S.gpos4, np));
    ARIEL_TRY(dalloc(s, &S.dens, np));
    ARIEL_TRY(dalloc(s, &s->d_dens_id, np));
    ARIEL_TRY(dalloc(s, &s->d_stage, 6 * (size_t)np));
    ARIEL_TRY(dalloc(s, &S.solid_start, nc + 1, true));
    ARIEL_TRY(dalloc(s, &S.flags, nc));
    ARIEL_TRY(dalloc(s, &S.L, nc));
    ARIEL_TRY(dalloc(s, &S.D, nc));
    ARIEL_TRY(dalloc(s, &S.P, nc, true));
    ARIEL_TRY(dalloc(s, &S.P64, nc, true));
    ARIEL_TRY(dalloc(s, &S.u, nf));
    ARIEL_TRY(dalloc(s, &S.pu, nf));
    ARIEL_TRY(dalloc(s, &S.dev_error, 1));
    size_t st_bytes = scan_tmp_bytes(nc);
    char* tmp = nullptr;
    ARIEL_TRY(dalloc(s, &tmp, st_bytes));
    s->scan_tmp = tmp;
    S.any_reseed = s->prm.reseed_every > 0;
    if (S.any_reseed) {
        ARIEL_TRY(dalloc(s, &S.rs_excess, nc));
        ARIEL_TRY(dalloc(s, &S.rs_escan, nc + 1));
        ARIEL_TRY(dalloc(s, &S.rs_deficit, nc));
        ARIEL_TRY(dalloc(s, &S.rs_dscan, nc + 1));
    }
    // pressure solve
    PcgArgs& A = s->PA;
    A = PcgArgs{};
    s->mode = mode_of(s->prm);
    A.mode = s->mode;
    A.precond = s->prm.precond;
    A.stop_rule = s->prm.stop_rule;
    A.max_iters = s->prm.max_iters;
    A.max_outer = s->prm.max_outer > 0 ? s->prm.max_outer : 8;
    A.fast = (k <= 128 && A.precond == ARIEL_PRECOND_REF) ? 1 : 0;
    // the reference preconditioner needs the ordered kernel only in the rare PRef == 1 case,
    // which only the device knows; keep launching it (it returns at once when not needed)
    A.may_be_ordered = 1;
    A.tol = s->prm.tol;
    A.inner_tol = s->prm.inner_tol > 0 ? s->prm.inner_tol : 1e-6;
    A.tau = s->prm.mic_tau;
    A.sigma = s->prm.mic_sigma;
    double tmo_ms = s->prm.barrier_timeout_ms > 0 ? s->prm.barrier_timeout_ms : 2000.0;
    A.timeout_ns = (unsigned long long)(tmo_ms * 1.0e6);
    uint32_t* fl = nullptr;
    long long *flp = nullptr, *chp = nullptr;
    ARIEL_TRY(dalloc(s, &fl, nc));
    ARIEL_TRY(dalloc(s, &flp, k + 1));
    ARIEL_TRY(dalloc(s, &chp, k + 1));
    A.fl = fl;
    ARIEL_TRY(dalloc(s, &A.rec, nc));
    A.fl_pref = flp;
    A.ch_pref = chp;
    ARIEL_TRY(dalloc(s, &s->flpred, nc));
    ARIEL_TRY(dalloc(s, &s->flscan, nc + 1));
    ARIEL_TRY(dalloc(s, &A.mask, nc));
    ARIEL_TRY(dalloc(s, &A.diag, nc));
    ARIEL_TRY(dalloc(s, &A.pc64, nc));
    ARIEL_TRY(dalloc(s, &A.pc32, nc));
    const size_t vb = s->mode == kFp64 ? 8 : 4;
    char* v[8];
    for (int i = 0; i < 8; ++i) ARIEL_TRY(dalloc(s, &v[i], vb * (size_t)nc));
    A.r = v[0];
    A.z = v[1];
    A.s0 = v[2];
    A.s1 = v[3];
    A.q = v[4];
    A.ordq = v[5];
    A.u = v[6];
    A.p = v[7];
    char* w4[3];
    for (int i = 0; i < 3; ++i) ARIEL_TRY(dalloc(s, &w4[i], (i < 2 ? 4 : 2) * vb * (size_t)nc));
    A.va0 = w4[0];
    A.va1 = w4[1];
    A.vb = w4[2];
    if (s->mode == kMixed) {
        ARIEL_TRY(dalloc(s, &A.r64, nc));
        ARIEL_TRY(dalloc(s, &A.d32, nc));
    }
    A.max_chunks = std::max(1ll, maxch);
    ARIEL_TRY(dalloc(s, &A.partial, 3 * A.max_chunks));
    // bricks of the ordered sweeps: every scene's brick grid, listed by level I+J+K, then scene
    // and position (the order the sweeps take them in)
    sweep_brick(s->prm, A.bx, A.by, A.bz);
    std::vector<int4> bricks;
    std::vector<int> bbase(k + 1, 0);
    for (int i = 0; i < k; ++i) {
        const int n = s->descs[i].dim;
        const int nbI = (n + A.bx - 1) / A.bx, nbJ = (n + A.by - 1) / A.by, nbK = (n + A.bz - 1) / A.bz;
        bbase[i + 1] = bbase[i] + nbI * nbJ * nbK;
        for (int I = 0; I < nbI; ++I)
            for (int J = 0; J < nbJ; ++J)
                for (int K = 0; K < nbK; ++K) bricks.push_back(make_int4(i, I, J, K));
    }
    std::stable_sort(bricks.begin(), bricks.end(),
                     [](const int4& a, const int4& b) { return a.y + a.z + a.w < b.y + b.z + b.w; });
    A.nbricks = (int)bricks.size();
    int4* dbr = nullptr;
    int* dbase = nullptr;
    ARIEL_TRY(dalloc(s, &dbr, bricks.size()));
    ARIEL_TRY(dalloc(s, &dbase, (size_t)k + 1));
    ARIEL_TRY(dalloc(s, &A.bflag, bricks.size()));
    A.bricks = dbr;
    A.brick_base = dbase;
    ARIEL_TRY(dalloc(s, &A.sc, k, true));
    ARIEL_TRY(dalloc(s, &A.totals, k, true));
    ARIEL_TRY(dalloc(s, &A.ctl, 1));
    ARIEL_TRY(dalloc(s, &A.bar, 1));
    ARIEL_TRY(dalloc(s, &S.solid_pos, s->spref[k], true));
    // solid meshes: every scene's tree and triangles back to back
    {
        long long tn = 0, tt = 0;
        for (int i = 0; i < k; ++i) {
            tn += (long long)s->meshes[i]->nodes.size();
            tt += (long long)s->meshes[i]->tris.size();
        }
        ARIEL_TRY(dalloc(s, &s->d_mesh_nodes, tn));
        ARIEL_TRY(dalloc(s, &s->d_mesh_tris, tt));
        long long on = 0, ot = 0;
        for (int i = 0; i < k; ++i) {
            const SceneMeshes& M = *s->meshes[i];
            s->sh[i].mesh_nodes = M.nodes.empty() ? nullptr : s->d_mesh_nodes + on;
            s->sh[i].mesh_tris = M.tris.empty() ? nullptr : s->d_mesh_tris + ot;
            if (!M.nodes.empty()) {
                ARIEL_CUDA(copy_sync(s->stream, s->d_mesh_nodes + on, M.nodes.data(), M.nodes.size() * sizeof(MeshNode),
                                     cudaMemcpyHostToDevice));
                ARIEL_CUDA(copy_sync(s->stream, s->d_mesh_tris + ot, M.tris.data(), M.tris.size() * sizeof(MeshTri),
                                     cudaMemcpyHostToDevice));
            }
            on += (long long)M.nodes.size();
            ot += (long long)M.tris.size();
        }
    }
    A.S = S;
    s->pcg_blocks = pcg_max_blocks(s->device, s->mode, s->prm.pcg_blocks_per_sm);
    if (s->prm.pcg_grid_blocks > 0) s->pcg_blocks = std::min(s->pcg_blocks, (int)s->prm.pcg_grid_blocks);
    cudaStream_t st = s->stream;
    // scene table and prefixes
    ARIEL_CUDA(cudaMemcpyAsync(s->d_scenes, s->sh.data(), sizeof(SceneDev) * k, cudaMemcpyHostToDevice, st));
    ARIEL_CUDA(cudaMemcpyAsync(s->d_ppref, s->ppref.data(), sizeof(long long) * (k + 1), cudaMemcpyHostToDevice, st));
    ARIEL_CUDA(cudaMemcpyAsync(s->d_cpref, s->cpref.data(), sizeof(long long) * (k + 1), cudaMemcpyHostToDevice, st));
    ARIEL_CUDA(cudaMemcpyAsync(s->d_fpref, s->fpref.data(), sizeof(long long) * (k + 1), cudaMemcpyHostToDevice, st));
    ARIEL_CUDA(cudaMemsetAsync(S.P, 0, sizeof(float) * nc, st));
    ARIEL_CUDA(cudaMemsetAsync(S.P64, 0, sizeof(double) * nc, st));
    ARIEL_CUDA(cudaMemsetAsync(S.dev_error, 0, sizeof(int), st));
    ARIEL_CUDA(cudaMemsetAsync(S.u, 0, sizeof(float) * nf, st));
    ARIEL_CUDA(cudaMemsetAsync(S.pu, 0, sizeof(float) * nf, st));
    ARIEL_CUDA(cudaMemsetAsync(S.flags, 0, nc, st));
    ARIEL_CUDA(cudaMemsetAsync(A.sc, 0, sizeof(PcgScene) * k, st));
    if (!bricks.empty())
        ARIEL_CUDA(copy_sync(st, dbr, bricks.data(), bricks.size() * sizeof(int4), cudaMemcpyHostToDevice));
    ARIEL_CUDA(copy_sync(st, dbase, bbase.data(), bbase.size() * sizeof(int), cudaMemcpyHostToDevice));
    ARIEL_CUDA(cudaMemsetAsync(A.totals, 0, sizeof(PcgTotals) * k, st));
    // per-scene persistent state
    uint32_t* stage_u32 = nullptr;
    for (int i = 0; i < k; ++i) {
        const long long pb = s->ppref[i], cnt = s->ppref[i + 1] - pb;
        const long long cb = s->cpref[i], ncell = s->cpref[i + 1] - cb;
        const long long sb = s->spref[i], scnt = s->spref[i + 1] - sb;
        if (from_src(i)) {
            // a scene carried over from another layout: device copies, solid offsets shifted
            const int j = (*src_idx)[i];
            const long long pb0 = src->ppref[j], cb0 = src->cpref[j], sb0 = src->spref[j];
            const DevState& T = src->S;
            if (cnt > 0) {
                ARIEL_CUDA(cudaMemcpyAsync(S.pos4 + pb, T.pos4 + pb0, cnt * sizeof(float4), cudaMemcpyDeviceToDevice, st));
                ARIEL_CUDA(cudaMemcpyAsync(S.vel4 + pb, T.vel4 + pb0, cnt * sizeof(float4), cudaMemcpyDeviceToDevice, st));
            }
            ARIEL_CUDA(cudaMemcpyAsync(S.P + cb, T.P + cb0, ncell * sizeof(float), cudaMemcpyDeviceToDevice, st));
            ARIEL_CUDA(cudaMemcpyAsync(S.P64 + cb, T.P64 + cb0, ncell * sizeof(double), cudaMemcpyDeviceToDevice, st));
            if (scnt > 0)
                ARIEL_CUDA(cudaMemcpyAsync(S.solid_pos + sb, T.solid_pos + sb0, scnt * sizeof(float4),
                                           cudaMemcpyDeviceToDevice, st));
            ARIEL_CUDA(launch_u32_offset(S.solid_start + cb, T.solid_start + cb0, ncell, 0u, st));
            if (sb != sb0) {
                // shift in place: offsets of this scene move from sb0 to sb
                ARIEL_CUDA(launch_u32_offset(S.solid_start + cb, S.solid_start + cb, ncell, (uint32_t)(sb - sb0), st));
            }
            ARIEL_CUDA(cudaMemcpyAsync(A.sc + i, src->PA.sc + j, sizeof(PcgScene), cudaMemcpyDeviceToDevice, st));
            ARIEL_CUDA(cudaMemcpyAsync(A.totals + i, src->PA.totals + j, sizeof(PcgTotals), cudaMemcpyDeviceToDevice, st));
            continue;
        }
        if (from_staged(i)) {
            // a new scene already uploaded: device copies only
            const DeviceParticles& g = (*staged)[i];
            if (cnt > 0) {
                ARIEL_CUDA(cudaMemcpyAsync(S.pos4 + pb, g.pos4, cnt * sizeof(float4), cudaMemcpyDeviceToDevice, st));
                ARIEL_CUDA(cudaMemcpyAsync(S.vel4 + pb, g.vel4, cnt * sizeof(float4), cudaMemcpyDeviceToDevice, st));
            }
            if (scnt > 0) {
                ARIEL_CUDA(cudaMemcpyAsync(S.solid_pos + sb, g.solid_pos, scnt * sizeof(float4),
                                           cudaMemcpyDeviceToDevice, st));
                ARIEL_CUDA(launch_u32_offset(S.solid_start + cb, g.solid_start, ncell, (uint32_t)sb, st));
            } else {
                ARIEL_CUDA(launch_u32_offset(S.solid_start + cb, nullptr, ncell, (uint32_t)sb, st));
            }
            continue;
        }
        if (cnt > 0) {
            ARIEL_CUDA(copy_sync(st, S.pos4 + pb, hp[i].pos4.data(), cnt * sizeof(float4), cudaMemcpyHostToDevice));
            ARIEL_CUDA(copy_sync(st, S.vel4 + pb, hp[i].vel4.data(), cnt * sizeof(float4), cudaMemcpyHostToDevice));
        }
        if (scnt > 0) {
            ARIEL_CUDA(copy_sync(st, S.solid_pos + sb, hp[i].solid_pos.data(), scnt * sizeof(float4), cudaMemcpyHostToDevice));
            if (!stage_u32) {
                // the scene-local offsets pass through the I/O staging area when it is large
                // enough, else through a temporary buffer
                ARIEL_CUDA(cudaMallocAsync(&stage_u32, sizeof(uint32_t) * (size_t)(s->nc + 1), st));
            }
            ARIEL_CUDA(copy_sync(st, stage_u32, hp[i].solid_start.data(), ncell * sizeof(uint32_t), cudaMemcpyHostToDevice));
            ARIEL_CUDA(launch_u32_offset(S.solid_start + cb, stage_u32, ncell, (uint32_t)sb, st));
        } else {
            ARIEL_CUDA(launch_u32_offset(S.solid_start + cb, nullptr, ncell, (uint32_t)sb, st));
        }
    }
    ARIEL_CUDA(launch_u32_offset(S.solid_start + nc, nullptr, 1, (uint32_t)s->spref[k], st));
    if (stage_u32) ARIEL_CUDA(cudaFreeAsync(stage_u32, st));
    s->PA.S = S;
    ARIEL_CUDA(cudaStreamSynchronize(st));
    return ARIEL_OK;
}

ariel_status check_device_error(ariel_sim* s) {
    int err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, s->S.dev_error, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return map_cuda_error(e);
    if (err & 1) return ARIEL_ERR_DEVICE_TIMEOUT;
    if (err & 2) {
        // non-finite uploaded state: report once
        cudaMemsetAsync(s->S.dev_error, 0, sizeof(int), s->stream);
        return ARIEL_ERR_NAN;
    }
    return ARIEL_OK;
}

ariel_status compute_max_density(ariel_sim* s) {
    k_max_density<<<s->k, 1024, 0, s->stream>>>(s->d_scenes, s->k);
    count_launch();
    ARIEL_CUDA(cudaGetLastError());
    std::vector<SceneDev> dev(s->k);
    ARIEL_CUDA(copy_sync(s->stream, dev.data(), s->d_scenes, sizeof(SceneDev) * s->k, cudaMemcpyDeviceToHost));
    for (int i = 0; i < s->k; ++i) s->sh[i].max_density = dev[i].max_density;
    return ARIEL_OK;
}

ariel_status refresh_scene_table(ariel_sim* s) {
    std::vector<SceneDev> dev(s->k);
    ARIEL_CUDA(copy_sync(s->stream, dev.data(), s->d_scenes, sizeof(SceneDev) * s->k, cudaMemcpyDeviceToHost));
    for (int i = 0; i < s->k; ++i) {
        s->sh[i].frame = dev[i].frame;
        s->sh[i].max_density = dev[i].max_density;
    }
    return ARIEL_OK;
}

ariel_status sort_and_classify_init(ariel_sim* s) {
    cudaError_t e = launch_sort(s->S, s->scan_tmp, s->stream);
    if (e == cudaSuccess) e = launch_fill_dens(s->S, 10.0f, s->stream);  // AddLiquidParticle: m_density = 10
    if (e == cudaSuccess) e = launch_classify(s->S, 1, s->stream);
    if (e != cudaSuccess) return map_cuda_error(e);
    return ARIEL_OK;
}

ariel_status new_sim(const AsimSceneDesc* descs, int k, const AsimParams& prm, cudaStream_t stream,
                     cudaMemPool_t pool, ariel_sim** out) {
    *out = nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    ariel_sim* s = new (std::nothrow) ariel_sim();
    if (!s) return ARIEL_ERR_OOM;
    s->device = dev;
    s->k = k;
    s->descs.assign(descs, descs + k);
    s->prm = prm;
    s->frames.assign(k, 0);
    for (int i = 0; i < k; ++i) s->sh.push_back(make_scene(descs[i], prm));
    s->meshes.resize(k);
    for (int i = 0; i < k; ++i) {
        ariel_status ms = scene_meshes(descs[i], s->meshes[i]);
        if (ms != ARIEL_OK) {
            delete s;
            return ms;
        }
    }
    s->pool = pool;
    if (stream) {
        s->stream = stream;
        s->own_stream = false;
    } else if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return ARIEL_ERR_CUDA;
    }
    for (auto& set : s->ev)
        for (auto& e : set) cudaEventCreate(&e);
    cudaEventCreate(&s->tb);
    cudaEventCreate(&s->te);
    *out = s;
    return ARIEL_OK;
}

void delete_sim(ariel_sim* s) {
    if (!s) return;
    cudaStreamSynchronize(s->stream);
    free_all(s);
    cudaStreamSynchronize(s->stream);
    for (auto& set : s->ev)
        for (auto& e : set) cudaEventDestroy(e);
    cudaEventDestroy(s->tb);
    cudaEventDestroy(s->te);
    if (s->own_stream) cudaStreamDestroy(s->stream);
    delete s;
}

}  // namespace hostimpl
}  // namespace ariel

using namespace ariel::hostimpl;

namespace {

const char* const kStageNames[ARIEL_STAGE_COUNT] = {
    "begin", "sort", "density", "forces", "p2g", "classify", "boundary_div", "solve", "gradient", "extrapolate",
    "g2p_advect", "resample"};

ariel_status enqueue_stage(ariel_sim* s, int g, cudaEvent_t* evs = nullptr) {
    NvtxRange range(g >= 0 && g < ARIEL_STAGE_COUNT ? kStageNames[g] : "stage");
    const DevState& S = s->S;
    cudaStream_t st = s->stream;
    cudaError_t e = cudaSuccess;
    switch (g) {
        case ARIEL_STAGE_BEGIN: e = launch_begin(S, st); break;
        case ARIEL_STAGE_SORT: e = launch_sort(S, s->scan_tmp, st); break;
        case ARIEL_STAGE_DENSITY: e = launch_density(S, st); break;
        case ARIEL_STAGE_FORCES: e = launch_forces(S, st); break;
        case ARIEL_STAGE_P2G: e = launch_p2g(S, s->prm.p2g_faces, st); break;
        case ARIEL_STAGE_CLASSIFY: e = launch_classify(S, 0, st); break;
        case ARIEL_STAGE_BOUNDARY_DIV: e = launch_boundary_div(S, st); break;
        case ARIEL_STAGE_SOLVE:
            e = launch_pcg_prepare(s->PA, s->flpred, s->flscan, s->scan_tmp, st);
            if (e == cudaSuccess && evs) e = cudaEventRecordWithFlags(evs[kEvSolveKernel], st, cudaEventRecordExternal);
            if (e == cudaSuccess) e = launch_pcg_solve(s->PA, s->pcg_blocks, st);
            break;
        case ARIEL_STAGE_GRADIENT: e = launch_gradient(S, st); break;
        case ARIEL_STAGE_EXTRAPOLATE: e = launch_extrapolate(S, st); break;
        case ARIEL_STAGE_G2P_ADVECT: e = launch_g2p_advect(S, st); break;
        case ARIEL_STAGE_RESAMPLE: e = launch_resample(S, s->scan_tmp, st); break;
        default: return ARIEL_ERR_INVALID_ARG;
    }
    if (e != cudaSuccess) return map_cuda_error(e, "stage launch");
    return ARIEL_OK;
}

// One step; with `evs` the stage boundaries (and the solve kernel's start) are recorded.
ariel_status enqueue_step(ariel_sim* s, cudaEvent_t* evs) {
    for (int g = 0; g < ARIEL_STAGE_COUNT; ++g) {
        if (evs) ARIEL_CUDA(cudaEventRecordWithFlags(evs[g], s->stream, cudaEventRecordExternal));
        ARIEL_TRY(enqueue_stage(s, g, evs));
    }
    if (evs) ARIEL_CUDA(cudaEventRecordWithFlags(evs[ARIEL_STAGE_COUNT], s->stream, cudaEventRecordExternal));
    return ARIEL_OK;
}

// Reads a finished step's events into the accumulators.
ariel_status collect_step_events(ariel_sim* s, int slot) {
    cudaEvent_t* evs = s->ev[slot];
    ARIEL_CUDA(cudaEventSynchronize(evs[ARIEL_STAGE_COUNT]));
    for (int g = 0; g < ARIEL_STAGE_COUNT; ++g) {
        float ms = 0;
        ARIEL_CUDA(cudaEventElapsedTime(&ms, evs[g], evs[g + 1]));
        s->stage_ms[g] = ms;
        s->acc_stage[g] += ms;
    }
    float ks = 0, tot = 0;
    ARIEL_CUDA(cudaEventElapsedTime(&ks, evs[kEvSolveKernel], evs[ARIEL_STAGE_SOLVE + 1]));
    ARIEL_CUDA(cudaEventElapsedTime(&tot, evs[0], evs[ARIEL_STAGE_COUNT]));
    s->acc_solve_kernel += ks;
    s->step_ms = tot;
    s->step_hist.push_back(tot);
    s->ev_pending[slot] = false;
    return ARIEL_OK;
}

// which: 0 plain step, 1/2 step recording event set 0/1.
void try_build_graph(ariel_sim* s, int which) {
    const auto t_start = std::chrono::steady_clock::now();
    struct Timer {
        ariel_sim* s;
        std::chrono::steady_clock::time_point t;
        ~Timer() { s->graph_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count(); }
    } timer{s, t_start};
    s->graph_tried[which] = true;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    long long before = launch_count();
    ariel_status st = enqueue_step(s, which == 0 ? nullptr : s->ev[which - 1]);
    long long kernels = launch_count() - before;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (st != ARIEL_OK || e != cudaSuccess || !g) {
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        return;
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    s->graph[which] = ex;
    s->graph_kernels[which] = kernels;
    count_launch(-(int)kernels);  // capture does not launch; replays are counted instead
}

ariel_status download_particles(ariel_sim* s, std::vector<HostParticles>& hp) {
    hp.assign(s->k, HostParticles{});
    for (int i = 0; i < s->k; ++i) {
        long long b = s->ppref[i], n = s->ppref[i + 1] - b;
        hp[i].pos4.resize(n);
        hp[i].vel4.resize(n);
        if (n == 0) continue;
        ARIEL_CUDA(copy_sync(s->stream, hp[i].pos4.data(), s->S.pos4 + b, n * sizeof(float4), cudaMemcpyDeviceToHost));
        ARIEL_CUDA(copy_sync(s->stream, hp[i].vel4.data(), s->S.vel4 + b, n * sizeof(float4), cudaMemcpyDeviceToHost));
    }
    return ARIEL_OK;
}

ariel_status check_params(const AsimParams* params) {
    if (params->precision < 0 || params->precision > 2 || params->precond < 0 || params->precond > 1 ||
        params->stop_rule < 0 || params->stop_rule > 1)
        return ARIEL_ERR_INVALID_ARG;
    int bx, by, bz;
    sweep_brick(*params, bx, by, bz);
    if (!brick_shape_ok(bx, by, bz)) return ARIEL_ERR_INVALID_ARG;
    if (params->p2g_faces != 0 && params->p2g_faces != 1 && params->p2g_faces != 2 && params->p2g_faces != 4)
        return ARIEL_ERR_INVALID_ARG;
    int rmin, rmax;
    reseed_bounds(*params, rmin, rmax);
    if (params->reseed_every < 0 || params->reseed_min < 0 || params->reseed_max < 0 || rmin > rmax ||
        rmax > 65535)
        return ARIEL_ERR_INVALID_ARG;
    return ARIEL_OK;
}

ariel_status check_device() {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return ARIEL_ERR_NO_DEVICE;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return ARIEL_ERR_NO_DEVICE;  // built for sm_100a only
    return ARIEL_OK;
}

ariel_status create_common(const AsimSceneDesc* descs, int32_t k, const AsimParams* params, ariel_sim** out) {
    if (!descs || !params || !out || k < 1 || k > kMaxScenes) return ARIEL_ERR_INVALID_ARG;
    *out = nullptr;
    for (int i = 0; i < k; ++i) ARIEL_TRY(validate(descs[i]));
    ARIEL_TRY(check_params(params));
    ARIEL_TRY(check_device());
    ariel_sim* s = nullptr;
    ARIEL_TRY(new_sim(descs, k, *params, nullptr, nullptr, &s));
    std::vector<HostParticles> empty(k);
    ariel_status st = build_state(s, empty);
    if (st != ARIEL_OK) {
        delete_sim(s);
        return st;
    }
    *out = s;
    return ARIEL_OK;
}

}  // namespace

namespace ariel {
namespace hostimpl {

ariel_status step_async(ariel_sim* s) {
    if (s->prm.timing) {
        const int slot = s->ev_slot;
        s->ev_slot ^= 1;
        if (s->ev_pending[slot]) ARIEL_TRY(collect_step_events(s, slot));
        if (s->prm.use_graph && !s->graph_tried[1 + slot]) try_build_graph(s, 1 + slot);
        if (s->graph[1 + slot]) {
            cudaError_t e = cudaGraphLaunch(s->graph[1 + slot], s->stream);
            if (e != cudaSuccess) return map_cuda_error(e);
            count_launch((int)s->graph_kernels[1 + slot]);
        } else {
            ARIEL_TRY(enqueue_step(s, s->ev[slot]));
        }
        s->ev_pending[slot] = true;
        // read the previous step while this one runs
        if (s->ev_pending[slot ^ 1]) ARIEL_TRY(collect_step_events(s, slot ^ 1));
    } else {
        if (s->prm.use_graph && !s->graph_tried[0]) try_build_graph(s, 0);
        if (s->graph[0]) {
            cudaError_t e = cudaGraphLaunch(s->graph[0], s->stream);
            if (e != cudaSuccess) return map_cuda_error(e);
            count_launch((int)s->graph_kernels[0]);
        } else {
            ARIEL_TRY(enqueue_step(s, nullptr));
        }
    }
    for (auto& f : s->frames) f++;
    return ARIEL_OK;
}

ariel_status collect_pending(ariel_sim* s) {
    // the older step first, so that the step history stays in step order
    const int older = s->ev_slot, newer = s->ev_slot ^ 1;
    if (s->ev_pending[older]) ARIEL_TRY(collect_step_events(s, older));
    if (s->ev_pending[newer]) ARIEL_TRY(collect_step_events(s, newer));
    return ARIEL_OK;
}

}  // namespace hostimpl
}  // namespace ariel

// ==============================================================================================
// C ABI
// ==============================================================================================
extern "C" {

int32_t ariel_abi_version(void) { return ARIEL_ABI_VERSION; }

void ariel_params_default(AsimParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->picflip = 0.95f;  // flip.cpp:27
    p->subcell = 1;      // flip.cpp:26
    p->precond = ARIEL_PRECOND_REF;
    p->precision = ARIEL_PREC_REF32;
    p->stop_rule = ARIEL_STOP_REF_ABS;
    p->max_iters = 0;
    p->tol = 1e-5;
    p->inner_tol = 1e-6;  // deep enough that one fp32 correction solve usually meets the target, shallow enough for fp32 to reach
    p->max_outer = 8;
    p->resample_every = 1;  // flip.cpp:121
    p->mic_tau = 0.97;
    p->mic_sigma = 0.25;
    p->rng_seed = 0x5EED;
    p->use_graph = 1;
    p->timing = 0;
    p->barrier_timeout_ms = 2000.0;
    p->fail_on_not_converged = 0;
}

void ariel_scene_dambreak(AsimSceneDesc* d, int32_t n) {
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->dim = n;
    d->density = 0.5f;
    d->stepsize = 1.0f / 240.0f;
    d->n_forces = 1;
    d->forces[0][1] = -9.8f;
    d->n_liquid = 1;
    d->liquid[0].hi[0] = 0.4f;
    d->liquid[0].hi[1] = 0.6f;
    d->liquid[0].hi[2] = 1.0f;
    d->seed = 1;
    d->jitter = 1.0f;
}

const char* ariel_status_string(ariel_status st) {
    switch (st) {
        case ARIEL_OK: return "ok";
        case ARIEL_ERR_INVALID_ARG: return "invalid argument";
        case ARIEL_ERR_OOM: return "device memory exhausted";
        case ARIEL_ERR_NOT_CONVERGED: return "pressure solve did not converge";
        case ARIEL_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
        case ARIEL_ERR_CUDA: return "CUDA error";
        case ARIEL_ERR_STATE: return "call out of order";
        case ARIEL_ERR_NO_DEVICE: return "no sm_100 device";
        case ARIEL_ERR_NAN: return "non-finite input";
        case ARIEL_ERR_PENDING: return "request not finished";
    }
    return "unknown status";
}

ariel_status ariel_create(const AsimSceneDesc* desc, const AsimParams* params, ariel_sim** out) {
    return create_common(desc, 1, params, out);
}

ariel_status ariel_create_batch(const AsimSceneDesc* descs, int32_t k, const AsimParams* params, ariel_sim** out) {
    return create_common(descs, k, params, out);
}

ariel_status ariel_destroy(ariel_sim* s) {
    if (!s) return ARIEL_ERR_INVALID_ARG;
    delete_sim(s);
    return ARIEL_OK;
}

ariel_status ariel_scene_count(ariel_sim* s, int32_t* k) {
    if (!s || !k) return ARIEL_ERR_INVALID_ARG;
    *k = s->k;
    return ARIEL_OK;
}

ariel_status ariel_init(ariel_sim* s) {
    if (!s) return ARIEL_ERR_INVALID_ARG;
    NvtxRange range("ariel_init");
    // m_max_density from the 10^3 lattice, per scene (flip.cpp:47-70)
    ARIEL_TRY(compute_max_density(s));
    for (int i = 0; i < s->k; ++i) {
        s->sh[i].frame = 0;
        s->frames[i] = 0;
    }
    std::vector<HostParticles> hp(s->k);
    {
        // scenes are seeded independently: one host thread per scene, up to the core count
        std::atomic<int> next{0};
        auto work = [&] {
            for (int i = next++; i < s->k; i = next++) generate_particles(s->descs[i], hp[i]);
        };
        const int nt = std::max(1, std::min(s->k, (int)std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
    }
    ARIEL_TRY(build_state(s, hp));
    ARIEL_TRY(sort_and_classify_init(s));
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    s->inited = true;
    return ARIEL_OK;
}

ariel_status ariel_set_particles(ariel_sim* s, int32_t scene, int64_t n, const float* pos, const float* vel,
                                 const float* mass, const int32_t* type) {
    if (!s || scene < 0 || scene >= s->k || n < 0 || (n > 0 && (!pos || !vel || !mass || !type)))
        return ARIEL_ERR_INVALID_ARG;
    for (int64_t i = 0; i < 3 * n; ++i)
        if (!std::isfinite(pos[i]) || !std::isfinite(vel[i])) return ARIEL_ERR_NAN;
    cudaStreamSynchronize(s->stream);
    ARIEL_TRY(refresh_scene_table(s));
    std::vector<HostParticles> hp;
    ARIEL_TRY(download_particles(s, hp));
    hp[scene].pos4.resize(n);
    hp[scene].vel4.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        hp[scene].pos4[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], mass[i]);
        hp[scene].vel4[i] = pack_vel(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], type[i]);
    }
    // keep the pressure warm start of every scene
    std::vector<float> P(s->nc);
    std::vector<double> P64(s->nc);
    ARIEL_CUDA(copy_sync(s->stream, P.data(), s->S.P, sizeof(float) * s->nc, cudaMemcpyDeviceToHost));
    ARIEL_CUDA(copy_sync(s->stream, P64.data(), s->S.P64, sizeof(double) * s->nc, cudaMemcpyDeviceToHost));
    ARIEL_TRY(build_state(s, hp));
    ARIEL_CUDA(copy_sync(s->stream, s->S.P, P.data(), sizeof(float) * s->nc, cudaMemcpyHostToDevice));
    ARIEL_CUDA(copy_sync(s->stream, s->S.P64, P64.data(), sizeof(double) * s->nc, cudaMemcpyHostToDevice));
    if (!s->inited) {
        // a handle fed directly with particles still needs the density normaliser
        ARIEL_TRY(compute_max_density(s));
        s->inited = true;
    }
    ARIEL_TRY(sort_and_classify_init(s));
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    return ARIEL_OK;
}

ariel_status ariel_stage(ariel_sim* s, int32_t stage) {
    if (!s || stage < 0 || stage >= ARIEL_STAGE_COUNT) return ARIEL_ERR_INVALID_ARG;
    if (!s->inited) return ARIEL_ERR_STATE;
    if (stage == ARIEL_STAGE_BEGIN)
        for (auto& f : s->frames) f++;
    ARIEL_TRY(enqueue_stage(s, stage));
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    return check_device_error(s);
}

ariel_status ariel_step(ariel_sim* s, int32_t nsteps) {
    if (!s || nsteps < 0) return ARIEL_ERR_INVALID_ARG;
    if (!s->inited) return ARIEL_ERR_STATE;
    NvtxRange range("ariel_step");
    for (int it = 0; it < nsteps; ++it) {
        ARIEL_TRY(step_async(s));
        if (s->prm.fail_on_not_converged) {
            std::vector<PcgScene> sc(s->k);
            ARIEL_CUDA(cudaMemcpyAsync(sc.data(), s->PA.sc, sizeof(PcgScene) * s->k, cudaMemcpyDeviceToHost, s->stream));
            ARIEL_CUDA(cudaStreamSynchronize(s->stream));
            ARIEL_TRY(check_device_error(s));
            for (auto& v : sc)
                if (!v.converged) {
                    s->last_status = ARIEL_ERR_NOT_CONVERGED;
                    return ARIEL_ERR_NOT_CONVERGED;
                }
        }
    }
    // the last step's events (its successor has not been launched)
    if (s->prm.timing) ARIEL_TRY(collect_pending(s));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return map_cuda_error(e);
    return ARIEL_OK;
}

ariel_status ariel_synchronize(ariel_sim* s) {
    if (!s) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    return check_device_error(s);
}

ariel_status ariel_particle_count(ariel_sim* s, int32_t scene, int64_t* n) {
    if (!s || !n || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    *n = s->ppref[scene + 1] - s->ppref[scene];
    return ARIEL_OK;
}

ariel_status ariel_get_particles(ariel_sim* s, int32_t scene, float* pos, float* vel, float* density, float* mass,
                                 int32_t* type) {
    if (!s || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    const long long b = s->ppref[scene], n = s->ppref[scene + 1] - b;
    if (n == 0) return ARIEL_OK;
    std::vector<float4> p4(n), v4(n);
    ARIEL_CUDA(copy_sync(s->stream, p4.data(), s->S.pos4 + b, n * sizeof(float4), cudaMemcpyDeviceToHost));
    ARIEL_CUDA(copy_sync(s->stream, v4.data(), s->S.vel4 + b, n * sizeof(float4), cudaMemcpyDeviceToHost));
    for (long long i = 0; i < n; ++i) {
        if (pos) {
            pos[3 * i] = p4[i].x;
            pos[3 * i + 1] = p4[i].y;
            pos[3 * i + 2] = p4[i].z;
        }
        if (vel) {
            vel[3 * i] = v4[i].x;
            vel[3 * i + 1] = v4[i].y;
            vel[3 * i + 2] = v4[i].z;
        }
        if (mass) mass[i] = p4[i].w;
        if (type) type[i] = type_bits(v4[i]);
    }
    if (density) {
        cudaError_t e = launch_scatter_density(s->S, s->d_dens_id, s->stream);
        if (e != cudaSuccess) return map_cuda_error(e);
        ARIEL_CUDA(cudaMemcpyAsync(density, s->d_dens_id + b, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
        ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    }
    return ARIEL_OK;
}

ariel_status ariel_get_cells(ariel_sim* s, int32_t scene, int32_t* particle_cell, int32_t* cell_count) {
    if (!s || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    const long long pb = s->ppref[scene], pn = s->ppref[scene + 1] - pb;
    const long long cb = s->cpref[scene], cn = s->cpref[scene + 1] - cb;
    if (particle_cell && pn > 0) {
        std::vector<uint32_t> key(pn);
        ARIEL_CUDA(copy_sync(s->stream, key.data(), s->S.key + pb, pn * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        for (long long i = 0; i < pn; ++i) particle_cell[i] = (int32_t)((long long)key[i] - cb);
    }
    if (cell_count) ARIEL_CUDA(copy_sync(s->stream, cell_count, s->S.count + cb, cn * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return ARIEL_OK;
}

static ariel_status grid_span(ariel_sim* s, int32_t scene, int32_t which, void** dptr, size_t* elems, size_t* esize,
                              bool* is_flags) {
    const long long n = s->descs[scene].dim;
    const long long per = n * n * (n + 1);
    const long long fb = s->fpref[scene], cb = s->cpref[scene];
    *is_flags = false;
    switch (which) {
        case ARIEL_GRID_UX: *dptr = s->S.u + fb; *elems = per; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_UY: *dptr = s->S.u + fb + per; *elems = per; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_UZ: *dptr = s->S.u + fb + 2 * per; *elems = per; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_PREV_UX: *dptr = s->S.pu + fb; *elems = per; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_PREV_UY: *dptr = s->S.pu + fb + per; *elems = per; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_PREV_UZ: *dptr = s->S.pu + fb + 2 * per; *elems = per; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_D: *dptr = s->S.D + cb; *elems = n * n * n; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_P: *dptr = s->S.P + cb; *elems = n * n * n; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_L: *dptr = s->S.L + cb; *elems = n * n * n; *esize = 4; return ARIEL_OK;
        case ARIEL_GRID_A: *dptr = s->S.flags + cb; *elems = n * n * n; *esize = 4; *is_flags = true; return ARIEL_OK;
        case ARIEL_GRID_P64: *dptr = s->S.P64 + cb; *elems = n * n * n; *esize = 8; return ARIEL_OK;
    }
    return ARIEL_ERR_INVALID_ARG;
}

ariel_status ariel_get_grid(ariel_sim* s, int32_t scene, int32_t which, void* buf, int64_t nbytes) {
    if (!s || !buf || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    void* d;
    size_t elems, esize;
    bool flags;
    ARIEL_TRY(grid_span(s, scene, which, &d, &elems, &esize, &flags));
    if ((size_t)nbytes != elems * esize) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    if (flags) {
        std::vector<uint8_t> f(elems);
        ARIEL_CUDA(copy_sync(s->stream, f.data(), d, elems, cudaMemcpyDeviceToHost));
        int32_t* o = (int32_t*)buf;
        for (size_t i = 0; i < elems; ++i) o[i] = f[i];
    } else {
        ARIEL_CUDA(copy_sync(s->stream, buf, d, elems * esize, cudaMemcpyDeviceToHost));
    }
    return ARIEL_OK;
}

ariel_status ariel_set_grid(ariel_sim* s, int32_t scene, int32_t which, const void* buf, int64_t nbytes) {
    if (!s || !buf || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    void* d;
    size_t elems, esize;
    bool flags;
    ARIEL_TRY(grid_span(s, scene, which, &d, &elems, &esize, &flags));
    if ((size_t)nbytes != elems * esize) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    if (flags) {
        const int32_t* in = (const int32_t*)buf;
        std::vector<uint8_t> f(elems);
        for (size_t i = 0; i < elems; ++i) {
            if (in[i] < 0 || in[i] > 2) return ARIEL_ERR_INVALID_ARG;
            f[i] = (uint8_t)in[i];
        }
        ARIEL_CUDA(copy_sync(s->stream, d, f.data(), elems, cudaMemcpyHostToDevice));
    } else {
        ARIEL_CUDA(copy_sync(s->stream, d, buf, elems * esize, cudaMemcpyHostToDevice));
    }
    return ARIEL_OK;
}

ariel_status ariel_get_dimensions(ariel_sim* s, int32_t scene, int32_t* n) {
    if (!s || !n || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    *n = s->descs[scene].dim;
    return ARIEL_OK;
}

ariel_status ariel_stats(ariel_sim* s, int32_t scene, AsimStats* out) {
    if (!s || !out || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    PcgScene sc{};
    ARIEL_CUDA(copy_sync(s->stream, &sc, s->PA.sc + scene, sizeof(PcgScene), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    out->frame = s->frames[scene];
    out->n_particles = s->ppref[scene + 1] - s->ppref[scene];
    out->n_fluid_cells = sc.nf;
    out->pcg_iterations = sc.iters;
    out->pcg_outer = s->mode == kMixed ? sc.outer : 1;
    out->pcg_rr = sc.rr;
    double rr = s->mode == kMixed ? sc.rr_out : sc.rr;
    out->pcg_rel_residual = sc.bb > 0 ? std::sqrt(rr / sc.bb) : 0.0;
    out->pcg_converged = sc.converged;
    out->precond_exact_path = sc.ordered;
    for (int g = 0; g < ARIEL_STAGE_COUNT; ++g) out->stage_ms[g] = s->stage_ms[g];
    out->step_ms = s->step_ms;
    out->last_status = s->last_status;
    return ARIEL_OK;
}

ariel_status ariel_get_max_density(ariel_sim* s, int32_t scene, float* md) {
    if (!s || !md || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    *md = s->sh[scene].max_density;
    return ARIEL_OK;
}

ariel_status ariel_timer_begin(ariel_sim* s) {
    if (!s) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaEventRecord(s->tb, s->stream));
    return ARIEL_OK;
}

ariel_status ariel_timer_end(ariel_sim* s, double* ms) {
    if (!s || !ms) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaEventRecord(s->te, s->stream));
    ARIEL_CUDA(cudaEventSynchronize(s->te));
    float f = 0;
    ARIEL_CUDA(cudaEventElapsedTime(&f, s->tb, s->te));
    *ms = f;
    return ARIEL_OK;
}

ariel_status ariel_timing_reset(ariel_sim* s) {
    if (!s) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    for (int g = 0; g < ARIEL_STAGE_COUNT; ++g) s->acc_stage[g] = 0;
    s->acc_solve_kernel = 0;
    s->step_hist.clear();
    ARIEL_CUDA(cudaMemsetAsync(s->PA.totals, 0, sizeof(PcgTotals) * s->k, s->stream));
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    return ARIEL_OK;
}

ariel_status ariel_solver_totals(ariel_sim* s, int32_t scene, AsimSolverTotals* out) {
    if (!s || !out || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    PcgTotals t{};
    ARIEL_CUDA(copy_sync(s->stream, &t, s->PA.totals + scene, sizeof(PcgTotals), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    out->solves = t.solves;
    out->iterations = t.iterations;
    out->outer = t.outer;
    out->cell_iterations = t.cell_iterations;
    out->cell_outer = t.cell_outer;
    out->not_converged = t.not_converged;
    return ARIEL_OK;
}

ariel_status ariel_timing_get(ariel_sim* s, double* ms, double* solve_kernel_ms, double* step_ms, int32_t max_steps,
                              int32_t* nsteps) {
    if (!s) return ARIEL_ERR_INVALID_ARG;
    if (ms)
        for (int g = 0; g < ARIEL_STAGE_COUNT; ++g) ms[g] = s->acc_stage[g];
    if (solve_kernel_ms) *solve_kernel_ms = s->acc_solve_kernel;
    int n = (int)s->step_hist.size();
    if (step_ms && max_steps > 0) {
        int m = std::min(n, (int)max_steps);
        for (int i = 0; i < m; ++i) step_ms[i] = s->step_hist[n - m + i];
    }
    if (nsteps) *nsteps = n;
    return ARIEL_OK;
}

ariel_status ariel_upload_state(ariel_sim* s, int32_t scene, const float* pos, const float* vel) {
    if (!s || !pos || !vel || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    const long long b = s->ppref[scene], n = s->ppref[scene + 1] - b;
    if (n == 0) return ARIEL_OK;
    float* sp = s->d_stage;
    float* sv = s->d_stage + 3 * n;
    ARIEL_CUDA(cudaMemcpyAsync(sp, pos, 12 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    ARIEL_CUDA(cudaMemcpyAsync(sv, vel, 12 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    ARIEL_CUDA(launch_unpack_state(s->S.pos4 + b, s->S.vel4 + b, sp, sv, n, s->S.dev_error, s->stream));
    return ARIEL_OK;
}

ariel_status ariel_download_state(ariel_sim* s, int32_t scene, float* pos, float* vel) {
    if (!s || !pos || !vel || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    const long long b = s->ppref[scene], n = s->ppref[scene + 1] - b;
    if (n > 0) {
        float* sp = s->d_stage;
        float* sv = s->d_stage + 3 * n;
        ARIEL_CUDA(launch_pack_state(s->S.pos4 + b, s->S.vel4 + b, sp, sv, n, s->stream));
        ARIEL_CUDA(cudaMemcpyAsync(pos, sp, 12 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
        ARIEL_CUDA(cudaMemcpyAsync(vel, sv, 12 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
    }
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    return check_device_error(s);
}

ariel_status ariel_selftest_barrier_timeout(double timeout_ms) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return ARIEL_ERR_NO_DEVICE;
    }
    Barrier* bar = nullptr;
    int* err = nullptr;
    ARIEL_CUDA(cudaMalloc(&bar, sizeof(Barrier)));
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
        cudaFree(bar);
        return ARIEL_ERR_OOM;
    }
    cudaMemset(err, 0, sizeof(int));
    cudaError_t e = launch_barrier_selftest(bar, err, (unsigned long long)(timeout_ms * 1.0e6), 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    int h = 0;
    if (e == cudaSuccess) e = copy_sync(0, &h, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(bar);
    cudaFree(err);
    if (e != cudaSuccess) return map_cuda_error(e);
    return h ? ARIEL_ERR_DEVICE_TIMEOUT : ARIEL_OK;
}

// ---- checkpoints -------------------------------------------------------------------------
// File: "ARIELCK1", int32 k, then per scene: AsimSceneDesc, int64 frame, float max_density,
// int64 particles, pos4[particles], vel4[particles] (float4), P[n^3] (float), P64[n^3] (double).
// That is every piece of state a step reads from the previous one (the particles, the pressure
// warm start, the frame counter that keys the resampling RNG, and the density normaliser), so a
// handle loaded from a checkpoint continues bit-identically.
static const char kCkMagic[8] = {'A', 'R', 'I', 'E', 'L', 'C', 'K', '1'};

ariel_status ariel_checkpoint_save(ariel_sim* s, const char* path) {
    if (!s || !path) return ARIEL_ERR_INVALID_ARG;
    if (!s->inited) return ARIEL_ERR_STATE;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    ARIEL_TRY(refresh_scene_table(s));
    FILE* f = std::fopen(path, "wb");
    if (!f) return ARIEL_ERR_INVALID_ARG;
    bool ok = std::fwrite(kCkMagic, 1, 8, f) == 8;
    const int32_t k = s->k;
    ok = ok && std::fwrite(&k, sizeof(k), 1, f) == 1;
    for (int i = 0; ok && i < k; ++i) {
        const long long pb = s->ppref[i], np = s->ppref[i + 1] - pb;
        const long long cb = s->cpref[i], nc = s->cpref[i + 1] - cb;
        const int64_t frame = s->sh[i].frame;
        const float md = s->sh[i].max_density;
        std::vector<float4> p4(np), v4(np);
        std::vector<float> P(nc);
        std::vector<double> P64(nc);
        if (np > 0) {
            ARIEL_CUDA(copy_sync(s->stream, p4.data(), s->S.pos4 + pb, np * sizeof(float4), cudaMemcpyDeviceToHost));
            ARIEL_CUDA(copy_sync(s->stream, v4.data(), s->S.vel4 + pb, np * sizeof(float4), cudaMemcpyDeviceToHost));
        }
        ARIEL_CUDA(copy_sync(s->stream, P.data(), s->S.P + cb, nc * sizeof(float), cudaMemcpyDeviceToHost));
        ARIEL_CUDA(copy_sync(s->stream, P64.data(), s->S.P64 + cb, nc * sizeof(double), cudaMemcpyDeviceToHost));
        const int64_t n64 = np;
        ok = std::fwrite(&s->descs[i], sizeof(AsimSceneDesc), 1, f) == 1 && std::fwrite(&frame, 8, 1, f) == 1 &&
             std::fwrite(&md, 4, 1, f) == 1 && std::fwrite(&n64, 8, 1, f) == 1 &&
             std::fwrite(p4.data(), sizeof(float4), np, f) == (size_t)np &&
             std::fwrite(v4.data(), sizeof(float4), np, f) == (size_t)np &&
             std::fwrite(P.data(), sizeof(float), nc, f) == (size_t)nc &&
             std::fwrite(P64.data(), sizeof(double), nc, f) == (size_t)nc;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? ARIEL_OK : ARIEL_ERR_INVALID_ARG;
}

ariel_status ariel_checkpoint_load(ariel_sim* s, const char* path) {
    if (!s || !path) return ARIEL_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return ARIEL_ERR_INVALID_ARG;
    char magic[8];
    int32_t k = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kCkMagic, 8) == 0 &&
              std::fread(&k, sizeof(k), 1, f) == 1 && k == s->k;
    std::vector<HostParticles> hp(ok ? k : 0);
    std::vector<std::vector<float>> P(hp.size());
    std::vector<std::vector<double>> P64(hp.size());
    std::vector<int64_t> frames(hp.size());
    std::vector<float> md(hp.size());
    for (int i = 0; ok && i < k; ++i) {
        AsimSceneDesc d;
        int64_t np = 0;
        ok = std::fread(&d, sizeof(d), 1, f) == 1 && std::fread(&frames[i], 8, 1, f) == 1 &&
             std::fread(&md[i], 4, 1, f) == 1 && std::fread(&np, 8, 1, f) == 1 && np >= 0 && np < (1ll << 31);
        // the checkpoint must describe the same scenes as the handle
        ok = ok && std::memcmp(&d, &s->descs[i], sizeof(d)) == 0;
        if (!ok) break;
        const long long nc = (long long)d.dim * d.dim * d.dim;
        hp[i].pos4.resize(np);
        hp[i].vel4.resize(np);
        P[i].resize(nc);
        P64[i].resize(nc);
        ok = std::fread(hp[i].pos4.data(), sizeof(float4), np, f) == (size_t)np &&
             std::fread(hp[i].vel4.data(), sizeof(float4), np, f) == (size_t)np &&
             std::fread(P[i].data(), sizeof(float), nc, f) == (size_t)nc &&
             std::fread(P64[i].data(), sizeof(double), nc, f) == (size_t)nc;
    }
    std::fclose(f);
    if (!ok) return ARIEL_ERR_INVALID_ARG;
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    for (int i = 0; i < k; ++i) {
        s->sh[i].frame = frames[i];
        s->sh[i].max_density = md[i];
        s->frames[i] = frames[i];
    }
    ARIEL_TRY(build_state(s, hp));
    for (int i = 0; i < k; ++i) {
        const long long cb = s->cpref[i], nc = s->cpref[i + 1] - cb;
        ARIEL_CUDA(copy_sync(s->stream, s->S.P + cb, P[i].data(), nc * sizeof(float), cudaMemcpyHostToDevice));
        ARIEL_CUDA(copy_sync(s->stream, s->S.P64 + cb, P64[i].data(), nc * sizeof(double), cudaMemcpyHostToDevice));
    }
    ARIEL_TRY(sort_and_classify_init(s));
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    s->inited = true;
    return ARIEL_OK;
}

// ---- particle export (Scene::ExportParticles' Partio branch, src/scene/scene.cpp:35-80) ----
// FLUID particles in id order with attributes position (grid units: unit position x maxd), v
// and id (their index in the export), to `path` with the four-digit frame inserted before the
// extension (".gz" counted as part of it, scene.cpp:52-58).  Written in Houdini's classic ASCII
// geometry form (the ".geo" one of Partio's formats), gzip-compressed for ".geo.gz"; other
// extensions are refused.
ariel_status ariel_export_particles(ariel_sim* s, int32_t scene, const char* path, int32_t frame) {
    if (!s || !path || scene < 0 || scene >= s->k || frame < 0) return ARIEL_ERR_INVALID_ARG;
    std::string name(path);
    bool gz = false;
    if (name.size() > 3 && name.compare(name.size() - 3, 3, ".gz") == 0) {
        gz = true;
        name = name.substr(0, name.size() - 3);
    }
    const size_t slash = name.find_last_of('/');
    const size_t dot = name.find_last_of('.');
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return ARIEL_ERR_INVALID_ARG;
    std::string ext = name.substr(dot);
    std::string stem = name.substr(0, dot);
    if (ext != ".geo") return ARIEL_ERR_INVALID_ARG;
    char fr[16];
    std::snprintf(fr, sizeof(fr), ".%04d", frame);
    const std::string out = stem + fr + ext + (gz ? ".gz" : "");
    const long long b = s->ppref[scene], n = s->ppref[scene + 1] - b;
    std::vector<float4> p4(n), v4(n);
    ARIEL_CUDA(cudaStreamSynchronize(s->stream));
    if (n > 0) {
        ARIEL_CUDA(copy_sync(s->stream, p4.data(), s->S.pos4 + b, n * sizeof(float4), cudaMemcpyDeviceToHost));
        ARIEL_CUDA(copy_sync(s->stream, v4.data(), s->S.vel4 + b, n * sizeof(float4), cudaMemcpyDeviceToHost));
    }
    const float maxd = s->sh[scene].maxd;
    std::vector<long long> fluid;
    for (long long i = 0; i < n; ++i)
        if (type_bits(v4[i]) == ARIEL_FLUID) fluid.push_back(i);
    std::string text;
    char line[256];
    std::snprintf(line, sizeof(line), "PGEOMETRY V5\nNPoints %lld NPrims 1\nNPointGroups 0 NPrimGroups 0\n",
                  (long long)fluid.size());
    text += line;
    text += "NPointAttrib 2 NVertexAttrib 0 NPrimAttrib 0 NAttrib 0\nPointAttrib\n";
    text += "v 3 vector 0 0 0\nid 1 int 0\n";
    for (size_t e = 0; e < fluid.size(); ++e) {
        const float4& p = p4[fluid[e]];
        const float4& v = v4[fluid[e]];
        std::snprintf(line, sizeof(line), "%.9g %.9g %.9g 1 (%.9g %.9g %.9g %zu)\n", p.x * maxd, p.y * maxd,
                      p.z * maxd, v.x, v.y, v.z, e);
        text += line;
    }
    std::snprintf(line, sizeof(line), "Part %lld", (long long)fluid.size());
    text += line;
    for (size_t e = 0; e < fluid.size(); ++e) {
        std::snprintf(line, sizeof(line), " %zu", e);
        text += line;
    }
    text += "\nbeginExtra\nendExtra\n";
    if (gz) {
        gzFile f = gzopen(out.c_str(), "wb");
        if (!f) return ARIEL_ERR_INVALID_ARG;
        const int wrote = text.empty() ? 0 : gzwrite(f, text.data(), (unsigned)text.size());
        const int closed = gzclose(f);
        return (wrote == (int)text.size() && closed == Z_OK) ? ARIEL_OK : ARIEL_ERR_INVALID_ARG;
    }
    FILE* f = std::fopen(out.c_str(), "w");
    if (!f) return ARIEL_ERR_INVALID_ARG;
    const size_t wrote = std::fwrite(text.data(), 1, text.size(), f);
    return (std::fclose(f) == 0 && wrote == text.size()) ? ARIEL_OK : ARIEL_ERR_INVALID_ARG;
}

int64_t ariel_kernel_launches(void) { return launch_count(); }

const char* ariel_last_error(void) { return g_last_error; }

}  // extern "C"
