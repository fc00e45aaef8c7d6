// particles.cu -- particle-side stages of FlipSim::Step on sm_100a:
//   sort-by-cell (ParticleGrid::Sort), ComputeDensity, ApplyExternalForces,
//   SplatParticlesToMACGrid (deterministic per-face gather), SolvePicFlip + AdvectParticles,
//   ResampleParticles, and the analytic-sphere solid constraints.
//
// Determinism: every sum runs in the reference's order -- neighbour cells sx -> sy -> sz
// ascending, particles inside a cell in ascending particle id (the order ParticleGrid::Sort
// appends them, particlegrid.cpp:150-171).  The cell sort therefore finishes each cell's
// segment with an insertion sort by id after the arrival-order scatter.
#include "mesh.cuh"
#include "state.cuh"

namespace ariel {

namespace {

#define SCENE_PREFIX(pref_src)                       \
    __shared__ long long pref_s[kMaxScenes + 1];     \
    load_prefix<kMaxScenes>(pref_s, (pref_src), S.k)

// ------------------------------------------------------------------------------------------
// Solids: analytic spheres, then static meshes (mesh.cuh), replacing
// Scene::IntersectSolidGeoms scene.cpp:425-434, CheckPointInsideSolidGeom scene.cpp:382-402 and
// LevelSet::ProjectPointsToSurface levelset.cpp:175-193.  World (grid) units.
// ------------------------------------------------------------------------------------------
struct Hit {
    bool hit;
    float3 point, normal;
};

__device__ __forceinline__ bool has_solids(const SceneDev& D) { return D.n_spheres > 0 || D.n_meshes > 0; }

__device__ bool inside_solid(const SceneDev& D, float3 p) {
    for (int i = 0; i < D.n_spheres; ++i) {
        float4 s = D.sphere[i];
        float3 d = f3sub(p, make_float3(s.x, s.y, s.z));
        if (gdot3(d, d) < s.w * s.w) return true;
    }
    return D.n_meshes > 0 && mesh_inside_bits(D.mesh_nodes, D.mesh_tris, p) != 0u;
}

__device__ Hit intersect_solids(const SceneDev& D, float3 o, float3 dir) {
    Hit best{false, make_float3(0, 0, 0), make_float3(0, 0, 0)};
    float bestd = 0.0f;
    for (int i = 0; i < D.n_spheres; ++i) {
        float4 s = D.sphere[i];
        float3 c = make_float3(s.x, s.y, s.z);
        float3 oc = f3sub(o, c);
        float b = gdot3(dir, oc);
        float cc = gdot3(oc, oc) - s.w * s.w;
        float disc = b * b - cc;
        if (!(disc >= 0.0f)) continue;
        float sq = sqrtf(disc);
        float t = -b - sq;
        if (!(t > 0.0f)) t = -b + sq;
        if (!(t > 0.0f)) continue;
        float3 pt = f3add(o, f3mul(dir, t));
        float3 nrm = gnormalize3(f3sub(pt, c));
        float d = glength3(f3sub(pt, o));
        if (!best.hit || !(bestd <= d)) {
            best.hit = true;
            best.point = pt;
            best.normal = nrm;
            bestd = d;
        }
    }
    if (D.n_meshes > 0) {
        // solid meshes after the spheres, as the scene lists its solids (scene.cpp:425-434)
        float3 pt;
        float d;
        const int t = mesh_nearest(D.mesh_nodes, D.mesh_tris, o, dir, pt, d);
        if (t >= 0 && (!best.hit || !(bestd <= d))) {
            const MeshTri& T = D.mesh_tris[t];
            const float3 v0 = m3(T.v0);
            best.hit = true;
            best.point = pt;
            best.normal = mnormalize(mcross(msub(m3(T.v1), v0), msub(m3(T.v2), v0)));
            bestd = d;
        }
    }
    return best;
}

__device__ float3 closest_solid_surface(const SceneDev& D, float3 p) {
    for (int i = 0; i < D.n_spheres; ++i) {
        float4 s = D.sphere[i];
        float3 c = make_float3(s.x, s.y, s.z);
        float3 d = f3sub(p, c);
        if (gdot3(d, d) < s.w * s.w) return f3add(c, f3mul(gnormalize3(d), s.w));
    }
    float3 q;
    if (D.n_meshes > 0 && mesh_closest(D.mesh_nodes, D.mesh_tris, p, q) >= 0) return q;
    return p;
}

// FlipSim::CheckParticleSolidConstraints for one FLUID particle (flip.cpp:183-227).
__device__ void solid_constraints(const SceneDev& D, float3& p, float3& u, float3 pt, float3 ut) {
    const float maxd = D.maxd;
    float3 origin = f3mul(pt, maxd);
    float3 dir = gnormalize3(f3sub(p, pt));
    float raynulltest = glength3(dir);
    if (!(raynulltest == raynulltest)) return;
    Hit hit = intersect_solids(D, origin, dir);
    float u_dir = glength3(ut);
    if (hit.hit) {
        float solidDistance = glength3(f3sub(origin, hit.point));
        float velocityDistance = glength3(f3sub(p, pt)) * maxd;
        if (solidDistance < velocityDistance) {
            p = f3div(f3add(origin, f3mul(f3mul(dir, .90f), solidDistance)), maxd);
            float3 r = f3sub(f3smul(2.0f * gdot3(dir, hit.normal), hit.normal), gnormalize3(dir));
            u = f3mul(gnormalize3(r), u_dir);
        }
    }
    float3 o2 = f3mul(p, maxd);
    if (inside_solid(D, o2)) {
        float3 nd = gnormalize3(dir);
        u = f3mul(make_float3(-nd.x, -nd.y, -nd.z), u_dir);
        p = f3add(pt, f3mul(u, D.dt));
    }
}

// ------------------------------------------------------------------------------------------
// BEGIN: frame++, AdjustParticlesStuckInSolids (flip.cpp:130-181), StoreTemp (flip.cpp:79-90)
// ------------------------------------------------------------------------------------------
__global__ void k_frame_inc(SceneDev* scenes, int k) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < k) scenes[s].frame += 1;
}

__global__ void k_begin_solids(DevState S) {
    SCENE_PREFIX(S.p_pref);
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= S.np) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, g)];
    float4 p4 = S.pos4[g];
    float4 v4 = S.vel4[g];
    if (has_solids(D) && type_of(v4) == ARIEL_FLUID) {
        const float maxd = D.maxd;
        float3 p = make_float3(p4.x, p4.y, p4.z);
        if (inside_solid(D, f3mul(p, maxd))) {
            float3 pt = p;
            float3 np = f3div(closest_solid_surface(D, f3mul(p, maxd)), maxd);
            float3 origin = f3mul(pt, maxd);
            float3 dir = gnormalize3(f3sub(np, pt));
            float d = glength3(f3sub(np, pt));
            float raynulltest = glength3(dir);
            p = np;
            if (raynulltest == raynulltest) {
                Hit hit = intersect_solids(D, origin, dir);
                float nearest = glength3(f3sub(origin, hit.point));
                p = f3div(f3add(origin, f3mul(f3mul(dir, 1.05f), nearest)), maxd);
                float3 u = f3mul(gnormalize3(dir), d);
                v4.x = u.x;
                v4.y = u.y;
                v4.z = u.z;
            }
            p4.x = p.x;
            p4.y = p.y;
            p4.z = p.z;
            S.pos4[g] = p4;
            S.vel4[g] = v4;
        }
    }
    S.pt4[g] = p4;
    S.ut4[g] = v4;
}

// ------------------------------------------------------------------------------------------
// Sort-by-cell (replaces ParticleGrid::Sort, particlegrid.cpp:140-172)
// ------------------------------------------------------------------------------------------
__global__ void k_sort_key(DevState S) {
    SCENE_PREFIX(S.p_pref);
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= S.np) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, g)];
    float4 p = S.pos4[g];
    const int n = D.n;
    int ci = cell_coord(D.maxd, p.x), cj = cell_coord(D.maxd, p.y), ck = cell_coord(D.maxd, p.z);
    uint32_t c = (uint32_t)(D.c_begin + ((long long)ci * n + cj) * n + ck);
    S.key[g] = c;
    S.off[g] = atomicAdd(&S.count[c], 1u);
}

__global__ void k_sort_scatter(DevState S) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= S.np) return;
    uint32_t c = S.key[g];
    S.sid[S.start[c] + S.off[g]] = (uint32_t)g;
}

// Restores ascending particle id inside each cell (the reference's append order): cells of up
// to kSortRegs particles are sorted in registers; larger ones are listed (in the arrival-offset
// array, free once the scatter has run; `nbig` counts them) for k_sort_big.
constexpr int kSortRegs = 16;
__global__ void k_sort_cells(DevState S, uint32_t* nbig) {
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= S.nc) return;
    uint32_t a = S.start[c], b = S.start[c + 1];
    if (b - a < 2) return;
    uint32_t* seg = S.sid + a;
    uint32_t m = b - a;
    if (m > kSortRegs) {
        S.off[atomicAdd(nbig, 1u)] = (uint32_t)c;  // fewer than np / kSortRegs such cells
        return;
    }
    {
        uint32_t v[kSortRegs];
#pragma unroll
        for (int i = 0; i < kSortRegs; ++i) v[i] = i < (int)m ? seg[i] : 0xffffffffu;
        // odd-even transposition sort of the fixed-size array (the padding sorts last)
#pragma unroll
        for (int r = 0; r < kSortRegs; ++r)
#pragma unroll
            for (int i = r & 1; i + 1 < kSortRegs; i += 2) {
                const uint32_t lo = min(v[i], v[i + 1]), hi = max(v[i], v[i + 1]);
                v[i] = lo;
                v[i + 1] = hi;
            }
#pragma unroll
        for (int i = 0; i < kSortRegs; ++i)
            if (i < (int)m) seg[i] = v[i];
    }
}

// The listed cells, one warp each: the segment is copied to shared memory and every id is
// written to its rank, the number of smaller ids in the cell (ids are distinct), so the cell
// ends in ascending id order as after an insertion sort, in m^2 / 32 comparisons per lane instead
// of a serial chain of global loads and stores.  A segment beyond the shared copy (more than
// kBigCell particles in one cell) falls back to one lane's insertion sort in place.
constexpr int kBigCell = 1024;
constexpr int kBigWarps = 8;
constexpr int kSortBigBlocks = 296;  // a grid-stride loop over the listed cells
__global__ void __launch_bounds__(32 * kBigWarps) k_sort_big(DevState S, const uint32_t* nbig) {
    __shared__ uint32_t buf[kBigWarps][kBigCell];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t count = *nbig;
    for (uint32_t q = blockIdx.x * kBigWarps + w; q < count; q += gridDim.x * kBigWarps) {
        const uint32_t c = S.off[q];
        const uint32_t a = S.start[c], m = S.start[c + 1] - a;
        uint32_t* seg = S.sid + a;
        if (m > (uint32_t)kBigCell) {
            if (lane == 0)
                for (uint32_t i = 1; i < m; ++i) {
                    const uint32_t v = seg[i];
                    uint32_t j = i;
                    while (j > 0 && seg[j - 1] > v) {
                        seg[j] = seg[j - 1];
                        --j;
                    }
                    seg[j] = v;
                }
            __syncwarp();
            continue;
        }
        for (uint32_t i = lane; i < m; i += 32) buf[w][i] = seg[i];
        __syncwarp();
        for (uint32_t i = lane; i < m; i += 32) {
            const uint32_t v = buf[w][i];
            uint32_t r = 0;
            for (uint32_t j = 0; j < m; ++j) r += buf[w][j] < v ? 1u : 0u;
            seg[r] = v;
        }
        __syncwarp();
    }
}

__global__ void k_sort_permute(DevState S) {
    SCENE_PREFIX(S.p_pref);
    long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S.np) return;
    uint32_t g = S.sid[s];
    float4 p = S.pos4[g];
    float4 v = S.vel4[g];
    S.spos4[s] = p;
    S.svel4[s] = v;
    // SplatParticlesToMACGrid's clamped grid position (particlegridoperations.inl:172-174);
    // non-FLUID particles are placed out of every face's reach (they are skipped, :170)
    const float maxd = S.scenes[find_scene(pref_s, S.k, s)].maxd;
    float4 gp;
    if (type_of(v) == ARIEL_FLUID) {
        gp.x = gmax(0.0f, gmin(maxd, maxd * p.x));
        gp.y = gmax(0.0f, gmin(maxd, maxd * p.y));
        gp.z = gmax(0.0f, gmin(maxd, maxd * p.z));
        gp.w = p.w;
    } else {
        gp = make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.0f);
    }
    S.gpos4[s] = gp;
}

// ------------------------------------------------------------------------------------------
// FlipSim::ComputeDensity (flip.cpp:697-733): one thread per slot, 27-cell gather.
// ------------------------------------------------------------------------------------------
// weightsum over slots [a, b) in slot order, with the Smooth kernel's division either exact
// (POW2: h^2 a power of two, so r2 / h^2 == r2 * inv_hh) or as written.
template <bool POW2>
__device__ __forceinline__ float density_run(const float4* __restrict__ sp, uint32_t a, uint32_t b, float px,
                                             float py, float pz, float hk, float inv_hh, float weightsum) {
    const float2 nxy = make_float2(-px, -py);
#pragma unroll 4
    for (uint32_t t = a; t < b; ++t) {
        const float4 q = sp[t];
        const float sqd = sqrlength_xy2(q, nxy, pz);
        const float weight = q.w * (POW2 ? gmax(1.0f - sqd * inv_hh, 0.0f) : smooth_k(sqd, hk));
        weightsum = weightsum + weight;
    }
    return weightsum;
}

// At most 40 registers (three 512-thread blocks per SM): the issue-bound gather gains from the
// extra resident warps more than it loses to an 8-byte spill (5-6% faster measured).
__global__ void __launch_bounds__(512, 3) k_density(DevState S) {
    SCENE_PREFIX(S.p_pref);
    long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S.np) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, s)];
    float4 p = S.spos4[s];
    if (type_of(S.svel4[s]) == ARIEL_SOLID) {
        S.dens[s] = 1.0f;
        return;
    }
    const int n = D.n;
    const float hk = D.dens_h;
    int ci = cell_coord(D.maxd, p.x), cj = cell_coord(D.maxd, p.y), ck = cell_coord(D.maxd, p.z);
    int z0 = max(ck - 1, 0), z1 = min(ck + 1, n - 1);
    float weightsum = 0.0f;
    for (int sx = ci - 1; sx <= ci + 1; ++sx) {
        if (sx < 0 || sx > n - 1) continue;
        for (int sy = cj - 1; sy <= cj + 1; ++sy) {
            if (sy < 0 || sy > n - 1) continue;
            long long cb = D.c_begin + ((long long)sx * n + sy) * n;
            uint32_t a = S.start[cb + z0], b = S.start[cb + z1 + 1];
            weightsum = D.dens_pow2 ? density_run<true>(S.spos4, a, b, p.x, p.y, p.z, hk, D.dens_inv_hh, weightsum)
                                    : density_run<false>(S.spos4, a, b, p.x, p.y, p.z, hk, D.dens_inv_hh, weightsum);
        }
    }
    S.dens[s] = weightsum / D.max_density;
}

__global__ void k_fill_dens(DevState S, float v) {
    long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S.np) S.dens[s] = v;
}

__global__ void k_scatter_density(DevState S, float* out) {
    long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S.np) out[S.sid[s]] = S.dens[s];
}

// ------------------------------------------------------------------------------------------
// FlipSim::ApplyExternalForces (flip.cpp:682-695): on the slot copy and the id-order state.
// ------------------------------------------------------------------------------------------
__global__ void k_forces(DevState S) {
    SCENE_PREFIX(S.p_pref);
    long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S.np) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, s)];
    float4 v = S.svel4[s];
    for (int j = 0; j < D.n_forces; ++j) {
        v.x = v.x + D.fdt[j][0];
        v.y = v.y + D.fdt[j][1];
        v.z = v.z + D.fdt[j][2];
    }
    S.svel4[s] = v;
    S.vel4[S.sid[s]] = v;
}

// ------------------------------------------------------------------------------------------
// SplatParticlesToMACGrid (particlegridoperations.inl:146-249): every face gathers the FLUID
// particles of its 2x4x4 cell block (GetWallNeighbors, particlegrid.cpp:52-73) with the
// Sharpen kernel of radius 1.4 cells.  Face-parallel, so no atomics and a fixed order.
//
// A thread takes F consecutive faces of one row (same axis, i and j; k, k+1, ...).
// Their blocks share the x and y cell columns, so the thread walks each column once over the
// union of the faces' z ranges: every candidate record is loaded once, its x and y distance
// terms computed once, and the velocity component read once for all the faces it reaches.
// Each face still sees exactly its own contributors in the reference's order (cells sx, sy, z
// ascending, ids ascending inside a cell).  For x and y faces a record in the union but outside
// a face's block (z cells k-2 .. k+1) lies at least 1.5 cells from it along z (gpos is maxd * p
// clamped, its cell the truncation of gpos clamped to maxd - 1), and one in a cell pruned for
// that face lies beyond 1.1 radii; both give r2 >= 1.4^2, the test that drops a record, exactly
// as the per-face walk drops its zero-weight records.  A z face's block spans only cells k-1
// and k, and records of cell k+1 can lie within the radius, so there each record's cell (from
// its gpos) selects the two faces whose blocks hold it.
// Blocks take thirds of the group range in turn (block b: third b % 3), so the three face axes
// of a region run together and read the particle records from L2 once instead of three times.
// ------------------------------------------------------------------------------------------
constexpr long long kP2gThreads = 2500000;

__device__ __forceinline__ float face_offset_z(int axis, int k) { return axis == 2 ? (float)k : k + 0.5f; }

template <int F>
__device__ __forceinline__ void p2g_row(const DevState& S, const SceneDev& D, int axis, int i, int j, int k, int nk,
                                        float* __restrict__ out) {
    const int n = D.n;
    // face centre (x, y shared by the row) and the union of the GetWallNeighbors blocks
    // [index - nn, index + nn - 1] of faces k .. k + nk - 1
    float fx, fy;
    int xlo, xhi, ylo, yhi, zlo, zhi;
    if (axis == 0) {
        fx = (float)i; fy = j + 0.5f;
        xlo = i - 1; xhi = i; ylo = j - 2; yhi = j + 1; zlo = k - 2; zhi = k + nk;
    } else if (axis == 1) {
        fx = i + 0.5f; fy = (float)j;
        xlo = i - 2; xhi = i + 1; ylo = j - 1; yhi = j; zlo = k - 2; zhi = k + nk;
    } else {
        fx = i + 0.5f; fy = j + 0.5f;
        xlo = i - 2; xhi = i + 1; ylo = j - 2; yhi = j + 1; zlo = k - 1; zhi = k + nk - 1;
    }
    xlo = max(xlo, 0); xhi = min(xhi, n - 1);
    ylo = max(ylo, 0); yhi = min(yhi, n - 1);
    zlo = max(zlo, 0); zhi = min(zhi, n - 1);
    const float RE = 1.4f;
    const float RE2 = RE * RE;
    // Cells whose nearest point is farther than the Sharpen radius (with a 10% margin over any
    // rounding) from every face of the run hold only particles whose weight is exactly 0.  A
    // cell below the run is nearest to its first face, one above it to its last.
    const float LIM = 1.1f * RE2;
    const float fz_lo = face_offset_z(axis, k), fz_hi = face_offset_z(axis, k + nk - 1);
    float fz[F];
#pragma unroll
    for (int f = 0; f < F; ++f) fz[f] = face_offset_z(axis, k + f);
    const float2 nfxy = make_float2(-fx, -fy);
    const float* __restrict__ vel = reinterpret_cast<const float*>(S.svel4) + axis;
    const float maxd_m1 = D.maxd - 1.0f;
    float sumw[F], sumu[F];
#pragma unroll
    for (int f = 0; f < F; ++f) sumw[f] = sumu[f] = 0.0f;
    if (zlo <= zhi) {
        for (int sx = xlo; sx <= xhi; ++sx) {
            const float gx = axis_gap2(fx, (float)sx, (float)(sx + 1));
            if (gx > LIM) continue;
            for (int sy = ylo; sy <= yhi; ++sy) {
                const float gxy = gx + axis_gap2(fy, (float)sy, (float)(sy + 1));
                if (gxy > LIM) continue;
                int z0 = zlo, z1 = zhi;
                while (z0 <= z1 && gxy + axis_gap2(fz_lo, (float)z0, (float)(z0 + 1)) > LIM) ++z0;
                while (z1 >= z0 && gxy + axis_gap2(fz_hi, (float)z1, (float)(z1 + 1)) > LIM) --z1;
                if (z0 > z1) continue;
                long long cb = D.c_begin + ((long long)sx * n + sy) * n;
                uint32_t a = S.start[cb + z0], b = S.start[cb + z1 + 1];
                for (uint32_t t = a; t < b; ++t) {
                    const float4 q = S.gpos4[t];
                    // sqrlength_xy2's sum, (dx^2 + dy^2) + dz^2, with the first term shared
                    const float2 d = __fadd2_rn(make_float2(q.x, q.y), nfxy);
                    const float2 s2 = __fmul2_rn(d, d);
                    const float sxy = s2.x + s2.y;
                    // faces f_lo .. f_hi of the run have this record's cell in their block
                    int f_lo = 0, f_hi = nk - 1;
                    if (axis == 2) {
                        const int cz = (int)gmin(q.z, maxd_m1);
                        f_lo = cz - k;
                        f_hi = min(cz - k + 1, nk - 1);
                    }
                    float r2[F];
                    bool any = false;
#pragma unroll
                    for (int f = 0; f < F; ++f) {
                        const float c = q.z - fz[f];
                        r2[f] = sxy + c * c;
                        // Sharpen is exactly 0 for r2 >= RE^2 (and non-FLUID records are far away)
                        any |= f >= f_lo && f <= f_hi && r2[f] < RE2;
                    }
                    if (!any) continue;
                    const float uc = vel[4 * (size_t)t];
#pragma unroll
                    for (int f = 0; f < F; ++f) {
                        if (f >= f_lo && f <= f_hi && r2[f] < RE2) {
                            const float w = q.w * sharpen_k(r2[f], RE);
                            sumu[f] += w * uc;
                            sumw[f] += w;
                        }
                    }
                }
            }
        }
    }
#pragma unroll
    for (int f = 0; f < F; ++f) {
        if (f < nk) {
            float val = 0.0f;
            if (sumw[f] > 0) val = sumu[f] / sumw[f];
            out[f] = val;
        }
    }
}

// Thread -> group of F faces, with the group range cut in thirds that blocks take in turn;
// `third` is the number of groups in one third (a multiple of the block size).  Five blocks per
// SM (48 registers; 50 unbounded, which the allocator rounds to four blocks): the latency-bound
// gather gains from the extra warps (64^3 16%, 160^3 4%, 256^3 5% faster; 128^3 level to 3%
// faster; six blocks, at 40 registers with spills, are slower).
template <int F>
__global__ void __launch_bounds__(kBlock, 5) k_p2g(DevState S, long long third) {
    SCENE_PREFIX(S.f_pref);
    const long long grp = (long long)(blockIdx.x % 3) * third + (long long)(blockIdx.x / 3) * blockDim.x + threadIdx.x;
    long long g = grp * F;
    if (g >= S.nf) return;
    const long long gend = min(g + F, S.nf);
    // a group that crosses a row (z faces: rows of n + 1) or a scene is walked in pieces
    while (g < gend) {
        const SceneDev& D = S.scenes[find_scene(pref_s, S.k, g)];
        int axis, i, j, k;
        face_ijk(D, g - D.f_begin, axis, i, j, k);
        const int ek = axis == 2 ? D.n + 1 : D.n;
        const int nk = (int)min((long long)(ek - k), gend - g);
        p2g_row<F>(S, D, axis, i, j, k, nk, S.u + g);
        g += nk;
    }
}

// ------------------------------------------------------------------------------------------
// Interpolate / InterpolateVelocity (particlegridoperations.inl:106-133)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float interp1(const float* __restrict__ q, int ey, int ez, float px, float py, float pz,
                                         float nx, float ny, float nz) {
    float x = gmax(0.0f, gmin(nx, px));
    float y = gmax(0.0f, gmin(ny, py));
    float z = gmax(0.0f, gmin(nz, pz));
    int i = (int)gmin(x, nx - 2);
    int j = (int)gmin(y, ny - 2);
    int k = (int)gmin(z, nz - 2);
    auto Q = [&](int a, int b, int c) { return q[((long long)a * ey + b) * ez + c]; };
    float fi1 = (float)(i + 1), fj1 = (float)(j + 1), fk1 = (float)(k + 1);
    float term1 = ((fi1 - x) * Q(i, j, k) + (x - i) * Q(i + 1, j, k)) * (fj1 - y);
    float term2 = ((fi1 - x) * Q(i, j + 1, k) + (x - i) * Q(i + 1, j + 1, k)) * (y - j);
    float term3 = ((fi1 - x) * Q(i, j, k + 1) + (x - i) * Q(i + 1, j, k + 1)) * (fj1 - y);
    float term4 = ((fi1 - x) * Q(i, j + 1, k + 1) + (x - i) * Q(i + 1, j + 1, k + 1)) * (y - j);
    return (fk1 - z) * (term1 + term2) + (z - k) * (term3 + term4);
}

__device__ __forceinline__ float3 interp_vel(const float* __restrict__ faces, int n, float3 p) {
    const long long per = (long long)n * n * (n + 1);
    const float X = (float)n;
    float3 u;
    u.x = interp1(faces, n, n, X * p.x, X * p.y - 0.5f, X * p.z - 0.5f, (float)(n + 1), X, X);
    u.y = interp1(faces + per, n + 1, n, X * p.x - 0.5f, X * p.y, X * p.z - 0.5f, X, (float)(n + 1), X);
    u.z = interp1(faces + 2 * per, n, n + 1, X * p.x - 0.5f, X * p.y - 0.5f, X * p.z, X, X, (float)(n + 1));
    return u;
}

// ------------------------------------------------------------------------------------------
// SolvePicFlip (flip.cpp:287-322) + AdvectParticles (flip.cpp:229-285) +
// CheckParticleSolidConstraints (flip.cpp:183-227), one thread per particle (id order).
// ------------------------------------------------------------------------------------------
__global__ void k_g2p_advect(DevState S) {
    SCENE_PREFIX(S.p_pref);
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= S.np) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, g)];
    const int n = D.n;
    float4 p4 = S.pos4[g];
    float4 v4 = S.vel4[g];
    const float* cur = S.u + D.f_begin;
    const float* prv = S.pu + D.f_begin;
    float3 p = make_float3(p4.x, p4.y, p4.z);
    float3 t = make_float3(v4.x, v4.y, v4.z);
    float3 du = interp_vel(prv, n, p);
    t = f3add(du, t);
    float3 pic = interp_vel(cur, n, p);
    const float pf = D.picflip;
    const float opf = 1.0f - pf;
    float3 u = f3add(f3smul(opf, pic), f3smul(pf, t));
    if (type_of(v4) == ARIEL_FLUID) {
        p = f3add(p, f3smul(D.dt, pic));
        const float r = 1.0f / D.maxd;
        p.x = gmax(r, gmin(1.0f - r, p.x));
        p.y = gmax(r, gmin(1.0f - r, p.y));
        p.z = gmax(r, gmin(1.0f - r, p.z));
        if (has_solids(D)) {
            // solid push-out against the static SOLID particles of the 27 cells
            const float maxd = D.maxd;
            unsigned ci = (unsigned)gmin((float)n - 1.0f, p.x * maxd);
            unsigned cj = (unsigned)gmin((float)n - 1.0f, p.y * maxd);
            unsigned ck = (unsigned)gmin((float)n - 1.0f, p.z * maxd);
            const float re = D.pushout_re;
            int z0 = max((int)ck - 1, 0), z1 = min((int)ck + 1, n - 1);
            for (int sx = (int)ci - 1; sx <= (int)ci + 1; ++sx) {
                if (sx < 0 || sx > n - 1) continue;
                for (int sy = (int)cj - 1; sy <= (int)cj + 1; ++sy) {
                    if (sy < 0 || sy > n - 1) continue;
                    long long cb = D.c_begin + ((long long)sx * n + sy) * n;
                    uint32_t a = S.solid_start[cb + z0], b = S.solid_start[cb + z1 + 1];
                    for (uint32_t q = a; q < b; ++q) {
                        float4 sp = S.solid_pos[q];
                        float3 d = f3sub(p, make_float3(sp.x, sp.y, sp.z));
                        float dist = glength3(d);
                        if (dist < re) {
                            float3 normal = make_float3(0, 0, 0);
                            if (glength3(normal) < 0.0000001f && dist != 0.0f) normal = gnormalize3(d);
                            p = f3add(p, f3smul(re - dist, normal));
                            u = f3sub(u, f3smul(gdot3(u, normal), normal));
                        }
                    }
                }
            }
            float4 pt = S.pt4[g], ut = S.ut4[g];
            solid_constraints(D, p, u, make_float3(pt.x, pt.y, pt.z), make_float3(ut.x, ut.y, ut.z));
        }
    }
    S.pos4[g] = make_float4(p.x, p.y, p.z, p4.w);
    S.vel4[g] = make_float4(u.x, u.y, u.z, v4.w);
}

// ------------------------------------------------------------------------------------------
// ResampleParticles + Resample (particleresampler.inl:35-148) + CheckParticleSolidConstraints,
// one thread per slot of the resampler's own Sort.  rand() becomes Philox keyed by
// (rng seed, frame, particle id, draw ordinal).
// ------------------------------------------------------------------------------------------
// Gap from x to cell c's box along one axis (unit coordinates); the boxes of the first and last
// cell extend to infinity because Sort clamps outside particles into them.
__device__ __forceinline__ float cell_gap2(float x, int c, int n, float ch) {
    float lo = c == 0 ? -INFINITY : c * ch;
    float hi = c == n - 1 ? INFINITY : (c + 1) * ch;
    return axis_gap2(x, lo, hi);
}

__device__ __forceinline__ void nb_range(float x, int n, int& lo, int& hi) {
    // GetCellNeighbors with a fractional index and radius 1 (particlegrid.cpp:32-35)
    lo = (int)(x - 1.0f);
    hi = (int)floorf(x + 1.0f);
    if (lo < 0) lo = 0;
    if (hi > n - 1) hi = n - 1;
}

constexpr int kResList = 16;

// Cells along one axis that can hold a particle within sqrt(lim) of x (unit coordinates):
// the particle's own cell c, plus c-1 / c+1 when their box is that close; clipped to the
// reference's neighbour range [lo, hi].  Visiting the selected cells in lexicographic order
// visits the contributing particles in ascending slot order, which is the reference's order.
__device__ __forceinline__ void axis_cells(float x, int c, int n, float ch, float lim, int& lo, int& hi) {
    int a = c, b = c;
    if (c - 1 >= lo && cell_gap2(x, c - 1, n, ch) <= lim) a = c - 1;
    if (c + 1 <= hi && cell_gap2(x, c + 1, n, ch) <= lim) b = c + 1;
    if (c < lo || c > hi) {  // own cell outside the range (clamped positions): keep the range
        a = lo;
        b = hi;
    }
    lo = a;
    hi = b;
}

// The slot range of column (sx, sy) over z cells [zl, zh], without the end cells whose box is
// farther than sqrt(lim) from x in 3D (gxy: the column's squared x-y gap); empty (a == b) when
// the whole column is.  Only cells at the ends of the range can drop out, since the gap grows
// away from the point, so the remaining slots stay contiguous and in order.
__device__ __forceinline__ void column_slots(const DevState& S, const SceneDev& D, int sx, int sy, int zl, int zh,
                                             float z, float gxy, float ch, float lim, uint32_t& a, uint32_t& b) {
    const int n = D.n;
    a = b = 0;
    if (gxy > lim) return;
    while (zl <= zh && gxy + cell_gap2(z, zl, n, ch) > lim) ++zl;
    while (zh >= zl && gxy + cell_gap2(z, zh, n, ch) > lim) --zh;
    if (zl > zh) return;
    const long long cb = D.c_begin + ((long long)sx * n + sy) * n;
    a = S.start[cb + zl];
    b = S.start[cb + zh + 1];
}

// The resampler runs as two kernels over the slots of its own Sort: springs (the target
// position t), then the velocity at t and the acceptance.  In both, each thread walks those of
// the reference's 27 neighbour cells that reach within the kernel radius (about half a cell,
// so usually 2 per axis), testing only distance, records the few candidates in ascending slot
// order -- the reference's summation order -- and then evaluates them with the reference's
// exact arithmetic.  Neighbours outside the radius contribute exactly nothing.
// Five blocks per SM (51 registers, a 12-byte spill): 1-2% faster than four.
__global__ void __launch_bounds__(kBlock, 5) k_resample_spring(DevState S) {
    SCENE_PREFIX(S.p_pref);
    __shared__ uint32_t lst[kResList][kBlock];
    const int me = threadIdx.x;
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S.np) return;
    const float4 p4 = S.spos4[s];
    if (type_of(S.svel4[s]) != ARIEL_FLUID) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, s)];
    if (D.resample_every <= 0 || D.frame % D.resample_every != 0) return;
    const int n = D.n;
    const float maxd = D.maxd;
    const float dt = D.dt;
    const float re = D.resample_re;
    // Beyond re the Smooth weight is 0 (dist*dist, with dist the rounded root of d2, reaches
    // re^2 once d2 exceeds it by a few ulp), and a zero weight adds +-0, which leaves the target
    // position unchanged; the 1% margin covers that rounding.  Draws for the jitter branch
    // (dist <= 0.1 re) are inside the radius, so their order is unchanged.
    const float near2 = 1.01f * re * re;
    const uint32_t gid = (uint32_t)(S.sid[s] - D.p_begin);
    uint32_t draws = 0;
    float3 spring = make_float3(0, 0, 0);
    // particleresampler.inl:58-78 for one neighbour slot t (the particle itself is skipped)
    auto eval = [&](uint32_t t) {
        if (t == (uint32_t)s) return;
        const float springforce = 50.0f;
        float4 q = S.spos4[t];
        float3 d = make_float3(p4.x - q.x, p4.y - q.y, p4.z - q.z);
        float dist = sqrtf(gdot3(d, d));
        float w = springforce * q.w * smooth_fast(dist * dist, re, D.re_pow2, D.re_inv_hh);
        if (dist > 0.1f * re) {
            spring.x += w * (p4.x - q.x) / dist * re;
            spring.y += w * (p4.y - q.y) / dist * re;
            spring.z += w * (p4.z - q.z) / dist * re;
        } else if (type_of(S.svel4[t]) == ARIEL_FLUID) {
            uint4 rv = philox4x32_10(make_uint4(gid, (uint32_t)D.frame, draws++, kTagResample),
                                     (uint32_t)D.rng_seed, (uint32_t)(D.rng_seed >> 32));
            spring.x += 0.01f * re / dt * (float)(rv.x % 101u) / 100.0f;
            spring.y += 0.01f * re / dt * (float)(rv.y % 101u) / 100.0f;
            spring.z += 0.01f * re / dt * (float)(rv.z % 101u) / 100.0f;
        } else {
            // SOLID neighbour: its normal m_n is zero for scene-generated solids
            spring.x += 0.05f * re / dt * 0.0f;
            spring.y += 0.05f * re / dt * 0.0f;
            spring.z += 0.05f * re / dt * 0.0f;
        }
    };
    int xl, xh, yl, yh, zl, zh;
    // of the reference's 27 cells, only those within the candidate radius (5% margin over the
    // test below, for the rounding of the cell boxes)
    const float ch = 1.0f / maxd, lim = 1.05f * near2;
    {
        const float gx = gmax(0.0f, gmin(maxd, maxd * p4.x)), gy = gmax(0.0f, gmin(maxd, maxd * p4.y)),
                    gz = gmax(0.0f, gmin(maxd, maxd * p4.z));
        nb_range(gx, n, xl, xh);
        nb_range(gy, n, yl, yh);
        nb_range(gz, n, zl, zh);
        axis_cells(p4.x, min((int)gx, n - 1), n, ch, lim, xl, xh);
        axis_cells(p4.y, min((int)gy, n - 1), n, ch, lim, yl, yh);
        axis_cells(p4.z, min((int)gz, n - 1), n, ch, lim, zl, zh);
    }
    int nl = 0;
    const float2 npxy = make_float2(-p4.x, -p4.y);
    if (zl <= zh) {
        for (int sx = xl; sx <= xh; ++sx)
            for (int sy = yl; sy <= yh; ++sy) {
                uint32_t a, b;
                column_slots(S, D, sx, sy, zl, zh, p4.z,
                             cell_gap2(p4.x, sx, n, ch) + cell_gap2(p4.y, sy, n, ch), ch, lim, a, b);
                for (uint32_t t = a; t < b;) {
                    // a run of at most the list's free room: the list cannot overflow inside it,
                    // so each candidate is stored unconditionally and kept by advancing nl
                    const uint32_t e = min(b, t + (uint32_t)(kResList - nl));
#pragma unroll 4
                    for (; t < e; ++t) {
                        const float4 q = S.spos4[t];
                        lst[nl][me] = t;
                        nl += sqrlength_xy2(q, npxy, p4.z) < near2 ? 1 : 0;
                    }
                    if (nl == kResList) {
                        for (int i = 0; i < nl; ++i) eval(lst[i][me]);
                        nl = 0;
                    }
                }
            }
    }
    for (int i = 0; i < nl; ++i) eval(lst[i][me]);
    float4 t4;
    t4.x = p4.x + dt * spring.x;
    t4.y = p4.y + dt * spring.y;
    t4.z = p4.z + dt * spring.z;
    t4.w = 0.0f;
    S.gpos4[s] = t4;  // the P2G records are rebuilt by the next Sort
}

__global__ void __launch_bounds__(kBlock, 4) k_resample_velocity(DevState S) {
    SCENE_PREFIX(S.p_pref);
    __shared__ uint32_t lst[kResList][kBlock];
    const int me = threadIdx.x;
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S.np) return;
    const float4 v4 = S.svel4[s];
    if (type_of(v4) != ARIEL_FLUID) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, s)];
    if (D.resample_every <= 0 || D.frame % D.resample_every != 0) return;
    const int n = D.n;
    const float maxd = D.maxd;
    const float re = D.resample_re;
    const float re2 = re * re;
    const float4 t4 = S.gpos4[s];
    const float3 t = make_float3(t4.x, t4.y, t4.z);
    float wsum = 0.0f;
    float3 ru = make_float3(0, 0, 0);
    // Resample (particleresampler.inl:133-141) for one neighbour slot
    auto eval = [&](uint32_t q) {
        float4 nv = S.svel4[q];
        if (type_of(nv) != ARIEL_FLUID) return;
        float4 np = S.spos4[q];
        float dist2 = sqrlength(t.x, t.y, t.z, np.x, np.y, np.z);
        float w = np.w * sharpen_k(dist2, re);
        ru.x = ru.x + w * nv.x;
        ru.y = ru.y + w * nv.y;
        ru.z = ru.z + w * nv.z;
        wsum += w;
    };
    int xl, xh, yl, yh, zl, zh;
    const float ch = 1.0f / maxd, lim = 1.05f * re2;
    {
        const float gx = gmax(0.0f, gmin(maxd - 1, maxd * t.x)), gy = gmax(0.0f, gmin(maxd - 1, maxd * t.y)),
                    gz = gmax(0.0f, gmin(maxd - 1, maxd * t.z));
        nb_range(gx, n, xl, xh);
        nb_range(gy, n, yl, yh);
        nb_range(gz, n, zl, zh);
        axis_cells(t.x, min((int)gx, n - 1), n, ch, lim, xl, xh);
        axis_cells(t.y, min((int)gy, n - 1), n, ch, lim, yl, yh);
        axis_cells(t.z, min((int)gz, n - 1), n, ch, lim, zl, zh);
    }
    int nl = 0;
    const float2 ntxy = make_float2(-t.x, -t.y);
    if (zl <= zh) {
        for (int sx = xl; sx <= xh; ++sx)
            for (int sy = yl; sy <= yh; ++sy) {
                uint32_t a, b;
                column_slots(S, D, sx, sy, zl, zh, t.z,
                             cell_gap2(t.x, sx, n, ch) + cell_gap2(t.y, sy, n, ch), ch, lim, a, b);
                for (uint32_t q = a; q < b;) {
                    // runs of at most the list's free room, as in k_resample_spring; Sharpen is
                    // exactly 0 for dist2 >= re^2
                    const uint32_t e = min(b, q + (uint32_t)(kResList - nl));
#pragma unroll 4
                    for (; q < e; ++q) {
                        const float4 np = S.spos4[q];
                        lst[nl][me] = q;
                        nl += sqrlength_xy2(np, ntxy, t.z) < re2 ? 1 : 0;
                    }
                    if (nl == kResList) {
                        for (int i = 0; i < nl; ++i) eval(lst[i][me]);
                        nl = 0;
                    }
                }
            }
    }
    for (int i = 0; i < nl; ++i) eval(lst[i][me]);
    if (wsum != 0.0f)
        ru = f3div(ru, wsum);
    else
        ru = make_float3(v4.x, v4.y, v4.z);
    const float4 p4 = S.spos4[s];
    float3 p = make_float3(p4.x, p4.y, p4.z);
    float3 u = make_float3(v4.x, v4.y, v4.z);
    if (!(has_solids(D) && inside_solid(D, f3mul(t, maxd)))) {
        p = t;
        u = ru;
    }
    if (has_solids(D))
        solid_constraints(D, p, u, make_float3(p4.x, p4.y, p4.z), make_float3(v4.x, v4.y, v4.z));
    const uint32_t g = S.sid[s];
    S.pos4[g] = make_float4(p.x, p.y, p.z, p4.w);
    S.vel4[g] = make_float4(u.x, u.y, u.z, v4.w);
}

// ------------------------------------------------------------------------------------------
// Reseeding (no counterpart in the reference, which never adds or removes particles).  On
// frames divisible by reseed_every, after the resampler, particles move from crowded cells to
// sparse interior ones; the particle count, ids, masses and types are kept.  The cells are
// counted by the resampler's own Sort (the positions after advection; the resampler's moves are
// a fraction of a cell).  A FLUID cell holding m > reseed_max particles gives m - reseed_max of
// them, its highest ids first; an interior FLUID cell (all six neighbours FLUID) holding
// m < reseed_min receives reseed_min - m.  Within each scene the r-th given particle (cells in
// index order) fills the r-th received place (cells in index order) while both last.  A moved
// particle lands at a Philox-drawn point of its new cell, at least 5% of a cell from its faces,
// and takes the grid's PIC velocity there.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ bool reseed_frame(const SceneDev& D) {
    return D.reseed_every > 0 && D.frame % D.reseed_every == 0;
}

__global__ void k_reseed_count(DevState S) {
    SCENE_PREFIX(S.c_pref);
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= S.nc) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, c)];
    uint32_t give = 0, take = 0;
    if (reseed_frame(D) && S.flags[c] == ARIEL_FLUID) {
        const uint32_t m = S.count[c];
        if (m > (uint32_t)D.reseed_max) {
            give = m - (uint32_t)D.reseed_max;
        } else if (m < (uint32_t)D.reseed_min) {
            const int n = D.n;
            int i, j, k;
            cell_ijk(D, c - D.c_begin, i, j, k);
            bool interior = i > 0 && i < n - 1 && j > 0 && j < n - 1 && k > 0 && k < n - 1;
            if (interior) {
                const long long nn = (long long)n * n;
                interior = S.flags[c - nn] == ARIEL_FLUID && S.flags[c + nn] == ARIEL_FLUID &&
                           S.flags[c - n] == ARIEL_FLUID && S.flags[c + n] == ARIEL_FLUID &&
                           S.flags[c - 1] == ARIEL_FLUID && S.flags[c + 1] == ARIEL_FLUID;
            }
            if (interior) take = (uint32_t)D.reseed_min - m;
        }
    }
    S.rs_excess[c] = give;
    S.rs_deficit[c] = take;
}

// One thread per given particle (grid-stride over the scan's total, so a crowded cell's
// particles spread over many threads): the giving cell and the receiving cell are found by
// binary search over the two scans.
__device__ __forceinline__ long long last_at_or_below(const uint32_t* __restrict__ scan, long long lo, long long hi,
                                                      uint32_t v) {
    // the largest q in [lo, hi] with scan[q] <= v (scan does not decrease; scan[lo] <= v)
    while (lo < hi) {
        const long long mid = (lo + hi + 1) >> 1;
        if (scan[mid] <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

constexpr int kReseedBlocks = 4 * 148;  // four blocks on each of a B200's SMs

__global__ void k_reseed_move(DevState S) {
    SCENE_PREFIX(S.c_pref);
    const uint32_t total = S.rs_escan[S.nc];
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < total; x += gridDim.x * blockDim.x) {
        // the giving cell c (rs_escan[c] <= x < rs_escan[c + 1]) and the unit u inside it
        const long long c = last_at_or_below(S.rs_escan, 0, S.nc - 1, x);
        const uint32_t u = x - S.rs_escan[c];
        const SceneDev& D = S.scenes[find_scene(pref_s, S.k, c)];
        const int n = D.n;
        const long long cb = D.c_begin, ce = cb + (long long)n * n * n;
        const uint32_t d0 = S.rs_dscan[cb], dtot = S.rs_dscan[ce] - d0;
        const uint32_t r = x - S.rs_escan[cb];  // rank of this unit in its scene
        if (r >= dtot) continue;
        const uint32_t g = S.sid[S.start[c + 1] - 1 - u];  // the cell's highest ids first
        if (type_of(S.vel4[g]) != ARIEL_FLUID) continue;
        const long long q = last_at_or_below(S.rs_dscan, cb, ce - 1, d0 + r);
        int i, j, k;
        cell_ijk(D, q - cb, i, j, k);
        const uint4 rv = philox4x32_10(make_uint4(g - (uint32_t)D.p_begin, (uint32_t)D.frame, 0u, kTagReseed),
                                       (uint32_t)D.rng_seed, (uint32_t)(D.rng_seed >> 32));
        const float maxd = D.maxd;
        const float k24 = 1.0f / 16777216.0f;
        const float fx = 0.05f + 0.9f * ((float)(rv.x >> 8) * k24);
        const float fy = 0.05f + 0.9f * ((float)(rv.y >> 8) * k24);
        const float fz = 0.05f + 0.9f * ((float)(rv.z >> 8) * k24);
        const float3 p = make_float3(((float)i + fx) / maxd, ((float)j + fy) / maxd, ((float)k + fz) / maxd);
        const float3 v = interp_vel(S.u + D.f_begin, n, p);
        const float4 p4 = S.pos4[g], v4 = S.vel4[g];
        S.pos4[g] = make_float4(p.x, p.y, p.z, p4.w);
        S.vel4[g] = make_float4(v.x, v.y, v.z, v4.w);
    }
}

__global__ void k_unpack_state(float4* pos4, float4* vel4, const float* __restrict__ pos,
                               const float* __restrict__ vel, long long n, int* err) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = pos4[i], v = vel4[i];
    p.x = pos[3 * i];
    p.y = pos[3 * i + 1];
    p.z = pos[3 * i + 2];
    v.x = vel[3 * i];
    v.y = vel[3 * i + 1];
    v.z = vel[3 * i + 2];
    if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z)))
        atomicOr(err, 2);
    pos4[i] = p;
    vel4[i] = v;
}

__global__ void k_pack_state(const float4* __restrict__ pos4, const float4* __restrict__ vel4, float* pos, float* vel,
                             long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = pos4[i], v = vel4[i];
    pos[3 * i] = p.x;
    pos[3 * i + 1] = p.y;
    pos[3 * i + 2] = p.z;
    vel[3 * i] = v.x;
    vel[3 * i + 1] = v.y;
    vel[3 * i + 2] = v.z;
}

}  // namespace

cudaError_t launch_unpack_state(float4* pos4, float4* vel4, const float* pos, const float* vel, long long n,
                                int* err, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_unpack_state<<<grid_for(n), kBlock, 0, st>>>(pos4, vel4, pos, vel, n, err);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_pack_state(const float4* pos4, const float4* vel4, float* pos, float* vel, long long n,
                              cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_pack_state<<<grid_for(n), kBlock, 0, st>>>(pos4, vel4, pos, vel, n);
    count_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------
cudaError_t launch_begin(const DevState& S, cudaStream_t st) {
    k_frame_inc<<<grid_for(S.k), kBlock, 0, st>>>(const_cast<SceneDev*>(S.scenes), S.k);
    count_launch();
    if (S.any_solid && S.np > 0) {
        k_begin_solids<<<grid_for(S.np), kBlock, 0, st>>>(S);
        count_launch();
    }
    return cudaGetLastError();
}

static cudaError_t sort_core(const DevState& S, void* scan_tmp, cudaStream_t st) {
    cudaMemsetAsync(S.count, 0, sizeof(uint32_t) * (size_t)S.nc, st);
    if (S.np > 0) {
        k_sort_key<<<grid_for(S.np), kBlock, 0, st>>>(S);
        count_launch();
    }
    cudaError_t e = launch_scan_u32(S.count, S.start, S.nc, scan_tmp, st);
    if (e != cudaSuccess) return e;
    if (S.np > 0) {
        // the scan's scratch is free again: its first word counts the cells for k_sort_big
        uint32_t* nbig = reinterpret_cast<uint32_t*>(scan_tmp);
        k_sort_scatter<<<grid_for(S.np), kBlock, 0, st>>>(S);
        cudaMemsetAsync(nbig, 0, sizeof(uint32_t), st);
        k_sort_cells<<<grid_for(S.nc), kBlock, 0, st>>>(S, nbig);
        k_sort_big<<<kSortBigBlocks, 32 * kBigWarps, 0, st>>>(S, nbig);
        k_sort_permute<<<grid_for(S.np), kBlock, 0, st>>>(S);
        count_launch(4);
    }
    return cudaGetLastError();
}

cudaError_t launch_sort(const DevState& S, void* scan_tmp, cudaStream_t st) { return sort_core(S, scan_tmp, st); }

cudaError_t launch_density(const DevState& S, cudaStream_t st) {
    if (S.np == 0) return cudaSuccess;
    // 512 threads: measured faster than 256 for this kernel alone (0.79 vs 0.90 ms at 128^3);
    // the kernel's launch bounds assume this block size
    constexpr int kDensityBlock = 512;
    k_density<<<grid_for(S.np, kDensityBlock), kDensityBlock, 0, st>>>(S);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_fill_dens(const DevState& S, float value, cudaStream_t st) {
    if (S.np == 0) return cudaSuccess;
    k_fill_dens<<<grid_for(S.np), kBlock, 0, st>>>(S, value);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_scatter_density(const DevState& S, float* out, cudaStream_t st) {
    if (S.np == 0) return cudaSuccess;
    k_scatter_density<<<grid_for(S.np), kBlock, 0, st>>>(S, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_forces(const DevState& S, cudaStream_t st) {
    if (S.np == 0) return cudaSuccess;
    k_forces<<<grid_for(S.np), kBlock, 0, st>>>(S);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_p2g(const DevState& S, int faces, cudaStream_t st) {
    if (S.nf == 0) return cudaSuccess;
    // Faces per thread: the largest of 4, 2, 1 that still leaves kP2gThreads threads (longer
    // runs read fewer records per face but leave too few warps to hide the gathers' latency on
    // small grids: measured best 1 at 64^3, 2 at 128^3, 4 at 256^3).
    const int F = faces ? faces : (S.nf >= 4 * kP2gThreads ? 4 : (S.nf >= 2 * kP2gThreads ? 2 : 1));
    const long long groups = (S.nf + F - 1) / F;
    const long long third_blocks = (groups + 3LL * kBlock - 1) / (3LL * kBlock);
    const unsigned blocks = (unsigned)(3 * third_blocks);
    if (F == 4)
        k_p2g<4><<<blocks, kBlock, 0, st>>>(S, third_blocks * kBlock);
    else if (F == 2)
        k_p2g<2><<<blocks, kBlock, 0, st>>>(S, third_blocks * kBlock);
    else
        k_p2g<1><<<blocks, kBlock, 0, st>>>(S, third_blocks * kBlock);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_g2p_advect(const DevState& S, cudaStream_t st) {
    if (S.np == 0) return cudaSuccess;
    k_g2p_advect<<<grid_for(S.np), kBlock, 0, st>>>(S);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_resample(const DevState& S, void* scan_tmp, cudaStream_t st) {
    // StoreTempParticleVelocities before the resampler (flip.cpp:119) needs no copy: the
    // resampler's constraint check reads pt/ut from the slot copies of its own Sort.
    cudaError_t e = sort_core(S, scan_tmp, st);
    if (e != cudaSuccess) return e;
    if (S.np == 0) return cudaSuccess;
    k_resample_spring<<<grid_for(S.np), kBlock, 0, st>>>(S);
    k_resample_velocity<<<grid_for(S.np), kBlock, 0, st>>>(S);
    count_launch(2);
    if (S.any_reseed) {
        // the kernels return at once on frames without reseeding; the scans stay (cheap)
        k_reseed_count<<<grid_for(S.nc), kBlock, 0, st>>>(S);
        count_launch();
        e = launch_scan_u32(S.rs_excess, S.rs_escan, S.nc, scan_tmp, st);
        if (e != cudaSuccess) return e;
        e = launch_scan_u32(S.rs_deficit, S.rs_dscan, S.nc, scan_tmp, st);
        if (e != cudaSuccess) return e;
        k_reseed_move<<<kReseedBlocks, kBlock, 0, st>>>(S);
        count_launch();
    }
    return cudaGetLastError();
}

}  // namespace ariel
