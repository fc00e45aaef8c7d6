// ariel_oracle.cpp -- TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline).
//
// CPU restatement of betajippity/Ariel's FLIP step.  Every function below names the reference
// function and lines it restates.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline load this file's library; the product never does.
//
// Pinned to the reference's own code compiled from its sources (oracle/ref_driver.cpp,
// oracle/_ref/): tests/test_reference_pin.py holds this file bit-identical to it.
//
// Restatement rules:
//  * float arithmetic in the reference's expression order, compiled with -ffp-contract=off so no
//    multiply-add is fused (the CUDA library is built with --fmad=false for the same reason);
//  * glm::min/max restated as glm's ternaries, glm::dot as (x*x + y*y) + z*z, glm::length as
//    sqrt(dot), glm::normalize as v * (1/sqrt(dot(v,v)));
//  * tbb::parallel_for -> OpenMP parallel for at the same loops; the reference's serial loops
//    (ParticleGrid::Sort, Product) stay serial;
//  * races of the reference are resolved as the serial lexicographic order would run them
//    (BuildPreconditioner solver.inl:108-134 and ApplyPreconditioner solver.inl:238-284 read
//    neighbours other workers write); rand() (particleresampler.inl:69-71) is replaced by a
//    Philox4x32-10 counter keyed by (seed, frame, particle id, draw ordinal);
//  * OpenVDB/mesh solids are replaced by analytic spheres (ray hit, inside test, closest point).

#include "ariel_oracle.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

// ---------------------------------------------------------------------------------------------
// glm restatement (the few operations the FLIP step uses)
// ---------------------------------------------------------------------------------------------
struct vec3 {
    float x, y, z;
};
inline vec3 mk(float x, float y, float z) { return vec3{x, y, z}; }
inline vec3 operator+(vec3 a, vec3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(vec3 a, vec3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(vec3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, vec3 a) { return mk(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(vec3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
inline vec3 operator-(vec3 a) { return mk(-a.x, -a.y, -a.z); }
inline float gmin(float x, float y) { return (y < x) ? y : x; }  // glm::min
inline float gmax(float x, float y) { return (x < y) ? y : x; }  // glm::max
inline float gdot(vec3 a, vec3 b) {
    vec3 t = mk(a.x * b.x, a.y * b.y, a.z * b.z);
    return (t.x + t.y) + t.z;
}
inline float glength(vec3 v) { return std::sqrt(gdot(v, v)); }
inline vec3 gnormalize(vec3 v) { return v * (1.0f / std::sqrt(gdot(v, v))); }

// src/math/kernels.inl:25-38
inline float Sqrlength(vec3 p0, vec3 p1) {
    float a = p0.x - p1.x;
    float b = p0.y - p1.y;
    float c = p0.z - p1.z;
    return a * a + b * b + c * c;
}
inline float Smooth(float r2, float h) { return gmax(1.0f - r2 / (h * h), 0.0f); }
inline float Sharpen(float r2, float h) { return gmax(h * h / gmax(r2, (float)1.0e-5) - 1.0f, 0.0f); }

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3",
// SC'11): ten rounds of two 32x32->64-bit products, Weyl key schedule.
// ---------------------------------------------------------------------------------------------
struct u4 {
    uint32_t v[4];
};
u4 philox(u4 c, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c.v[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c.v[2];
        u4 o;
        o.v[0] = (uint32_t)(p1 >> 32) ^ c.v[1] ^ k0;
        o.v[1] = (uint32_t)p1;
        o.v[2] = (uint32_t)(p0 >> 32) ^ c.v[3] ^ k1;
        o.v[3] = (uint32_t)p0;
        c = o;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}
const uint32_t kTagSeed = 0x53454544u;      // "SEED": initial lattice jitter
const uint32_t kTagResample = 0x5245534Du;  // "RESM": resampling jitter

// ---------------------------------------------------------------------------------------------
// Grid<T> (src/grid/grid.hpp:18-38, grid.inl:11-62): (dim+1)^3 storage, background value.
// ---------------------------------------------------------------------------------------------
template <class T>
struct Grid {
    int X = 0, Y = 0, Z = 0;
    T bg{};
    std::vector<T> v;
    void make(int dx, int dy, int dz, T b) {
        X = dx + 1;
        Y = dy + 1;
        Z = dz + 1;
        bg = b;
        v.assign((size_t)X * Y * Z, b);
    }
    T get(int i, int j, int k) const { return v[((size_t)i * Y + j) * Z + k]; }
    void set(int i, int j, int k, T val) { v[((size_t)i * Y + j) * Z + k] = val; }
    void clear() { std::fill(v.begin(), v.end(), bg); }
};

// Particle (src/grid/macgrid.inl:36-50)
struct Particle {
    vec3 p, u, n;
    float density, mass;
    int type;
    vec3 t, t2, ut, pt;
};

struct Sphere {
    vec3 c;  // world (grid) units
    float r;
};

struct Hit {
    bool hit;
    vec3 point, normal;
};

// A static solid mesh's triangle in world (grid) coordinates, with its mesh and its index across
// the scene's meshes (the tie-break key).
struct MTri {
    vec3 a, b, c;
    int mesh, key;
};

}  // namespace

struct ariel_ref {
    AsimSceneDesc desc;
    AsimParams prm;
    int n = 0;
    float maxd = 0;
    bool faithful = false;
    std::vector<Particle> parts;
    // ParticleGrid (src/grid/particlegrid.hpp:20-48): cell -> list index map (never reset) and
    // per-cell particle lists.
    Grid<int> pmap;
    std::vector<std::vector<int>> cells;
    std::vector<int> pcell;  // linear cell of each particle at the last Sort (for parity tests)
    // MacGrid m_mgrid / m_mgrid_previous (macgrid.inl:21-34)
    Grid<float> ux, uy, uz, D, P, L;
    Grid<int> A;
    Grid<float> pux, puy, puz;
    std::vector<double> P64;  // FP64-mode pressure (warm start)
    float max_density = 0;
    int frame = 0;
    bool inited = false;
    std::vector<Sphere> solids;
    std::vector<MTri> mtris;         // solid meshes, brute force (no tree)
    std::vector<vec3> mlo, mhi;      // per mesh world bounding box
    AsimStats st{};
    double stage_ms[ARIEL_STAGE_COUNT] = {};
};

namespace {

using Sim = ariel_ref;

// ---------------------------------------------------------------------------------------------
// Analytic solid spheres (replaces the mesh BVH of Scene::IntersectSolidGeoms scene.cpp:425-434,
// CheckPointInsideSolidGeom scene.cpp:382-402 and the OpenVDB closest-point projection
// levelset.cpp:175-193).  All in world (grid) units.
// ---------------------------------------------------------------------------------------------
// Static solid meshes, by brute force over every triangle (the CUDA library walks a tree; the
// results must not depend on it).  Ray-triangle test: Obj::RayTriangleTest
// (src/geom/obj/obj.cpp:354-398) with glm::cross / glm::dot as glm writes them.
inline vec3 gcross(vec3 x, vec3 y) {
    return mk(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
bool TriRay(const MTri& T, vec3 o, vec3 d, float& t) {
    vec3 e1 = T.b - T.a, e2 = T.c - T.a;
    vec3 pvec = gcross(d, e2);
    float det = gdot(e1, pvec);
    if (det == 0.0f) return false;
    float inv_det = 1.0f / det;
    vec3 tvec = o - T.a;
    float bx = gdot(tvec, pvec) * inv_det;
    vec3 qvec = gcross(tvec, e1);
    float by = gdot(d, qvec) * inv_det;
    t = gdot(e2, qvec) * inv_det;
    return bx >= 0.0f && by >= 0.0f && (bx + by) <= 1.0f;
}
// Closest point of a triangle (Ericson, Real-Time Collision Detection, 2005, section 5.1.5).
vec3 TriClosest(const MTri& T, vec3 p) {
    vec3 a = T.a, b = T.b, c = T.c;
    vec3 ab = b - a, ac = c - a, ap = p - a;
    float d1 = gdot(ab, ap), d2 = gdot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return a;
    vec3 bp = p - b;
    float d3 = gdot(ab, bp), d4 = gdot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return b;
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return a + ab * (d1 / (d1 - d3));
    vec3 cp = p - c;
    float d5 = gdot(ab, cp), d6 = gdot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return c;
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return a + ac * (d2 / (d2 - d6));
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f)
        return b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
    float denom = 1.0f / ((va + vb) + vc);
    return (a + ab * (vb * denom)) + ac * (vc * denom);
}
// Scene::CheckPointInsideSolidGeom (scene.cpp:382-402): odd hit count along +z, per mesh.
uint32_t MeshInsideBits(const Sim& s, vec3 p) {
    uint32_t bits = 0;
    for (const MTri& T : s.mtris) {
        float t;
        if (TriRay(T, p, mk(0, 0, 1), t) && t > 0.0f) bits ^= 1u << (T.mesh & 31);
    }
    return bits;
}
bool HasSolids(const Sim& s) { return !s.solids.empty() || !s.mtris.empty(); }

bool InsideSolid(const Sim& s, vec3 p) {
    for (const Sphere& sp : s.solids) {
        vec3 d = p - sp.c;
        if (gdot(d, d) < sp.r * sp.r) return true;
    }
    return !s.mtris.empty() && MeshInsideBits(s, p) != 0u;
}

Hit IntersectSolids(const Sim& s, vec3 o, vec3 dir) {
    Hit best{false, mk(0, 0, 0), mk(0, 0, 0)};
    float bestd = 0.0f;
    for (const Sphere& sp : s.solids) {
        vec3 oc = o - sp.c;
        float b = gdot(dir, oc);
        float c = gdot(oc, oc) - sp.r * sp.r;
        float disc = b * b - c;
        if (!(disc >= 0.0f)) continue;
        float sq = std::sqrt(disc);
        float t = -b - sq;
        if (!(t > 0.0f)) t = -b + sq;
        if (!(t > 0.0f)) continue;
        vec3 pt = o + dir * t;
        vec3 nrm = gnormalize(pt - sp.c);
        float d = glength(pt - o);
        // Intersection::CompareClosestAgainst (src/ray/ray.cpp:83-98): keep the nearer hit.
        if (!best.hit || !(bestd <= d)) {
            best = Hit{true, pt, nrm};
            bestd = d;
        }
    }
    // solid meshes after the spheres: the nearest triangle hit (t > 0), ties to the lower key
    int bt = -1;
    float bdist = 0.0f;
    vec3 bpt = mk(0, 0, 0);
    for (size_t i = 0; i < s.mtris.size(); ++i) {
        const MTri& T = s.mtris[i];
        float t;
        if (!TriRay(T, o, dir, t) || !(t > 0.0f)) continue;
        vec3 pt = o + dir * t;
        vec3 dv = pt - o;
        float dd = std::sqrt(gdot(dv, dv));
        if (bt < 0 || dd < bdist || (dd == bdist && T.key < s.mtris[bt].key)) {
            bt = (int)i;
            bdist = dd;
            bpt = pt;
        }
    }
    if (bt >= 0 && (!best.hit || !(bestd <= bdist))) {
        const MTri& T = s.mtris[bt];
        best = Hit{true, bpt, gnormalize(gcross(T.b - T.a, T.c - T.a))};
        bestd = bdist;
    }
    return best;
}

vec3 ClosestSolidSurface(const Sim& s, vec3 p) {
    for (const Sphere& sp : s.solids) {
        vec3 d = p - sp.c;
        if (gdot(d, d) < sp.r * sp.r) return sp.c + gnormalize(d) * sp.r;
    }
    // solid meshes: the closest surface point, ties to the lower key
    int bt = -1;
    float bd = 0.0f;
    vec3 q = p;
    for (size_t i = 0; i < s.mtris.size(); ++i) {
        const MTri& T = s.mtris[i];
        vec3 c = TriClosest(T, p);
        vec3 e = p - c;
        float d2 = gdot(e, e);
        if (bt < 0 || d2 < bd || (d2 == bd && T.key < s.mtris[bt].key)) {
            bt = (int)i;
            bd = d2;
            q = c;
        }
    }
    return q;
}

// ---------------------------------------------------------------------------------------------
// ParticleGrid (src/grid/particlegrid.cpp)
// ---------------------------------------------------------------------------------------------
inline int CellCoord(float maxd, float x) {
    // particlegrid.cpp:156-158 / flip.cpp:711-713
    return (int)gmax(0.0f, gmin((int)maxd - 1.0f, (float)(int(maxd)) * x));
}

// ParticleGrid::Sort (particlegrid.cpp:140-172): serial, m_grid never reset.
void Sort(Sim& s) {
    for (auto& c : s.cells) c.clear();
    const float maxd = s.maxd;
    int np = (int)s.parts.size();
    int cellscount = (int)s.cells.size();
    s.pcell.resize(np);
    for (int i = 0; i < np; ++i) {
        const Particle& p = s.parts[i];
        int cx = CellCoord(maxd, p.p.x), cy = CellCoord(maxd, p.p.y), cz = CellCoord(maxd, p.p.z);
        int idx = s.pmap.get(cx, cy, cz);
        if (idx >= 0) {
            s.cells[idx].push_back(i);
        } else {
            s.cells.push_back(std::vector<int>(1, i));
            s.pmap.set(cx, cy, cz, cellscount);
            cellscount++;
        }
        s.pcell[i] = (cx * s.n + cy) * s.n + cz;
    }
}

// ParticleGrid::GetCellNeighbors (particlegrid.cpp:28-50)
std::vector<int> GetCellNeighbors(const Sim& s, vec3 index, vec3 nn) {
    std::vector<int> out;
    const float dim = (float)s.n;
    for (int sx = (int)(index.x - nn.x); (float)sx <= index.x + nn.x; sx++) {
        for (int sy = (int)(index.y - nn.y); (float)sy <= index.y + nn.y; sy++) {
            for (int sz = (int)(index.z - nn.z); (float)sz <= index.z + nn.z; sz++) {
                if (sx < 0 || (float)sx > dim - 1 || sy < 0 || (float)sy > dim - 1 || sz < 0 ||
                    (float)sz > dim - 1)
                    continue;
                int ci = s.pmap.get(sx, sy, sz);
                if (ci >= 0)
                    for (int a : s.cells[ci]) out.push_back(a);
            }
        }
    }
    return out;
}

// ParticleGrid::GetWallNeighbors (particlegrid.cpp:52-73)
std::vector<int> GetWallNeighbors(const Sim& s, vec3 index, vec3 nn) {
    std::vector<int> out;
    const float dim = (float)s.n;
    for (int sx = (int)(index.x - nn.x); (float)sx <= index.x + nn.x - 1; sx++) {
        for (int sy = (int)(index.y - nn.y); (float)sy <= index.y + nn.y - 1; sy++) {
            for (int sz = (int)(index.z - nn.z); (float)sz <= index.z + nn.z - 1; sz++) {
                if (sx < 0 || (float)sx > dim - 1 || sy < 0 || (float)sy > dim - 1 || sz < 0 ||
                    (float)sz > dim - 1)
                    continue;
                int ci = s.pmap.get(sx, sy, sz);
                if (ci >= 0)
                    for (int a : s.cells[ci]) out.push_back(a);
            }
        }
    }
    return out;
}

// ParticleGrid::CellSDF (particlegrid.cpp:75-90)
float CellSDF(const Sim& s, int i, int j, int k, float density, int type) {
    float accm = 0.0f;
    int ci = s.pmap.get(i, j, k);
    if (ci >= 0) {
        for (int a : s.cells[ci]) {
            if (s.parts[a].type == type)
                accm += s.parts[a].density;
            else
                return 1.0f;
        }
    }
    float n0 = 1.0f / (density * density * density);
    return 0.2f * n0 - accm;
}

// ParticleGrid::BuildSDF (particlegrid.cpp:92-106)
void BuildSDF(Sim& s) {
    const int n = s.n;
    const float density = s.desc.density;
    s.L.clear();
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) s.L.set(i, j, k, CellSDF(s, i, j, k, density, ARIEL_FLUID));
}

// ParticleGrid::MarkCellTypes (particlegrid.cpp:108-138)
void MarkCellTypes(Sim& s) {
    const int n = s.n;
    const float density = s.desc.density;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) {
            for (int k = 0; k < n; ++k) {
                s.A.set(i, j, k, ARIEL_AIR);
                int ci = s.pmap.get(i, j, k);
                if (ci >= 0 && ci < (int)s.cells.size())
                    for (int a : s.cells[ci])
                        if (s.parts[a].type == ARIEL_SOLID) s.A.set(i, j, k, ARIEL_SOLID);
                if (s.A.get(i, j, k) != ARIEL_SOLID) {
                    bool isfluid = CellSDF(s, i, j, k, density, ARIEL_FLUID) < 0.0;
                    s.A.set(i, j, k, isfluid ? ARIEL_FLUID : ARIEL_AIR);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// FlipSim (src/sim/flip.cpp)
// ---------------------------------------------------------------------------------------------

// FlipSim::ComputeDensity (flip.cpp:697-733)
void ComputeDensity(Sim& s) {
    const float maxd = s.maxd;
    const long np = (long)s.parts.size();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < np; ++i) {
        Particle& pi = s.parts[i];
        if (pi.type == ARIEL_SOLID) {
            pi.density = 1.0f;
        } else {
            vec3 position = pi.p;
            position.x = (float)(int)gmax(0.0f, gmin((int)maxd - 1.0f, (int)maxd * position.x));
            position.y = (float)(int)gmax(0.0f, gmin((int)maxd - 1.0f, (int)maxd * position.y));
            position.z = (float)(int)gmax(0.0f, gmin((int)maxd - 1.0f, (int)maxd * position.z));
            std::vector<int> nb = GetCellNeighbors(s, position, mk(1, 1, 1));
            float weightsum = 0.0f;
            for (int m : nb) {
                float sqd = Sqrlength(s.parts[m].p, pi.p);
                float weight = s.parts[m].mass * Smooth(sqd, 4.0f * s.desc.density / maxd);
                weightsum = weightsum + weight;
            }
            pi.density = weightsum / s.max_density;
        }
    }
}

// FlipSim::ApplyExternalForces (flip.cpp:682-695)
void ApplyExternalForces(Sim& s) {
    const long np = (long)s.parts.size();
    const float dt = s.desc.stepsize;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < np; ++i)
        for (int j = 0; j < s.desc.n_forces; ++j) {
            vec3 f = mk(s.desc.forces[j][0], s.desc.forces[j][1], s.desc.forces[j][2]);
            s.parts[i].u = s.parts[i].u + f * dt;
        }
}

// FlipSim::StoreTempParticleVelocities (flip.cpp:79-90)
void StoreTemp(Sim& s) {
    const long np = (long)s.parts.size();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < np; ++i) {
        s.parts[i].pt = s.parts[i].p;
        s.parts[i].ut = s.parts[i].u;
    }
}

// SplatParticlesToMACGrid (particlegridoperations.inl:146-249)
void SplatParticlesToMACGrid(Sim& s) {
    const float RE = 1.4f;
    const int x = s.n, y = s.n, z = s.n;
    const float maxd = gmax(gmax((float)x, (float)y), (float)z);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < x + 1; ++i) {
        for (int j = 0; j < y + 1; ++j) {
            for (int k = 0; k < z + 1; ++k) {
                for (int axis = 0; axis < 3; ++axis) {
                    vec3 fc, nn;
                    if (axis == 0) {
                        if (!(j < y && k < z)) continue;
                        fc = mk((float)i, j + 0.5f, k + 0.5f);
                        nn = mk(1, 2, 2);
                    } else if (axis == 1) {
                        if (!(i < x && k < z)) continue;
                        fc = mk(i + 0.5f, (float)j, k + 0.5f);
                        nn = mk(2, 1, 2);
                    } else {
                        if (!(i < x && j < y)) continue;
                        fc = mk(i + 0.5f, j + 0.5f, (float)k);
                        nn = mk(2, 2, 1);
                    }
                    float sumw = 0.0f, sumu = 0.0f;
                    std::vector<int> nb = GetWallNeighbors(s, mk((float)i, (float)j, (float)k), nn);
                    for (int m : nb) {
                        const Particle& p = s.parts[m];
                        if (p.type == ARIEL_FLUID) {
                            vec3 pos;
                            pos.x = gmax(0.0f, gmin(maxd, maxd * p.p.x));
                            pos.y = gmax(0.0f, gmin(maxd, maxd * p.p.y));
                            pos.z = gmax(0.0f, gmin(maxd, maxd * p.p.z));
                            float w = p.mass * Sharpen(Sqrlength(pos, fc), RE);
                            float uc = axis == 0 ? p.u.x : (axis == 1 ? p.u.y : p.u.z);
                            sumu += w * uc;
                            sumw += w;
                        }
                    }
                    float val = 0.0f;
                    if (sumw > 0) val = sumu / sumw;
                    (axis == 0 ? s.ux : (axis == 1 ? s.uy : s.uz)).set(i, j, k, val);
                }
            }
        }
    }
}

// FlipSim::StorePreviousGrid (flip.cpp:324-363)
void StorePreviousGrid(Sim& s) {
    s.pux.v = s.ux.v;
    s.puy.v = s.uy.v;
    s.puz.v = s.uz.v;
}

// CheckWall (particlegridoperations.inl:37-43)
inline float CheckWall(const Grid<int>& A, int x, int y, int z) {
    return A.get(x, y, z) == ARIEL_SOLID ? 1.0f : -1.0f;
}

// EnforceBoundaryVelocity (particlegridoperations.inl:45-104)
void EnforceBoundaryVelocity(Sim& s) {
    const int x = s.n, y = s.n, z = s.n;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x + 1; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k) {
                if (i == 0 || i == x) s.ux.set(i, j, k, 0.0f);
                if (i < x && i > 0 && CheckWall(s.A, i, j, k) * CheckWall(s.A, i - 1, j, k) < 0)
                    s.ux.set(i, j, k, 0.0f);
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y + 1; ++j)
            for (int k = 0; k < z; ++k) {
                if (j == 0 || j == y) s.uy.set(i, j, k, 0.0f);
                if (j < y && j > 0 && CheckWall(s.A, i, j, k) * CheckWall(s.A, i, j - 1, k) < 0)
                    s.uy.set(i, j, k, 0.0f);
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z + 1; ++k) {
                if (k == 0 || k == z) s.uz.set(i, j, k, 0.0f);
                if (k < z && k > 0 && CheckWall(s.A, i, j, k) * CheckWall(s.A, i, j, k - 1) < 0)
                    s.uz.set(i, j, k, 0.0f);
            }
}

// Project divergence part (flip.cpp:420-437) and FlipGrid (solver.inl:42-56)
void DivergenceAndFlip(Sim& s) {
    const int x = s.n, y = s.n, z = s.n;
    const float h = 1.0f / s.maxd;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k) {
                float divergence = (s.ux.get(i + 1, j, k) - s.ux.get(i, j, k) + s.uy.get(i, j + 1, k) -
                                    s.uy.get(i, j, k) + s.uz.get(i, j, k + 1) - s.uz.get(i, j, k)) /
                                   h;
                s.D.set(i, j, k, divergence);
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k) s.D.set(i, j, k, -s.D.get(i, j, k));
}

// ---------------------------------------------------------------------------------------------
// Pressure solve (src/sim/solver.inl)
// ---------------------------------------------------------------------------------------------
struct Dims {
    int x, y, z;
};

// ARef (solver.inl:59-69)
inline float ARef(const Grid<int>& A, int i, int j, int k, int qi, int qj, int qk, Dims d) {
    if (i < 0 || i > d.x - 1 || j < 0 || j > d.y - 1 || k < 0 || k > d.z - 1 || A.get(i, j, k) != ARIEL_FLUID)
        return 0.0;
    if (qi < 0 || qi > d.x - 1 || qj < 0 || qj > d.y - 1 || qk < 0 || qk > d.z - 1 ||
        A.get(qi, qj, qk) != ARIEL_FLUID)
        return 0.0;
    return -1.0;
}

// PRef (solver.inl:72-78): returns the value only when it equals FLUID (1.0f) -- kept verbatim.
template <class G>
inline float PRef(const G& p, int i, int j, int k, Dims d) {
    if (i < 0 || i > d.x - 1 || j < 0 || j > d.y - 1 || k < 0 || k > d.z - 1 || p.get(i, j, k) != ARIEL_FLUID)
        return 0.0f;
    return p.get(i, j, k);
}

// ADiag (solver.inl:81-101)
inline float ADiag(const Grid<int>& A, const Grid<float>& L, int i, int j, int k, Dims d, int subcell) {
    float diag = 6.0;
    if (A.get(i, j, k) != ARIEL_FLUID) return diag;
    const int q[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
    for (int m = 0; m < 6; ++m) {
        int qi = q[m][0], qj = q[m][1], qk = q[m][2];
        if (qi < 0 || qi > d.x - 1 || qj < 0 || qj > d.y - 1 || qk < 0 || qk > d.z - 1 ||
            A.get(qi, qj, qk) == ARIEL_SOLID)
            diag -= 1.0;
        else if (A.get(qi, qj, qk) == ARIEL_AIR && subcell)
            diag -= L.get(qi, qj, qk) / gmin(1.0e-6f, L.get(i, j, k));
    }
    return diag;
}

// One cell of BuildPreconditioner (solver.inl:113-128)
inline void BuildPCCell(Grid<float>& pc, const Grid<int>& A, const Grid<float>& L, int i, int j, int k, Dims d,
                        int subcell, float a) {
    if (A.get(i, j, k) == ARIEL_FLUID) {
        float left = ARef(A, i - 1, j, k, i, j, k, d) * PRef(pc, i - 1, j, k, d);
        float bottom = ARef(A, i, j - 1, k, i, j, k, d) * PRef(pc, i, j - 1, k, d);
        float back = ARef(A, i, j, k - 1, i, j, k, d) * PRef(pc, i, j, k - 1, d);
        float diag = ADiag(A, L, i, j, k, d, subcell);
        float e = diag - (left * left) - (bottom * bottom) - (back * back);
        if (diag > 0) {
            if (e < a * diag) e = diag;
            pc.set(i, j, k, 1.0f / std::sqrt(e));
        }
    }
}

// BuildPreconditioner (solver.inl:104-135) with the serial-order meaning of its PRef reads:
// the neighbour terms are non-zero only where a FLUID neighbour's value is exactly 1.0f.  If the
// order-free evaluation yields no such value, it equals the serial evaluation; otherwise the
// serial order is run.
bool BuildPreconditioner(Grid<float>& pc, const Sim& s, int subcell) {
    const Dims d{s.n, s.n, s.n};
    const float a = 0.25f;
    Grid<float> pc0 = pc;  // fresh zero grid
    const int x = s.n;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < d.y; ++j)
            for (int k = 0; k < d.z; ++k) {
                if (s.A.get(i, j, k) == ARIEL_FLUID) {
                    float diag = ADiag(s.A, s.L, i, j, k, d, subcell);
                    float e = diag - (0.0f * 0.0f) - (0.0f * 0.0f) - (0.0f * 0.0f);
                    if (diag > 0) {
                        if (e < a * diag) e = diag;
                        pc0.set(i, j, k, 1.0f / std::sqrt(e));
                    }
                }
            }
    long ones = 0;
#pragma omp parallel for reduction(+ : ones) schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < d.y; ++j)
            for (int k = 0; k < d.z; ++k)
                if (s.A.get(i, j, k) == ARIEL_FLUID && pc0.get(i, j, k) == 1.0f) ones++;
    if (ones == 0) {
        pc = pc0;
        return false;
    }
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < d.y; ++j)
            for (int k = 0; k < d.z; ++k) BuildPCCell(pc, s.A, s.L, i, j, k, d, subcell, a);
    return true;
}

// XRef (solver.inl:138-154)
template <class G>
inline float XRef(const Grid<int>& A, const Grid<float>& L, const G& X, int fi, int fj, int fk, int pi, int pj,
                  int pk, Dims d, int subcell) {
    int i = std::min(std::max(0, pi), d.x - 1);
    int j = std::min(std::max(0, pj), d.y - 1);
    int k = std::min(std::max(0, pk), d.z - 1);
    if (A.get(i, j, k) == ARIEL_FLUID) return X.get(i, j, k);
    if (A.get(i, j, k) == ARIEL_SOLID) return X.get(fi, fj, fk);
    if (subcell) return L.get(i, j, k) / gmin(1.0e-6f, L.get(fi, fj, fk)) * X.get(fi, fj, fk);
    return 0.0f;
}

// ComputeAx (solver.inl:196-230)
void ComputeAx(const Sim& s, const Grid<float>& X, Grid<float>& target, int subcell) {
    const Dims d{s.n, s.n, s.n};
    float nn = (float)std::max(std::max(d.x, d.y), d.z);
    float h = 1.0f / (nn * nn);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.x; ++i)
        for (int j = 0; j < d.y; ++j)
            for (int k = 0; k < d.z; ++k) {
                if (s.A.get(i, j, k) == ARIEL_FLUID) {
                    float result = (6.0f * X.get(i, j, k) - XRef(s.A, s.L, X, i, j, k, i + 1, j, k, d, subcell) -
                                    XRef(s.A, s.L, X, i, j, k, i - 1, j, k, d, subcell) -
                                    XRef(s.A, s.L, X, i, j, k, i, j + 1, k, d, subcell) -
                                    XRef(s.A, s.L, X, i, j, k, i, j - 1, k, d, subcell) -
                                    XRef(s.A, s.L, X, i, j, k, i, j, k + 1, d, subcell) -
                                    XRef(s.A, s.L, X, i, j, k, i, j, k - 1, d, subcell)) /
                                   h;
                    target.set(i, j, k, result);
                } else {
                    target.set(i, j, k, 0.0f);
                }
            }
}

// Op (solver.inl:157-177): target = X + alpha*Y on FLUID cells, 0 elsewhere.  The reference
// runs one parallel_for over i per (j,k) line.
void Op(const Sim& s, const Grid<float>& X, const Grid<float>& Y, Grid<float>& target, float alpha) {
    const int x = s.n, y = s.n, z = s.n;
    auto cell = [&](int i, int j, int k) {
        if (s.A.get(i, j, k) == ARIEL_FLUID)
            target.set(i, j, k, X.get(i, j, k) + alpha * Y.get(i, j, k));
        else
            target.set(i, j, k, 0.0f);
    };
    if (s.faithful) {
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k) {
#pragma omp parallel for schedule(static)
                for (int i = 0; i < x; ++i) cell(i, j, k);
            }
    } else {
#pragma omp parallel for schedule(static)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k)
                for (int i = 0; i < x; ++i) cell(i, j, k);
    }
}

// Product (solver.inl:180-193): serial float accumulation in i,j,k order.
float Product(const Sim& s, const Grid<float>& X, const Grid<float>& Y) {
    float result = 0.0f;
    for (int i = 0; i < s.n; i++)
        for (int j = 0; j < s.n; j++)
            for (int k = 0; k < s.n; k++)
                if (s.A.get(i, j, k) == ARIEL_FLUID) result += X.get(i, j, k) * Y.get(i, j, k);
    return result;
}

// ApplyPreconditioner (solver.inl:232-286).  The neighbour terms need a FLUID cell whose
// preconditioner value is exactly 1.0f; when none exists the sweeps are elementwise, otherwise
// they run in serial order.
void ApplyPreconditioner(const Sim& s, Grid<float>& Z, const Grid<float>& R, const Grid<float>& P, bool ordered) {
    const Dims d{s.n, s.n, s.n};
    const int x = d.x, y = d.y, z = d.z;
    Grid<float> Q;
    Q.make(x, y, z, 0.0f);
    if (!ordered) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < x; ++i)
            for (int j = 0; j < y; ++j)
                for (int k = 0; k < z; ++k)
                    if (s.A.get(i, j, k) == ARIEL_FLUID) {
                        float t = R.get(i, j, k) - 0.0f - 0.0f - 0.0f;
                        Q.set(i, j, k, t * P.get(i, j, k));
                    }
        auto bcell = [&](int i, int j, int k) {
            if (s.A.get(i, j, k) == ARIEL_FLUID) {
                float t = Q.get(i, j, k) - 0.0f - 0.0f - 0.0f;
                Z.set(i, j, k, t * P.get(i, j, k));
            }
        };
        if (s.faithful) {
            for (int j = y - 1; j >= 0; j--)
                for (int k = z - 1; k >= 0; k--) {
#pragma omp parallel for schedule(static)
                    for (int i = x - 1; i >= 0; i--) bcell(i, j, k);
                }
        } else {
#pragma omp parallel for schedule(static)
            for (int j = y - 1; j >= 0; j--)
                for (int k = z - 1; k >= 0; k--)
                    for (int i = x - 1; i >= 0; i--) bcell(i, j, k);
        }
        return;
    }
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k)
                if (s.A.get(i, j, k) == ARIEL_FLUID) {
                    float left = ARef(s.A, i - 1, j, k, i, j, k, d) * PRef(P, i - 1, j, k, d) * PRef(Q, i - 1, j, k, d);
                    float bottom = ARef(s.A, i, j - 1, k, i, j, k, d) * PRef(P, i, j - 1, k, d) * PRef(Q, i, j - 1, k, d);
                    float back = ARef(s.A, i, j, k - 1, i, j, k, d) * PRef(P, i, j, k - 1, d) * PRef(Q, i, j, k - 1, d);
                    float t = R.get(i, j, k) - left - bottom - back;
                    Q.set(i, j, k, t * P.get(i, j, k));
                }
    for (int j = y - 1; j >= 0; j--)
        for (int k = z - 1; k >= 0; k--)
            for (int i = x - 1; i >= 0; i--)
                if (s.A.get(i, j, k) == ARIEL_FLUID) {
                    float right = ARef(s.A, i, j, k, i + 1, j, k, d) * PRef(P, i, j, k, d) * PRef(Z, i + 1, j, k, d);
                    float top = ARef(s.A, i, j, k, i, j + 1, k, d) * PRef(P, i, j, k, d) * PRef(Z, i, j + 1, k, d);
                    float front = ARef(s.A, i, j, k, i, j, k + 1, d) * PRef(P, i, j, k, d) * PRef(Z, i, j, k + 1, d);
                    float t = Q.get(i, j, k) - right - top - front;
                    Z.set(i, j, k, t * P.get(i, j, k));
                }
}

bool AnyFluidOne(const Sim& s, const Grid<float>& pc) {
    long ones = 0;
#pragma omp parallel for reduction(+ : ones) schedule(static)
    for (int i = 0; i < s.n; ++i)
        for (int j = 0; j < s.n; ++j)
            for (int k = 0; k < s.n; ++k)
                if (s.A.get(i, j, k) == ARIEL_FLUID && pc.get(i, j, k) == 1.0f) ones++;
    return ones != 0;
}

double FluidNorm2(const Sim& s, const Grid<float>& X) {
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (int i = 0; i < s.n; ++i)
        for (int j = 0; j < s.n; ++j)
            for (int k = 0; k < s.n; ++k)
                if (s.A.get(i, j, k) == ARIEL_FLUID) acc += (double)X.get(i, j, k) * (double)X.get(i, j, k);
    return acc;
}

// SolveConjugateGradient (solver.inl:289-354) in fp32, the reference's precision.  The
// per-iteration progress print (:336-337) is omitted.
void SolveConjugateGradient32(Sim& s, Grid<float>& PC, bool ordered) {
    const int x = s.n, y = s.n, z = s.n;
    const int subcell = s.prm.subcell;
    Grid<float> R, Z, S;
    R.make(x, y, z, 0.0f);
    Z.make(x, y, z, 0.0f);
    S.make(x, y, z, 0.0f);
    ComputeAx(s, s.P, Z, subcell);
    Op(s, s.D, Z, R, -1.0f);
    float error0 = Product(s, R, R);
    ApplyPreconditioner(s, Z, R, PC, ordered);
    if (s.faithful) {
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k) {
#pragma omp parallel for schedule(static)
                for (int i = 0; i < x; ++i) S.set(i, j, k, Z.get(i, j, k));
            }
    } else {
        S.v = Z.v;
    }
    float eps = 1.0e-2f * (x * y * z);
    double bnorm = std::sqrt(FluidNorm2(s, s.D));
    if (s.prm.stop_rule == ARIEL_STOP_REL) {
        double lim = s.prm.tol * bnorm;
        eps = (float)(lim * lim);
    }
    float a = Product(s, Z, R);
    long maxit = s.prm.max_iters > 0 ? s.prm.max_iters : (long)x * y * z;
    int it = 0;
    float error1 = error0;
    bool conv = false;
    if (s.prm.stop_rule == ARIEL_STOP_REL && error0 <= eps) {
        // relative rule: an already-converged warm start needs no iteration; non-FLUID
        // pressure is still zeroed as the reference's first Op would do (solver.inl:329)
        conv = true;
        Op(s, s.P, S, s.P, 0.0f);
    } else {
        for (long kk = 0; kk < maxit; kk++) {
            ComputeAx(s, S, Z, subcell);
            float alpha = a / Product(s, Z, S);
            Op(s, s.P, S, s.P, alpha);
            Op(s, R, Z, R, -alpha);
            error1 = Product(s, R, R);
            error0 = gmax(error0, error1);
            it = (int)kk + 1;
            if (error1 <= eps) {
                conv = true;
                break;
            }
            ApplyPreconditioner(s, Z, R, PC, ordered);
            float a2 = Product(s, Z, R);
            float beta = a2 / a;
            Op(s, Z, S, S, beta);
            a = a2;
        }
    }
    s.st.pcg_iterations = it;
    s.st.pcg_outer = 1;
    s.st.pcg_rr = error1;
    s.st.pcg_rel_residual = bnorm > 0 ? std::sqrt((double)error1) / bnorm : 0.0;
    s.st.pcg_converged = conv;
}

// ---------------------------------------------------------------------------------------------
// FP64 pressure solve on the same ghost-fluid operator (the oracle of the FP64 / MIXED paths).
// Operator: for a FLUID cell c, (A x)_c = (diag_c x_c - sum_{FLUID q} x_q) / h with
// diag_c = 6 - #(SOLID or outside) - sum_{AIR q} L_q / min(1e-6, L_c) and h = 1/(n*n) in float
// (solver.inl:81-101, 138-154, 196-230).
// ---------------------------------------------------------------------------------------------
struct Op64 {
    int n;
    const int* A;
    const float* L;
    std::vector<double> diag;
    std::vector<uint8_t> mask;  // bit m: neighbour m (order -x,+x,-y,+y,-z,+z) is FLUID
    double scale;
    std::vector<long> fluid;
};

inline long cid(int n, int i, int j, int k) { return ((long)i * n + j) * n + k; }

void BuildOp64(Op64& op, int n, const int* A, const float* L, int subcell) {
    op.n = n;
    op.A = A;
    op.L = L;
    long nc = (long)n * n * n;
    op.diag.assign(nc, 0.0);
    op.mask.assign(nc, 0);
    float nn = (float)n;
    float h = 1.0f / (nn * nn);
    op.scale = 1.0 / (double)h;
    op.fluid.clear();
    for (long c = 0; c < nc; ++c)
        if (A[c] == ARIEL_FLUID) op.fluid.push_back(c);
    long nf = (long)op.fluid.size();
#pragma omp parallel for schedule(static)
    for (long t = 0; t < nf; ++t) {
        long c = op.fluid[t];
        int i = (int)(c / ((long)n * n)), j = (int)((c / n) % n), k = (int)(c % n);
        const int q[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
        double dg = 6.0;
        uint8_t m = 0;
        for (int d = 0; d < 6; ++d) {
            int qi = q[d][0], qj = q[d][1], qk = q[d][2];
            if (qi < 0 || qi > n - 1 || qj < 0 || qj > n - 1 || qk < 0 || qk > n - 1) {
                dg -= 1.0;
                continue;
            }
            int tq = A[cid(n, qi, qj, qk)];
            if (tq == ARIEL_SOLID)
                dg -= 1.0;
            else if (tq == ARIEL_FLUID)
                m |= (uint8_t)(1u << d);
            else if (subcell)
                dg -= (double)L[cid(n, qi, qj, qk)] / (double)gmin(1.0e-6f, L[c]);
        }
        op.diag[c] = dg;
        op.mask[c] = m;
    }
}

void Apply64(const Op64& op, const double* x, double* y) {
    const int n = op.n;
    const long offs[6] = {-(long)n * n, (long)n * n, -(long)n, (long)n, -1, 1};
    long nf = (long)op.fluid.size();
#pragma omp parallel for schedule(static)
    for (long t = 0; t < nf; ++t) {
        long c = op.fluid[t];
        double acc = op.diag[c] * x[c];
        uint8_t m = op.mask[c];
        for (int d = 0; d < 6; ++d)
            if (m & (1u << d)) acc -= x[c + offs[d]];
        y[c] = acc * op.scale;
    }
}

double Dot64(const Op64& op, const double* a, const double* b) {
    long nf = (long)op.fluid.size();
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (long t = 0; t < nf; ++t) acc += a[op.fluid[t]] * b[op.fluid[t]];
    return acc;
}

// FP64 preconditioner: the reference's construction evaluated in fp64 (diagonal unless a
// FLUID value is exactly 1.0), or MIC(0) (Bridson) when asked.  Returns per-cell values.
struct Pre64 {
    std::vector<double> pc;
    bool mic = false;
    bool ordered = false;
};

inline bool fluidAt(const Op64& op, int i, int j, int k) {
    int n = op.n;
    if (i < 0 || j < 0 || k < 0 || i >= n || j >= n || k >= n) return false;
    return op.A[cid(n, i, j, k)] == ARIEL_FLUID;
}

void BuildPre64(Pre64& pre, const Op64& op, int kind, double tau, double sigma) {
    const int n = op.n;
    long nc = (long)n * n * n;
    pre.pc.assign(nc, 0.0);
    pre.mic = (kind == ARIEL_PRECOND_MIC0);
    pre.ordered = false;
    if (!pre.mic) {
        bool any_one = false;
        for (long c : op.fluid) {
            double dg = op.diag[c];
            if (dg > 0) {
                pre.pc[c] = 1.0 / std::sqrt(dg);
                if (pre.pc[c] == 1.0) any_one = true;
            }
        }
        if (!any_one) return;
        pre.ordered = true;
        std::fill(pre.pc.begin(), pre.pc.end(), 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    long c = cid(n, i, j, k);
                    if (op.A[c] != ARIEL_FLUID) continue;
                    double left = (fluidAt(op, i - 1, j, k) && pre.pc[cid(n, i - 1, j, k)] == 1.0) ? -1.0 : 0.0;
                    double bottom = (fluidAt(op, i, j - 1, k) && pre.pc[cid(n, i, j - 1, k)] == 1.0) ? -1.0 : 0.0;
                    double back = (fluidAt(op, i, j, k - 1) && pre.pc[cid(n, i, j, k - 1)] == 1.0) ? -1.0 : 0.0;
                    double dg = op.diag[c];
                    double e = dg - left * left - bottom * bottom - back * back;
                    if (dg > 0) {
                        if (e < 0.25 * dg) e = dg;
                        pre.pc[c] = 1.0 / std::sqrt(e);
                    }
                }
        return;
    }
    // MIC(0): e = Adiag - sum (Aplus_q * pc_q)^2 - tau * sum Aplus_q (other two Aplus of q) pc_q^2
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                long c = cid(n, i, j, k);
                if (op.A[c] != ARIEL_FLUID) continue;
                double e = op.diag[c];
                if (fluidAt(op, i - 1, j, k)) {
                    double p = pre.pc[cid(n, i - 1, j, k)];
                    double ap = -1.0;
                    double oth = (fluidAt(op, i - 1, j + 1, k) ? -1.0 : 0.0) + (fluidAt(op, i - 1, j, k + 1) ? -1.0 : 0.0);
                    e -= (ap * p) * (ap * p) + tau * (ap * oth * p * p);
                }
                if (fluidAt(op, i, j - 1, k)) {
                    double p = pre.pc[cid(n, i, j - 1, k)];
                    double ap = -1.0;
                    double oth = (fluidAt(op, i + 1, j - 1, k) ? -1.0 : 0.0) + (fluidAt(op, i, j - 1, k + 1) ? -1.0 : 0.0);
                    e -= (ap * p) * (ap * p) + tau * (ap * oth * p * p);
                }
                if (fluidAt(op, i, j, k - 1)) {
                    double p = pre.pc[cid(n, i, j, k - 1)];
                    double ap = -1.0;
                    double oth = (fluidAt(op, i + 1, j, k - 1) ? -1.0 : 0.0) + (fluidAt(op, i, j + 1, k - 1) ? -1.0 : 0.0);
                    e -= (ap * p) * (ap * p) + tau * (ap * oth * p * p);
                }
                if (e < sigma * op.diag[c]) e = op.diag[c];
                pre.pc[c] = e > 0 ? 1.0 / std::sqrt(e) : 0.0;
            }
}

void ApplyPre64(const Pre64& pre, const Op64& op, const double* r, double* z, std::vector<double>& q) {
    const int n = op.n;
    if (!pre.mic && !pre.ordered) {
        long nf = (long)op.fluid.size();
#pragma omp parallel for schedule(static)
        for (long t = 0; t < nf; ++t) {
            long c = op.fluid[t];
            z[c] = (r[c] * pre.pc[c]) * pre.pc[c];
        }
        return;
    }
    long nc = (long)n * n * n;
    q.assign(nc, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                long c = cid(n, i, j, k);
                if (op.A[c] != ARIEL_FLUID) continue;
                double t = r[c];
                const int lo[3][3] = {{i - 1, j, k}, {i, j - 1, k}, {i, j, k - 1}};
                for (int m = 0; m < 3; ++m) {
                    if (!fluidAt(op, lo[m][0], lo[m][1], lo[m][2])) continue;
                    long qc = cid(n, lo[m][0], lo[m][1], lo[m][2]);
                    if (pre.mic)
                        t -= -1.0 * pre.pc[qc] * q[qc];
                    else if (pre.pc[qc] == 1.0 && q[qc] == 1.0)
                        t -= -1.0;
                }
                q[c] = t * pre.pc[c];
            }
    for (int i = n - 1; i >= 0; --i)
        for (int j = n - 1; j >= 0; --j)
            for (int k = n - 1; k >= 0; --k) {
                long c = cid(n, i, j, k);
                if (op.A[c] != ARIEL_FLUID) continue;
                double t = q[c];
                const int hi[3][3] = {{i + 1, j, k}, {i, j + 1, k}, {i, j, k + 1}};
                for (int m = 0; m < 3; ++m) {
                    if (!fluidAt(op, hi[m][0], hi[m][1], hi[m][2])) continue;
                    long qc = cid(n, hi[m][0], hi[m][1], hi[m][2]);
                    if (pre.mic)
                        t -= -1.0 * pre.pc[c] * z[qc];
                    else if (pre.pc[c] == 1.0 && z[qc] == 1.0)
                        t -= -1.0;
                }
                z[c] = t * pre.pc[c];
            }
}

struct Solve64Result {
    int iterations;
    double rel;
    double rr;
    bool converged;
};

// Preconditioned CG in fp64; stop on the recursive residual, report the true one.
Solve64Result PCG64(const Op64& op, const Pre64& pre, const double* b, double* x, int stop_rule, double tol,
                    long maxit) {
    const int n = op.n;
    long nc = (long)n * n * n;
    std::vector<double> r(nc, 0.0), z(nc, 0.0), s(nc, 0.0), q(nc, 0.0), tmp;
    Apply64(op, x, q.data());
    for (long c : op.fluid) r[c] = b[c] - q[c];
    // non-fluid entries of x are zero after a solve (reference Op writes 0 there)
    for (long c = 0; c < nc; ++c)
        if (op.A[c] != ARIEL_FLUID) x[c] = 0.0;
    double bb = Dot64(op, b, b);
    double rr = Dot64(op, r.data(), r.data());
    double lim2 = stop_rule == ARIEL_STOP_REL ? tol * tol * bb : 1.0e-2 * (double)n * n * n;
    Solve64Result res{0, 0.0, rr, false};
    if (!(rr > lim2) && stop_rule == ARIEL_STOP_REL) {
        res.converged = true;
    } else {
        ApplyPre64(pre, op, r.data(), z.data(), tmp);
        for (long c : op.fluid) s[c] = z[c];
        double rho = Dot64(op, z.data(), r.data());
        for (long it = 0; it < maxit; ++it) {
            Apply64(op, s.data(), q.data());
            double sq = Dot64(op, s.data(), q.data());
            double alpha = sq != 0.0 ? rho / sq : 0.0;
            for (long c : op.fluid) {
                x[c] += alpha * s[c];
                r[c] -= alpha * q[c];
            }
            rr = Dot64(op, r.data(), r.data());
            res.iterations = (int)it + 1;
            if (rr <= lim2) {
                res.converged = true;
                break;
            }
            ApplyPre64(pre, op, r.data(), z.data(), tmp);
            double rho2 = Dot64(op, z.data(), r.data());
            double beta = rho != 0.0 ? rho2 / rho : 0.0;
            for (long c : op.fluid) s[c] = z[c] + beta * s[c];
            rho = rho2;
        }
    }
    Apply64(op, x, q.data());
    double tr = 0.0;
    for (long c : op.fluid) {
        double d = b[c] - q[c];
        tr += d * d;
    }
    res.rr = rr;
    res.rel = bb > 0 ? std::sqrt(tr / bb) : 0.0;
    return res;
}

// Solve (solver.inl:356-379)
void Solve(Sim& s) {
    const int n = s.n;
    if (s.prm.precision == ARIEL_PREC_REF32 && s.prm.precond == ARIEL_PRECOND_REF) {
        Grid<float> pc;
        pc.make(n, n, n, 0.0f);
        bool ordered = BuildPreconditioner(pc, s, s.prm.subcell);
        ordered = ordered || AnyFluidOne(s, pc);
        s.st.precond_exact_path = ordered;
        SolveConjugateGradient32(s, pc, ordered);
        long nf = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) nf += s.A.get(i, j, k) == ARIEL_FLUID;
        s.st.n_fluid_cells = nf;
        return;
    }
    // FP64 (also the oracle of MIXED): warm start from the fp64 pressure.
    long nc = (long)n * n * n;
    std::vector<int> A(nc);
    std::vector<float> L(nc);
    std::vector<double> b(nc);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                long c = cid(n, i, j, k);
                A[c] = s.A.get(i, j, k);
                L[c] = s.L.get(i, j, k);
                b[c] = (double)s.D.get(i, j, k);
            }
    Op64 op;
    BuildOp64(op, n, A.data(), L.data(), s.prm.subcell);
    Pre64 pre;
    BuildPre64(pre, op, s.prm.precond, s.prm.mic_tau, s.prm.mic_sigma);
    long maxit = s.prm.max_iters > 0 ? s.prm.max_iters : nc;
    Solve64Result r = PCG64(op, pre, b.data(), s.P64.data(), s.prm.stop_rule, s.prm.tol, maxit);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) s.P.set(i, j, k, (float)s.P64[cid(n, i, j, k)]);
    s.st.pcg_iterations = r.iterations;
    s.st.pcg_outer = 1;
    s.st.pcg_rr = r.rr;
    s.st.pcg_rel_residual = r.rel;
    s.st.pcg_converged = r.converged;
    s.st.precond_exact_path = pre.ordered;
    s.st.n_fluid_cells = (long)op.fluid.size();
}

// FlipSim::SubtractPressureGradient (flip.cpp:568-680)
void SubtractPressureGradient(Sim& s) {
    const int x = s.n, y = s.n, z = s.n;
    const float h = 1.0f / s.maxd;
    const int subcell = s.prm.subcell;
    const Grid<float>& P = s.P;
    const Grid<float>& L = s.L;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x + 1; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k)
                if (i > 0 && i < x) {
                    float pf = P.get(i, j, k), pb = P.get(i - 1, j, k);
                    if (subcell && L.get(i, j, k) * L.get(i - 1, j, k) < 0.0f) {
                        pf = L.get(i, j, k) < 0.0f ? P.get(i, j, k)
                                                   : L.get(i, j, k) / gmin(1.0e-3f, L.get(i - 1, j, k)) * P.get(i - 1, j, k);
                        pb = L.get(i - 1, j, k) < 0.0f ? P.get(i - 1, j, k)
                                                       : L.get(i - 1, j, k) / gmin(1.0e-6f, L.get(i, j, k)) * P.get(i, j, k);
                    }
                    float v = s.ux.get(i, j, k);
                    v -= (pf - pb) / h;
                    s.ux.set(i, j, k, v);
                }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y + 1; ++j)
            for (int k = 0; k < z; ++k)
                if (j > 0 && j < y) {
                    float pf = P.get(i, j, k), pb = P.get(i, j - 1, k);
                    if (subcell && L.get(i, j, k) * L.get(i, j - 1, k) < 0.0f) {
                        pf = L.get(i, j, k) < 0.0f ? P.get(i, j, k)
                                                   : L.get(i, j, k) / gmin(1.0e-3f, L.get(i, j - 1, k)) * P.get(i, j - 1, k);
                        pb = L.get(i, j - 1, k) < 0.0f ? P.get(i, j - 1, k)
                                                       : L.get(i, j - 1, k) / gmin(1.0e-6f, L.get(i, j, k)) * P.get(i, j, k);
                    }
                    float v = s.uy.get(i, j, k);
                    v -= (pf - pb) / h;
                    s.uy.set(i, j, k, v);
                }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z + 1; ++k)
                if (k > 0 && k < z) {
                    float pf = P.get(i, j, k), pb = P.get(i, j, k - 1);
                    if (subcell && L.get(i, j, k) * L.get(i, j, k - 1) < 0.0f) {
                        pf = L.get(i, j, k) < 0.0f ? P.get(i, j, k)
                                                   : L.get(i, j, k) / gmin(1.0e-3f, L.get(i, j, k - 1)) * P.get(i, j, k - 1);
                        pb = L.get(i, j, k - 1) < 0.0f ? P.get(i, j, k - 1)
                                                       : L.get(i, j, k - 1) / gmin(1.0e-6f, L.get(i, j, k)) * P.get(i, j, k);
                    }
                    float v = s.uz.get(i, j, k);
                    v -= (pf - pb) / h;
                    s.uz.set(i, j, k, v);
                }
}

// FlipSim::ExtrapolateVelocity (flip.cpp:452-566)
void ExtrapolateVelocity(Sim& s) {
    const int x = s.n, y = s.n, z = s.n;
    Grid<int> mark[3], wall[3];
    for (int d = 0; d < 3; ++d) {
        mark[d].make(x, y, z, 0);
        wall[d].make(x, y, z, 0);
    }
    const Grid<int>& A = s.A;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x + 1; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z; ++k) {
                mark[0].set(i, j, k, (i > 0 && A.get(i - 1, j, k) == ARIEL_FLUID) || (i < x && A.get(i, j, k) == ARIEL_FLUID));
                wall[0].set(i, j, k, (i <= 0 || A.get(i - 1, j, k) == ARIEL_SOLID) && (i >= x || A.get(i, j, k) == ARIEL_SOLID));
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y + 1; ++j)
            for (int k = 0; k < z; ++k) {
                mark[1].set(i, j, k, (j > 0 && A.get(i, j - 1, k) == ARIEL_FLUID) || (j < y && A.get(i, j, k) == ARIEL_FLUID));
                wall[1].set(i, j, k, (j <= 0 || A.get(i, j - 1, k) == ARIEL_SOLID) && (j >= y || A.get(i, j, k) == ARIEL_SOLID));
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x; ++i)
        for (int j = 0; j < y; ++j)
            for (int k = 0; k < z + 1; ++k) {
                mark[2].set(i, j, k, (k > 0 && A.get(i, j, k - 1) == ARIEL_FLUID) || (k < z && A.get(i, j, k) == ARIEL_FLUID));
                wall[2].set(i, j, k, (k <= 0 || A.get(i, j, k - 1) == ARIEL_SOLID) && (k >= z || A.get(i, j, k) == ARIEL_SOLID));
            }
    Grid<float>* U[3] = {&s.ux, &s.uy, &s.uz};
#pragma omp parallel for schedule(static)
    for (int i = 0; i < x + 1; ++i)
        for (int j = 0; j < y + 1; ++j)
            for (int k = 0; k < z + 1; ++k)
                for (int n = 0; n < 3; ++n) {
                    if (n != 0 && i > x - 1) continue;
                    if (n != 1 && j > y - 1) continue;
                    if (n != 2 && k > z - 1) continue;
                    if (!mark[n].get(i, j, k) && wall[n].get(i, j, k)) {
                        unsigned wsum = 0;
                        float sum = 0.0f;
                        const int q[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
                        for (int qk = 0; qk < 6; ++qk) {
                            int a = q[qk][0], b = q[qk][1], c = q[qk][2];
                            if (a >= 0 && a < x + (n == 0) && b >= 0 && b < y + (n == 1) && c >= 0 && c < z + (n == 2)) {
                                if (mark[n].get(a, b, c)) {
                                    wsum++;
                                    sum += U[n]->get(a, b, c);
                                }
                            }
                        }
                        if (wsum) U[n]->set(i, j, k, sum / wsum);
                    }
                }
}

// FlipSim::SubtractPreviousGrid (flip.cpp:365-410)
void SubtractPreviousGrid(Sim& s) {
    for (size_t c = 0; c < s.ux.v.size(); ++c) s.pux.v[c] = s.ux.v[c] - s.pux.v[c];
    for (size_t c = 0; c < s.uy.v.size(); ++c) s.puy.v[c] = s.uy.v[c] - s.puy.v[c];
    for (size_t c = 0; c < s.uz.v.size(); ++c) s.puz.v[c] = s.uz.v[c] - s.puz.v[c];
}

// Interpolate (particlegridoperations.inl:106-118)
inline float Interpolate(const Grid<float>& q, vec3 p, vec3 n) {
    float x = gmax(0.0f, gmin(n.x, p.x));
    float y = gmax(0.0f, gmin(n.y, p.y));
    float z = gmax(0.0f, gmin(n.z, p.z));
    int i = (int)gmin(x, n.x - 2);
    int j = (int)gmin(y, n.y - 2);
    int k = (int)gmin(z, n.z - 2);
    float term1 = ((i + 1 - x) * q.get(i, j, k) + (x - i) * q.get(i + 1, j, k)) * (j + 1 - y);
    float term2 = ((i + 1 - x) * q.get(i, j + 1, k) + (x - i) * q.get(i + 1, j + 1, k)) * (y - j);
    float term3 = ((i + 1 - x) * q.get(i, j, k + 1) + (x - i) * q.get(i + 1, j, k + 1)) * (j + 1 - y);
    float term4 = ((i + 1 - x) * q.get(i, j + 1, k + 1) + (x - i) * q.get(i + 1, j + 1, k + 1)) * (y - j);
    return (k + 1 - z) * (term1 + term2) + (z - k) * (term3 + term4);
}

// InterpolateVelocity (particlegridoperations.inl:120-133)
inline vec3 InterpolateVelocity(vec3 p, const Grid<float>& gx, const Grid<float>& gy, const Grid<float>& gz, int n) {
    int x = n, y = n, z = n;
    float maxd = gmax(gmax((float)x, (float)y), (float)z);
    x = (int)maxd;
    y = (int)maxd;
    z = (int)maxd;
    vec3 u;
    u.x = Interpolate(gx, mk(x * p.x, y * p.y - 0.5f, z * p.z - 0.5f), mk((float)(x + 1), (float)y, (float)z));
    u.y = Interpolate(gy, mk(x * p.x - 0.5f, y * p.y, z * p.z - 0.5f), mk((float)x, (float)(y + 1), (float)z));
    u.z = Interpolate(gz, mk(x * p.x - 0.5f, y * p.y - 0.5f, z * p.z), mk((float)x, (float)y, (float)(z + 1)));
    return u;
}

// FlipSim::CheckParticleSolidConstraints (flip.cpp:183-227) with analytic solids.
void CheckParticleSolidConstraints(Sim& s) {
    if (!HasSolids(s)) return;
    const float maxd = s.maxd;
    const long np = (long)s.parts.size();
#pragma omp parallel for schedule(static)
    for (long p = 0; p < np; ++p) {
        Particle& P = s.parts[p];
        if (P.type != ARIEL_FLUID) continue;
        vec3 origin = P.pt * maxd;
        vec3 dir = gnormalize(P.p - P.pt);
        float raynulltest = glength(dir);
        if (raynulltest == raynulltest) {
            Hit hit = IntersectSolids(s, origin, dir);
            float u_dir = glength(P.ut);
            if (hit.hit) {
                float solidDistance = glength(origin - hit.point);
                float velocityDistance = glength(P.p - P.pt) * maxd;
                if (solidDistance < velocityDistance) {
                    P.p = (origin + dir * .90f * solidDistance) / maxd;
                    P.u = 2.0f * gdot(dir, hit.normal) * hit.normal - gnormalize(dir);
                    P.u = gnormalize(P.u) * u_dir;
                }
            }
            vec3 o2 = P.p * maxd;
            if (InsideSolid(s, o2)) {
                P.u = -gnormalize(dir) * u_dir;
                P.p = P.pt + P.u * s.desc.stepsize;
            }
        }
    }
}

// FlipSim::AdjustParticlesStuckInSolids (flip.cpp:130-181) with analytic solids.
void AdjustParticlesStuckInSolids(Sim& s) {
    if (!HasSolids(s)) return;
    const float maxd = s.maxd;
    const long np = (long)s.parts.size();
    for (long p = 0; p < np; ++p) {
        Particle& P = s.parts[p];
        if (P.type != ARIEL_FLUID) continue;
        vec3 point = P.p * maxd;
        if (!InsideSolid(s, point)) continue;
        P.pt = P.p;
        P.p = ClosestSolidSurface(s, point) / maxd;
        vec3 origin = P.pt * maxd;
        vec3 dir = gnormalize(P.p - P.pt);
        float d = glength(P.p - P.pt);
        float raynulltest = glength(dir);
        if (raynulltest == raynulltest) {
            Hit hit = IntersectSolids(s, origin, dir);
            float nearest = glength(origin - hit.point);
            P.p = (origin + dir * 1.05f * nearest) / maxd;
            P.u = gnormalize(dir) * d;
        }
    }
}

// FlipSim::SolvePicFlip (flip.cpp:287-322) and AdvectParticles (flip.cpp:229-285)
void SolvePicFlipAndAdvect(Sim& s) {
    const long np = (long)s.parts.size();
    const int n = s.n;
    const float r = 1.0f / s.maxd;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < np; ++i) {
        Particle& P = s.parts[i];
        P.t = P.u;
        vec3 du = InterpolateVelocity(P.p, s.pux, s.puy, s.puz, n);
        P.t = du + P.t;
        vec3 pic = InterpolateVelocity(P.p, s.ux, s.uy, s.uz, n);
        P.u = (1.0f - s.prm.picflip) * pic + s.prm.picflip * P.t;
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < np; ++i) {
        Particle& P = s.parts[i];
        if (P.type == ARIEL_FLUID) {
            vec3 velocity = InterpolateVelocity(P.p, s.ux, s.uy, s.uz, n);
            P.p = P.p + s.desc.stepsize * velocity;
        }
    }
    Sort(s);
    const unsigned x = (unsigned)n, y = (unsigned)n, z = (unsigned)n;
    const float maxd = s.maxd;
#pragma omp parallel for schedule(static)
    for (long p0 = 0; p0 < np; ++p0) {
        Particle& P = s.parts[p0];
        if (P.type == ARIEL_FLUID) {
            P.p.x = gmax(r, gmin(1.0f - r, P.p.x));
            P.p.y = gmax(r, gmin(1.0f - r, P.p.y));
            P.p.z = gmax(r, gmin(1.0f - r, P.p.z));
        }
        // The reference queries the 27 neighbour cells of every FLUID particle even when no
        // SOLID particle exists; the faithful (timed) mode keeps that cost.
        if (P.type == ARIEL_FLUID && (s.faithful || HasSolids(s))) {
            unsigned i = (unsigned)gmin(x - 1.0f, P.p.x * maxd);
            unsigned j = (unsigned)gmin(y - 1.0f, P.p.y * maxd);
            unsigned k = (unsigned)gmin(z - 1.0f, P.p.z * maxd);
            std::vector<int> nb = GetCellNeighbors(s, mk((float)i, (float)j, (float)k), mk(1, 1, 1));
            for (int q : nb) {
                const Particle& np_ = s.parts[q];
                float re = 1.5f * s.desc.density / maxd;
                if (np_.type == ARIEL_SOLID) {
                    float dist = glength(P.p - np_.p);
                    if (dist < re) {
                        vec3 normal = np_.n;
                        if (glength(normal) < 0.0000001f && dist) normal = gnormalize(P.p - np_.p);
                        P.p = P.p + (re - dist) * normal;
                        P.u = P.u - gdot(P.u, normal) * normal;
                    }
                }
            }
        }
    }
    CheckParticleSolidConstraints(s);
}

// ResampleParticles / Resample (particleresampler.inl:35-148)
vec3 Resample(const Sim& s, vec3 p, vec3 u, float re) {
    const float maxd = s.maxd;
    float wsum = 0.0f;
    vec3 ru = mk(0, 0, 0);
    float x = gmax(0.0f, gmin((float)maxd - 1, maxd * p.x));
    float y = gmax(0.0f, gmin((float)maxd - 1, maxd * p.y));
    float z = gmax(0.0f, gmin((float)maxd - 1, maxd * p.z));
    std::vector<int> nb = GetCellNeighbors(s, mk(x, y, z), mk(1, 1, 1));
    for (int m : nb) {
        const Particle& np_ = s.parts[m];
        if (np_.type == ARIEL_FLUID) {
            float dist2 = Sqrlength(p, np_.p);
            float w = np_.mass * Sharpen(dist2, re);
            ru = ru + w * np_.u;
            wsum += w;
        }
    }
    if (wsum)
        ru = ru / wsum;
    else
        ru = u;
    return ru;
}

void ResampleParticles(Sim& s) {
    StoreTemp(s);
    const float maxd = s.maxd;
    const float dt = s.desc.stepsize;
    const float re = s.desc.density / maxd;
    Sort(s);
    const float springforce = 50.0f;
    const long np = (long)s.parts.size();
    const uint32_t k0 = (uint32_t)s.prm.rng_seed, k1 = (uint32_t)(s.prm.rng_seed >> 32);
    const uint32_t frame = (uint32_t)s.frame;
#pragma omp parallel for schedule(static)
    for (long n0 = 0; n0 < np; ++n0) {
        if (s.parts[n0].type != ARIEL_FLUID) continue;
        Particle& p = s.parts[n0];
        vec3 spring = mk(0, 0, 0);
        float x = gmax(0.0f, gmin((float)maxd, maxd * p.p.x));
        float y = gmax(0.0f, gmin((float)maxd, maxd * p.p.y));
        float z = gmax(0.0f, gmin((float)maxd, maxd * p.p.z));
        std::vector<int> nb = GetCellNeighbors(s, mk(x, y, z), mk(1, 1, 1));
        uint32_t draws = 0;
        for (int n1 : nb) {
            if (n1 == n0) continue;
            const Particle& np_ = s.parts[n1];
            float dist = glength(p.p - np_.p);
            float w = springforce * np_.mass * Smooth(dist * dist, re);
            if (dist > 0.1f * re) {
                spring.x += w * (p.p.x - np_.p.x) / dist * re;
                spring.y += w * (p.p.y - np_.p.y) / dist * re;
                spring.z += w * (p.p.z - np_.p.z) / dist * re;
            } else if (np_.type == ARIEL_FLUID) {
                u4 c{{(uint32_t)n0, frame, draws++, kTagResample}};
                u4 rv = philox(c, k0, k1);
                spring.x += 0.01f * re / dt * (float)(rv.v[0] % 101u) / 100.0f;
                spring.y += 0.01f * re / dt * (float)(rv.v[1] % 101u) / 100.0f;
                spring.z += 0.01f * re / dt * (float)(rv.v[2] % 101u) / 100.0f;
            } else {
                spring.x += 0.05f * re / dt * np_.n.x;
                spring.y += 0.05f * re / dt * np_.n.y;
                spring.z += 0.05f * re / dt * np_.n.z;
            }
        }
        p.t.x = p.p.x + dt * spring.x;
        p.t.y = p.p.y + dt * spring.y;
        p.t.z = p.p.z + dt * spring.z;
    }
#pragma omp parallel for schedule(static)
    for (long n = 0; n < np; ++n) {
        if (s.parts[n].type != ARIEL_FLUID) continue;
        Particle& p = s.parts[n];
        p.t2 = p.u;
        p.t2 = Resample(s, p.t, p.t2, re);
    }
#pragma omp parallel for schedule(static)
    for (long n = 0; n < np; ++n) {
        if (s.parts[n].type != ARIEL_FLUID) continue;
        Particle& p = s.parts[n];
        if (!InsideSolid(s, p.t * maxd)) {
            p.p = p.t;
            p.u = p.t2;
        }
    }
    CheckParticleSolidConstraints(s);
}

// ---------------------------------------------------------------------------------------------
// Scene seeding: Scene::GenerateParticles (src/scene/scene.cpp:257-360) for box liquids and
// sphere solids, in lexicographic (i,j,k) order, with optional Philox jitter inside each
// lattice sub-cell.
// ---------------------------------------------------------------------------------------------
void GenerateParticles(Sim& s) {
    const int n = s.n;
    const float maxdim = (float)n;
    const float thickness = 1.0f / maxdim;
    const float density = s.desc.density;
    const float w = density * thickness;
    const uint32_t k0 = (uint32_t)s.desc.seed, k1 = (uint32_t)(s.desc.seed >> 32);
    std::vector<Particle> liquid, solid;
    for (int l = 0; l < s.desc.n_liquid; ++l) {
        const AsimBox& bx = s.desc.liquid[l];
        float lminx = gmax(std::floor(bx.lo[0] * maxdim), 0.0f) / density;
        float lminy = gmax(std::floor(bx.lo[1] * maxdim), 0.0f) / density;
        float lminz = gmax(std::floor(bx.lo[2] * maxdim), 0.0f) / density;
        float lmaxx = gmin(std::ceil(bx.hi[0] * maxdim), maxdim + 1.0f) / density;
        float lmaxy = gmin(std::ceil(bx.hi[1] * maxdim), maxdim + 1.0f) / density;
        float lmaxz = gmin(std::ceil(bx.hi[2] * maxdim), maxdim + 1.0f) / density;
        for (unsigned i = (unsigned)lminx; i < (unsigned)lmaxx; ++i)
            for (unsigned j = (unsigned)lminy; (float)j < lmaxy; ++j)
                for (unsigned k = (unsigned)lminz; (float)k < lmaxz; ++k) {
                    vec3 c = mk((i * w) + (w / 2.0f), (j * w) + (w / 2.0f), (k * w) + (w / 2.0f));
                    vec3 wp = c * maxdim;
                    bool inside = wp.x > bx.lo[0] * maxdim && wp.x < bx.hi[0] * maxdim && wp.y > bx.lo[1] * maxdim &&
                                  wp.y < bx.hi[1] * maxdim && wp.z > bx.lo[2] * maxdim && wp.z < bx.hi[2] * maxdim;
                    if (!inside || InsideSolid(s, wp)) continue;
                    Particle p{};
                    p.p = c;
                    if (s.desc.jitter > 0.0f) {
                        uint32_t id = (uint32_t)liquid.size();
                        u4 rv = philox(u4{{id, (uint32_t)l, 0u, kTagSeed}}, k0, k1);
                        float ux = (float)(rv.v[0] >> 8) * (1.0f / 16777216.0f);
                        float uy = (float)(rv.v[1] >> 8) * (1.0f / 16777216.0f);
                        float uz = (float)(rv.v[2] >> 8) * (1.0f / 16777216.0f);
                        p.p = mk((i * w) + (ux * w), (j * w) + (uy * w), (k * w) + (uz * w));
                    }
                    p.u = mk(bx.vel[0], bx.vel[1], bx.vel[2]);
                    p.n = mk(0, 0, 0);
                    p.density = 10.0f;
                    p.type = ARIEL_FLUID;
                    p.mass = 1.0f;
                    liquid.push_back(p);
                }
    }
    for (const Sphere& sp : s.solids) {
        float lminx = gmax(std::floor(sp.c.x - sp.r), 0.0f) / density;
        float lminy = gmax(std::floor(sp.c.y - sp.r), 0.0f) / density;
        float lminz = gmax(std::floor(sp.c.z - sp.r), 0.0f) / density;
        float lmaxx = gmin(std::ceil(sp.c.x + sp.r), maxdim + 1.0f) / density;
        float lmaxy = gmin(std::ceil(sp.c.y + sp.r), maxdim + 1.0f) / density;
        float lmaxz = gmin(std::ceil(sp.c.z + sp.r), maxdim + 1.0f) / density;
        for (unsigned i = (unsigned)lminx; i < (unsigned)lmaxx; ++i)
            for (unsigned j = (unsigned)lminy; (float)j < lmaxy; ++j)
                for (unsigned k = (unsigned)lminz; (float)k < lmaxz; ++k) {
                    vec3 c = mk((i * w) + (w / 2.0f), (j * w) + (w / 2.0f), (k * w) + (w / 2.0f));
                    vec3 wp = c * maxdim;
                    vec3 d = wp - sp.c;
                    if (!(gdot(d, d) < sp.r * sp.r)) continue;
                    Particle p{};
                    p.p = c;
                    p.u = mk(0, 0, 0);
                    p.n = mk(0, 0, 0);
                    p.density = 10.0f;
                    p.type = ARIEL_SOLID;
                    p.mass = 10.0f;
                    solid.push_back(p);
                }
    }
    // solid meshes after the spheres, each over the lattice of its world bounding box
    for (size_t m = 0; m < s.mlo.size(); ++m) {
        vec3 lo = s.mlo[m], hi = s.mhi[m];
        float lminx = gmax(std::floor(lo.x), 0.0f) / density;
        float lminy = gmax(std::floor(lo.y), 0.0f) / density;
        float lminz = gmax(std::floor(lo.z), 0.0f) / density;
        float lmaxx = gmin(std::ceil(hi.x), maxdim + 1.0f) / density;
        float lmaxy = gmin(std::ceil(hi.y), maxdim + 1.0f) / density;
        float lmaxz = gmin(std::ceil(hi.z), maxdim + 1.0f) / density;
        for (unsigned i = (unsigned)lminx; i < (unsigned)lmaxx; ++i)
            for (unsigned j = (unsigned)lminy; (float)j < lmaxy; ++j)
                for (unsigned k = (unsigned)lminz; (float)k < lmaxz; ++k) {
                    vec3 c = mk((i * w) + (w / 2.0f), (j * w) + (w / 2.0f), (k * w) + (w / 2.0f));
                    if (!((MeshInsideBits(s, c * maxdim) >> m) & 1u)) continue;
                    Particle p{};
                    p.p = c;
                    p.u = mk(0, 0, 0);
                    p.n = mk(0, 0, 0);
                    p.density = 10.0f;
                    p.type = ARIEL_SOLID;
                    p.mass = 10.0f;
                    solid.push_back(p);
                }
    }
    s.parts = liquid;
    s.parts.insert(s.parts.end(), solid.begin(), solid.end());
}

void AllocGrids(Sim& s) {
    const int n = s.n;
    s.pmap.make(n, n, n, -1);
    s.cells.clear();
    s.ux.make(n + 1, n, n, 0.0f);
    s.uy.make(n, n + 1, n, 0.0f);
    s.uz.make(n, n, n + 1, 0.0f);
    s.pux.make(n + 1, n, n, 0.0f);
    s.puy.make(n, n + 1, n, 0.0f);
    s.puz.make(n, n, n + 1, 0.0f);
    s.D.make(n, n, n, 0.0f);
    s.P.make(n, n, n, 0.0f);
    s.A.make(n, n, n, 0);
    s.L.make(n, n, n, 1.6f);
    s.P64.assign((size_t)n * n * n, 0.0);
}

// FlipSim::Init's density normaliser (flip.cpp:42-70), leaving the particle set untouched.
void ComputeMaxDensity(Sim& s) {
    std::vector<Particle> keep;
    keep.swap(s.parts);
    const float maxd = s.maxd;
    const float h = s.desc.density / maxd;
    for (unsigned i = 0; i < 10; i++)
        for (unsigned j = 0; j < 10; j++)
            for (unsigned k = 0; k < 10; k++) {
                Particle p{};
                p.p = (mk((float)i, (float)j, (float)k) + mk(0.5f, 0.5f, 0.5f)) * h;
                p.type = ARIEL_FLUID;
                p.mass = 1.0f;
                s.parts.push_back(p);
            }
    Sort(s);
    s.max_density = 1.0f;
    ComputeDensity(s);
    s.max_density = 0.0f;
    for (const Particle& p : s.parts) s.max_density = gmax(s.max_density, p.density);
    s.parts.swap(keep);
}

// FlipSim::Init (flip.cpp:42-77)
void Init(Sim& s) {
    s.parts.clear();
    ComputeMaxDensity(s);
    GenerateParticles(s);
    Sort(s);
    MarkCellTypes(s);
    s.inited = true;
}

using Clock = std::chrono::steady_clock;

void RunStage(Sim& s, int stage) {
    switch (stage) {
        case ARIEL_STAGE_BEGIN:
            s.frame++;
            AdjustParticlesStuckInSolids(s);
            StoreTemp(s);
            break;
        case ARIEL_STAGE_SORT: Sort(s); break;
        case ARIEL_STAGE_DENSITY: ComputeDensity(s); break;
        case ARIEL_STAGE_FORCES: ApplyExternalForces(s); break;
        case ARIEL_STAGE_P2G: SplatParticlesToMACGrid(s); break;
        case ARIEL_STAGE_CLASSIFY:
            MarkCellTypes(s);
            BuildSDF(s);
            break;
        case ARIEL_STAGE_BOUNDARY_DIV:
            StorePreviousGrid(s);
            EnforceBoundaryVelocity(s);
            DivergenceAndFlip(s);
            break;
        case ARIEL_STAGE_SOLVE: Solve(s); break;
        case ARIEL_STAGE_GRADIENT:
            SubtractPressureGradient(s);
            EnforceBoundaryVelocity(s);
            break;
        case ARIEL_STAGE_EXTRAPOLATE:
            ExtrapolateVelocity(s);
            SubtractPreviousGrid(s);
            break;
        case ARIEL_STAGE_G2P_ADVECT: SolvePicFlipAndAdvect(s); break;
        case ARIEL_STAGE_RESAMPLE: {
            bool run = s.prm.resample_every > 0 && (s.frame % s.prm.resample_every) == 0;
            if (run) ResampleParticles(s);
            break;
        }
        default: break;
    }
}

size_t GridBytes(const Sim& s, int which) {
    size_t n = (size_t)s.n;
    switch (which) {
        case ARIEL_GRID_UX:
        case ARIEL_GRID_UY:
        case ARIEL_GRID_UZ:
        case ARIEL_GRID_PREV_UX:
        case ARIEL_GRID_PREV_UY:
        case ARIEL_GRID_PREV_UZ: return (n + 1) * n * n * 4;
        case ARIEL_GRID_D:
        case ARIEL_GRID_P:
        case ARIEL_GRID_L:
        case ARIEL_GRID_A: return n * n * n * 4;
        case ARIEL_GRID_P64: return n * n * n * 8;
        default: return 0;
    }
}

template <class T, class F>
void ForGrid(Grid<T>& g, int ex, int ey, int ez, F f) {
    size_t t = 0;
    for (int i = 0; i < ex; ++i)
        for (int j = 0; j < ey; ++j)
            for (int k = 0; k < ez; ++k) f(g, i, j, k, t++);
}

}  // namespace

extern "C" {

ariel_status ariel_ref_create(const AsimSceneDesc* desc, const AsimParams* params, ariel_ref** out) {
    if (!desc || !params || !out || desc->dim < 2 || desc->density <= 0.0f) return ARIEL_ERR_INVALID_ARG;
    ariel_ref* s = new ariel_ref();
    s->desc = *desc;
    s->prm = *params;
    s->n = desc->dim;
    s->maxd = (float)desc->dim;
    for (int i = 0; i < desc->n_solid; ++i) {
        const AsimSphere& sp = desc->solid[i];
        s->solids.push_back(Sphere{mk(sp.center[0], sp.center[1], sp.center[2]) * s->maxd, sp.radius * s->maxd});
    }
    AllocGrids(*s);
    *out = s;
    return ARIEL_OK;
}

void ariel_ref_destroy(ariel_ref* r) { delete r; }

int32_t ariel_ref_tri_ray(const float* v, const float* o, const float* d, float* point) {
    MTri T{};
    T.a = mk(v[0], v[1], v[2]);
    T.b = mk(v[3], v[4], v[5]);
    T.c = mk(v[6], v[7], v[8]);
    const vec3 ro = mk(o[0], o[1], o[2]), rd = mk(d[0], d[1], d[2]);
    float t = 0.0f;
    if (!TriRay(T, ro, rd, t)) return 0;
    const vec3 pt = ro + rd * t;
    point[0] = pt.x;
    point[1] = pt.y;
    point[2] = pt.z;
    return 1;
}

ariel_status ariel_ref_add_mesh(ariel_ref* r, const float* vertices, int32_t n_vertices, const int32_t* triangles,
                                int32_t n_triangles, const float* translate, float scale) {
    if (!r || !vertices || !triangles || !translate || n_vertices < 3 || n_triangles < 1 || r->inited)
        return ARIEL_ERR_INVALID_ARG;
    const float maxd = r->maxd;
    const int mesh = (int)r->mlo.size();
    int key = (int)r->mtris.size();
    auto world = [&](int vi) {
        return mk((vertices[3 * vi] * scale + translate[0]) * maxd, (vertices[3 * vi + 1] * scale + translate[1]) * maxd,
                  (vertices[3 * vi + 2] * scale + translate[2]) * maxd);
    };
    vec3 lo = mk(3.0e38f, 3.0e38f, 3.0e38f), hi = mk(-3.0e38f, -3.0e38f, -3.0e38f);
    for (int t = 0; t < n_triangles; ++t) {
        MTri T;
        T.a = world(triangles[3 * t]);
        T.b = world(triangles[3 * t + 1]);
        T.c = world(triangles[3 * t + 2]);
        T.mesh = mesh;
        T.key = key++;
        for (vec3 v : {T.a, T.b, T.c}) {
            lo = mk(std::min(lo.x, v.x), std::min(lo.y, v.y), std::min(lo.z, v.z));
            hi = mk(std::max(hi.x, v.x), std::max(hi.y, v.y), std::max(hi.z, v.z));
        }
        r->mtris.push_back(T);
    }
    r->mlo.push_back(lo);
    r->mhi.push_back(hi);
    return ARIEL_OK;
}
void ariel_ref_set_faithful(ariel_ref* r, int32_t f) { r->faithful = f != 0; }
void ariel_ref_set_threads(int32_t nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
}
int32_t ariel_ref_max_threads(void) { return omp_get_max_threads(); }

ariel_status ariel_ref_init(ariel_ref* r) {
    if (!r) return ARIEL_ERR_INVALID_ARG;
    Init(*r);
    return ARIEL_OK;
}

ariel_status ariel_ref_stage(ariel_ref* r, int32_t stage) {
    if (!r || stage < 0 || stage >= ARIEL_STAGE_COUNT) return ARIEL_ERR_INVALID_ARG;
    RunStage(*r, stage);
    return ARIEL_OK;
}

ariel_status ariel_ref_step(ariel_ref* r, int32_t nsteps) {
    if (!r || nsteps < 0) return ARIEL_ERR_INVALID_ARG;
    if (!r->inited) return ARIEL_ERR_STATE;
    for (int st = 0; st < nsteps; ++st) {
        for (int g = 0; g < ARIEL_STAGE_COUNT; ++g) {
            auto t0 = Clock::now();
            RunStage(*r, g);
            r->stage_ms[g] = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        }
    }
    return ARIEL_OK;
}

ariel_status ariel_ref_particle_count(ariel_ref* r, int64_t* n) {
    if (!r || !n) return ARIEL_ERR_INVALID_ARG;
    *n = (int64_t)r->parts.size();
    return ARIEL_OK;
}

ariel_status ariel_ref_get_particles(ariel_ref* r, float* pos, float* vel, float* density, float* mass,
                                     int32_t* type) {
    if (!r) return ARIEL_ERR_INVALID_ARG;
    for (size_t i = 0; i < r->parts.size(); ++i) {
        const Particle& p = r->parts[i];
        if (pos) {
            pos[3 * i] = p.p.x;
            pos[3 * i + 1] = p.p.y;
            pos[3 * i + 2] = p.p.z;
        }
        if (vel) {
            vel[3 * i] = p.u.x;
            vel[3 * i + 1] = p.u.y;
            vel[3 * i + 2] = p.u.z;
        }
        if (density) density[i] = p.density;
        if (mass) mass[i] = p.mass;
        if (type) type[i] = p.type;
    }
    return ARIEL_OK;
}

ariel_status ariel_ref_set_particles(ariel_ref* r, int64_t n, const float* pos, const float* vel, const float* mass,
                                     const int32_t* type) {
    if (!r || n < 0 || (n > 0 && (!pos || !vel || !mass || !type))) return ARIEL_ERR_INVALID_ARG;
    r->parts.assign((size_t)n, Particle{});
    for (int64_t i = 0; i < n; ++i) {
        Particle& p = r->parts[i];
        p.p = mk(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        p.u = mk(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        p.n = mk(0, 0, 0);
        p.mass = mass[i];
        p.type = type[i];
        p.density = 10.0f;
    }
    if (!r->inited) {
        ComputeMaxDensity(*r);
        r->inited = true;
    }
    return ARIEL_OK;
}

ariel_status ariel_ref_get_cells(ariel_ref* r, int32_t* particle_cell, int32_t* cell_count) {
    if (!r) return ARIEL_ERR_INVALID_ARG;
    const int n = r->n;
    if (particle_cell)
        for (size_t i = 0; i < r->pcell.size(); ++i) particle_cell[i] = r->pcell[i];
    if (cell_count) {
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    int ci = r->pmap.get(i, j, k);
                    cell_count[cid(n, i, j, k)] = ci >= 0 ? (int32_t)r->cells[ci].size() : 0;
                }
    }
    return ARIEL_OK;
}

ariel_status ariel_ref_get_grid(ariel_ref* r, int32_t which, void* buf, int64_t nbytes) {
    if (!r || !buf || (size_t)nbytes != GridBytes(*r, which) || nbytes == 0) return ARIEL_ERR_INVALID_ARG;
    const int n = r->n;
    float* f = (float*)buf;
    int32_t* iv = (int32_t*)buf;
    auto getf = [&](Grid<float>& g, int ex, int ey, int ez) {
        ForGrid(g, ex, ey, ez, [&](Grid<float>& gg, int i, int j, int k, size_t t) { f[t] = gg.get(i, j, k); });
    };
    switch (which) {
        case ARIEL_GRID_UX: getf(r->ux, n + 1, n, n); break;
        case ARIEL_GRID_UY: getf(r->uy, n, n + 1, n); break;
        case ARIEL_GRID_UZ: getf(r->uz, n, n, n + 1); break;
        case ARIEL_GRID_PREV_UX: getf(r->pux, n + 1, n, n); break;
        case ARIEL_GRID_PREV_UY: getf(r->puy, n, n + 1, n); break;
        case ARIEL_GRID_PREV_UZ: getf(r->puz, n, n, n + 1); break;
        case ARIEL_GRID_D: getf(r->D, n, n, n); break;
        case ARIEL_GRID_P: getf(r->P, n, n, n); break;
        case ARIEL_GRID_L: getf(r->L, n, n, n); break;
        case ARIEL_GRID_A:
            ForGrid(r->A, n, n, n, [&](Grid<int>& gg, int i, int j, int k, size_t t) { iv[t] = gg.get(i, j, k); });
            break;
        case ARIEL_GRID_P64: std::memcpy(buf, r->P64.data(), (size_t)nbytes); break;
        default: return ARIEL_ERR_INVALID_ARG;
    }
    return ARIEL_OK;
}

ariel_status ariel_ref_set_grid(ariel_ref* r, int32_t which, const void* buf, int64_t nbytes) {
    if (!r || !buf || (size_t)nbytes != GridBytes(*r, which) || nbytes == 0) return ARIEL_ERR_INVALID_ARG;
    const int n = r->n;
    const float* f = (const float*)buf;
    const int32_t* iv = (const int32_t*)buf;
    auto setf = [&](Grid<float>& g, int ex, int ey, int ez) {
        ForGrid(g, ex, ey, ez, [&](Grid<float>& gg, int i, int j, int k, size_t t) { gg.set(i, j, k, f[t]); });
    };
    switch (which) {
        case ARIEL_GRID_UX: setf(r->ux, n + 1, n, n); break;
        case ARIEL_GRID_UY: setf(r->uy, n, n + 1, n); break;
        case ARIEL_GRID_UZ: setf(r->uz, n, n, n + 1); break;
        case ARIEL_GRID_PREV_UX: setf(r->pux, n + 1, n, n); break;
        case ARIEL_GRID_PREV_UY: setf(r->puy, n, n + 1, n); break;
        case ARIEL_GRID_PREV_UZ: setf(r->puz, n, n, n + 1); break;
        case ARIEL_GRID_D: setf(r->D, n, n, n); break;
        case ARIEL_GRID_P: setf(r->P, n, n, n); break;
        case ARIEL_GRID_L: setf(r->L, n, n, n); break;
        case ARIEL_GRID_A:
            ForGrid(r->A, n, n, n, [&](Grid<int>& gg, int i, int j, int k, size_t t) { gg.set(i, j, k, iv[t]); });
            break;
        case ARIEL_GRID_P64: std::memcpy(r->P64.data(), buf, (size_t)nbytes); break;
        default: return ARIEL_ERR_INVALID_ARG;
    }
    return ARIEL_OK;
}

ariel_status ariel_ref_stats(ariel_ref* r, AsimStats* st) {
    if (!r || !st) return ARIEL_ERR_INVALID_ARG;
    *st = r->st;
    st->frame = r->frame;
    st->n_particles = (int64_t)r->parts.size();
    for (int g = 0; g < ARIEL_STAGE_COUNT; ++g) st->stage_ms[g] = r->stage_ms[g];
    return ARIEL_OK;
}

ariel_status ariel_ref_get_max_density(ariel_ref* r, float* md) {
    if (!r || !md) return ARIEL_ERR_INVALID_ARG;
    *md = r->max_density;
    return ARIEL_OK;
}

ariel_status ariel_ref_stage_ms(ariel_ref* r, double* ms) {
    if (!r || !ms) return ARIEL_ERR_INVALID_ARG;
    for (int g = 0; g < ARIEL_STAGE_COUNT; ++g) ms[g] = r->stage_ms[g];
    return ARIEL_OK;
}

ariel_status ariel_ref_solve_fp64(int32_t n, const int32_t* flags, const float* L, const double* b, double* x,
                                  double tol, int32_t max_iters, int32_t* iterations, double* rel_residual) {
    if (n < 1 || !flags || !L || !b || !x) return ARIEL_ERR_INVALID_ARG;
    Op64 op;
    BuildOp64(op, n, flags, L, 1);
    Pre64 pre;
    BuildPre64(pre, op, ARIEL_PRECOND_REF, 0.97, 0.25);
    long maxit = max_iters > 0 ? max_iters : (long)n * n * n;
    Solve64Result r = PCG64(op, pre, b, x, ARIEL_STOP_REL, tol, maxit);
    if (iterations) *iterations = r.iterations;
    if (rel_residual) *rel_residual = r.rel;
    return r.converged ? ARIEL_OK : ARIEL_ERR_NOT_CONVERGED;
}

ariel_status ariel_ref_apply_fp64(int32_t n, const int32_t* flags, const float* L, const double* x, double* y) {
    if (n < 1 || !flags || !L || !x || !y) return ARIEL_ERR_INVALID_ARG;
    Op64 op;
    BuildOp64(op, n, flags, L, 1);
    long nc = (long)n * n * n;
    for (long c = 0; c < nc; ++c) y[c] = 0.0;
    Apply64(op, x, y);
    return ARIEL_OK;
}

// ---- liquid surface (the checker of ariel_get_level_set / ariel_surface_mesh) ----
// LevelSet(particles) (levelset.cpp:101-111) as spheres of radius 0.5 cells on the integer grid
// points padded 2 cells beyond the walls, band 1.5 cells, then surface nets at level 0: serial
// loops over the particles in id order, the cubes and the edges in grid order.
namespace {
const int kSPad = 2;
const float kSRadius = 0.5f, kSBand = 1.5f;

void LevelSetOf(const Sim& s, std::vector<float>& phi, int& N) {
    N = s.n + 1 + 2 * kSPad;
    phi.assign((size_t)N * N * N, kSBand);
    const float maxd = s.maxd;
    const float R = kSRadius + kSBand, R2 = R * R;
    for (const Particle& P : s.parts) {
        if (P.type != ARIEL_FLUID) continue;
        const float px = P.p.x * maxd, py = P.p.y * maxd, pz = P.p.z * maxd;
        const float pp[3] = {px, py, pz};
        int lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::max((int)std::ceil(pp[a] - R), -kSPad);
            hi[a] = std::min((int)std::floor(pp[a] + R), N - 1 - kSPad);
        }
        for (int i = lo[0]; i <= hi[0]; ++i) {
            const float dx = (float)i - px;
            for (int j = lo[1]; j <= hi[1]; ++j) {
                const float dy = (float)j - py;
                for (int k = lo[2]; k <= hi[2]; ++k) {
                    const float dz = (float)k - pz;
                    const float d2 = (dx * dx + dy * dy) + dz * dz;
                    if (!(d2 < R2)) continue;
                    const float v = std::sqrt(d2) - kSRadius;
                    float& c = phi[((size_t)(i + kSPad) * N + (j + kSPad)) * N + (k + kSPad)];
                    if (v < c) c = v;
                }
            }
        }
    }
}
}  // namespace

ariel_status ariel_ref_level_set(ariel_ref* r, float* phi, int64_t nbytes) {
    if (!r || !phi) return ARIEL_ERR_INVALID_ARG;
    std::vector<float> ls;
    int N = 0;
    LevelSetOf(*r, ls, N);
    if ((size_t)nbytes != ls.size() * sizeof(float)) return ARIEL_ERR_INVALID_ARG;
    std::memcpy(phi, ls.data(), (size_t)nbytes);
    return ARIEL_OK;
}

ariel_status ariel_ref_surface_mesh(ariel_ref* r, float* vertices, int64_t max_vertices, int32_t* quads,
                                    int64_t max_quads, int64_t* n_vertices, int64_t* n_quads) {
    if (!r || !n_vertices || !n_quads) return ARIEL_ERR_INVALID_ARG;
    std::vector<float> phi;
    int N = 0;
    LevelSetOf(*r, phi, N);
    const int M = N - 1;
    auto at = [&](int i, int j, int k) { return phi[((size_t)i * N + j) * N + k]; };
    std::vector<int> vidx((size_t)M * M * M, -1);
    std::vector<float> V;
    const int E[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < M; ++j)
            for (int k = 0; k < M; ++k) {
                float c[8];
                int inside = 0;
                for (int b = 0; b < 8; ++b) {
                    c[b] = at(i + (b & 1), j + ((b >> 1) & 1), k + ((b >> 2) & 1));
                    inside += c[b] < 0.0f ? 1 : 0;
                }
                if (inside == 0 || inside == 8) continue;
                float sx = 0.0f, sy = 0.0f, sz = 0.0f;
                int cnt = 0;
                for (int e = 0; e < 12; ++e) {
                    const int a = E[e][0], b = E[e][1];
                    if ((c[a] < 0.0f) == (c[b] < 0.0f)) continue;
                    const float t = c[a] / (c[a] - c[b]);
                    const float ax = (float)(i + (a & 1)), ay = (float)(j + ((a >> 1) & 1)), az = (float)(k + ((a >> 2) & 1));
                    const int axis = e / 4;
                    sx += axis == 0 ? ax + t : ax;
                    sy += axis == 1 ? ay + t : ay;
                    sz += axis == 2 ? az + t : az;
                    ++cnt;
                }
                const float fc = (float)cnt;
                vidx[((size_t)i * M + j) * M + k] = (int)(V.size() / 3);
                V.push_back(sx / fc - (float)kSPad);
                V.push_back(sy / fc - (float)kSPad);
                V.push_back(sz / fc - (float)kSPad);
            }
    std::vector<int32_t> Q;
    const int du[4] = {-1, 0, 0, -1}, dw[4] = {-1, -1, 0, 0};
    for (int axis = 0; axis < 3; ++axis)
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j)
                for (int k = 0; k < N; ++k) {
                    const int p[3] = {i, j, k};
                    if (p[axis] >= N - 1) continue;
                    const int u = (axis + 1) % 3, w = (axis + 2) % 3;
                    if (p[u] < 1 || p[u] > N - 2 || p[w] < 1 || p[w] > N - 2) continue;
                    int q[3] = {i, j, k};
                    q[axis] += 1;
                    const float a = at(i, j, k), b = at(q[0], q[1], q[2]);
                    if ((a < 0.0f) == (b < 0.0f)) continue;
                    int v[4];
                    for (int c = 0; c < 4; ++c) {
                        int rr[3] = {i, j, k};
                        rr[u] += du[c];
                        rr[w] += dw[c];
                        v[c] = vidx[((size_t)rr[0] * M + rr[1]) * M + rr[2]];
                    }
                    if (!(a < 0.0f)) {
                        Q.insert(Q.end(), {v[0], v[3], v[2], v[1]});
                    } else {
                        Q.insert(Q.end(), {v[0], v[1], v[2], v[3]});
                    }
                }
    *n_vertices = (int64_t)(V.size() / 3);
    *n_quads = (int64_t)(Q.size() / 4);
    if (vertices && *n_vertices <= max_vertices) std::memcpy(vertices, V.data(), V.size() * sizeof(float));
    if (quads && *n_quads <= max_quads) std::memcpy(quads, Q.data(), Q.size() * sizeof(int32_t));
    return ARIEL_OK;
}

void ariel_ref_philox4x32_10(const uint32_t* c, const uint32_t* k, uint32_t* out) {
    u4 in{{c[0], c[1], c[2], c[3]}};
    u4 o = philox(in, k[0], k[1]);
    for (int i = 0; i < 4; ++i) out[i] = o.v[i];
}

}  // extern "C"
