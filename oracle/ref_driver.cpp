// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.  Builds betajippity/Ariel's own FLIP step into
// oracle/_ref/libariel_reference.so so that the oracle (oracle/ariel_oracle.cpp) can be held to
// the reference's arithmetic instead of only to hand-derived answers.
//
// The reference's sources are compiled where they lie (-I <reference>/src, then #include of
// src/grid/particlegrid.cpp and src/sim/flip.cpp, which pulls in src/sim/solver.inl,
// particlegridoperations.inl, particleresampler.inl, src/math/kernels.inl, src/grid/grid.inl,
// macgrid.inl and gridutils.inl).  Nothing of them is copied or edited.  oracle/refshim/ stands
// in for the libraries they need and this environment lacks (glm, TBB, OpenVDB, the Takua
// utility header, the ray and scene headers); see oracle/refshim/prelude.hpp.
//
// Two test-only devices reach into the unmodified sources:
//  * `#define private public` around the includes, so the driver can call FlipSim's stage
//    functions (src/sim/flip.hpp:35-48) one at a time;
//  * `#define rand() ...` around the includes: the resampler's three rand() calls per close
//    fluid neighbour (src/sim/particleresampler.inl:69-71) draw from Philox4x32-10 keyed by
//    (seed, frame, particle index, draw ordinal / 3) and take word (ordinal % 3) -- the stream
//    the oracle and the CUDA library use.  The macro returns the word reduced modulo 101, so the
//    reference's `rand()%101` sees exactly the oracle's `word % 101`.
//
// Solids are analytic spheres (the benchmark scenes' only solids): the Scene stand-in answers
// CheckPointInsideSolidGeom, IntersectSolidGeoms and the level set's ProjectPointsToSurface for
// spheres, in place of the reference's mesh BVH and OpenVDB (src/scene/scene.cpp:382-434,
// src/grid/levelset.cpp:175-193).  Those three answers are therefore the oracle's own formulas,
// not the reference's; everything that calls them is the reference's code.
//
// Scene::GenerateParticles hands the reference, at frame 0, the particle list the test supplies
// (the oracle's seeded lattice); at later frames it leaves the list alone, which is what the
// reference's rebuild of the same pointers in the same order amounts to for scenes whose liquid
// is emitted once and whose solids are static (src/scene/scene.cpp:335-358).
#include <cstring>
#include <unordered_map>

extern "C" int ariel_pin_rand_draw(unsigned int n0, float frame);

#define private public
#define rand() ariel_pin_rand_draw(n0, frame)
#include "grid/particlegrid.cpp"
#include "sim/flip.cpp"
#undef rand
#undef private

namespace {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): ten rounds of two 32x32->64-bit products
// with the Weyl key schedule.
void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t o0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        uint32_t o1 = (uint32_t)p1;
        uint32_t o2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        uint32_t o3 = (uint32_t)p0;
        c[0] = o0;
        c[1] = o1;
        c[2] = o2;
        c[3] = o3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

const uint32_t kTagResample = 0x5245534Du;  // "RESM": the resampling jitter's stream

struct RandState {
    unsigned int last_n0 = 0xFFFFFFFFu;
    float last_frame = -1.0f;
    uint32_t draws = 0;
};
uint64_t g_rand_seed = 0;
// per thread: the timing build's OpenMP workers each draw for their own particles
thread_local RandState g_rand;

// A null stream buffer: the reference prints every step and every PCG iteration
// (src/sim/flip.cpp:94, src/sim/solver.inl:336-337); the driver silences std::cout while it runs.
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
} g_null;

struct Quiet {
    std::streambuf* old;
    Quiet() : old(std::cout.rdbuf(&g_null)) {}
    ~Quiet() { std::cout.rdbuf(old); }
};

}  // namespace

extern "C" int ariel_pin_rand_draw(unsigned int n0, float frame) {
    if (n0 != g_rand.last_n0 || frame != g_rand.last_frame) {
        g_rand.last_n0 = n0;
        g_rand.last_frame = frame;
        g_rand.draws = 0;
    }
    uint32_t d = g_rand.draws++;
    uint32_t c[4] = {(uint32_t)n0, (uint32_t)frame, d / 3u, kTagResample};
    philox4x32_10(c, (uint32_t)g_rand_seed, (uint32_t)(g_rand_seed >> 32));
    return (int)(c[d % 3u] % 101u);
}

// ---------------------------------------------------------------------------------------------
// Scene and level-set stand-ins (declared in oracle/refshim/prelude.hpp)
// ---------------------------------------------------------------------------------------------
namespace sceneCore {

void Scene::GenerateParticles(std::vector<fluidCore::Particle*>& particles, const glm::vec3&, const float&,
                              fluidCore::ParticleGrid*, const int& frame) {
    if (frame != 0) return;
    for (fluidCore::Particle* p : m_initialParticles) particles.push_back(p);
    m_initialParticles.clear();
}

std::vector<glm::vec3>& Scene::GetExternalForces() { return m_externalForces; }
fluidCore::LevelSet* Scene::GetSolidLevelSet() { return &m_solidLevelSet; }
fluidCore::LevelSet* Scene::GetLiquidLevelSet() { return &m_liquidLevelSet; }
void Scene::BuildSolidGeomLevelSet(const int&) {}
void Scene::BuildPermaSolidGeomLevelSet() {}
void Scene::ExportParticles(std::vector<fluidCore::Particle*>, const float&, const int&, const bool&, const bool&,
                            const bool&) {}

bool Scene::CheckPointInsideSolidGeom(const glm::vec3& p, const float&, unsigned int& solidGeomID) {
    for (size_t i = 0; i < m_sphereCenters.size(); ++i) {
        glm::vec3 d = p - m_sphereCenters[i];
        if (glm::dot(d, d) < m_sphereRadii[i] * m_sphereRadii[i]) {
            solidGeomID = (unsigned int)i;
            return true;
        }
    }
    return false;
}

rayCore::Intersection Scene::IntersectSolidGeoms(const rayCore::Ray& r) {
    rayCore::Intersection bestHit;
    for (size_t i = 0; i < m_sphereCenters.size(); ++i) {
        rayCore::Intersection hit;
        glm::vec3 oc = r.m_origin - m_sphereCenters[i];
        float b = glm::dot(r.m_direction, oc);
        float c = glm::dot(oc, oc) - m_sphereRadii[i] * m_sphereRadii[i];
        float disc = b * b - c;
        if (disc >= 0.0f) {
            float sq = std::sqrt(disc);
            float t = -b - sq;
            if (!(t > 0.0f)) t = -b + sq;
            if (t > 0.0f) {
                glm::vec3 pt = r.m_origin + r.m_direction * t;
                hit = rayCore::Intersection(true, pt, glm::normalize(pt - m_sphereCenters[i]));
            }
        }
        bestHit = bestHit.CompareClosestAgainst(hit, r.m_origin);
    }
    return bestHit;
}

}  // namespace sceneCore

namespace fluidCore {

void LevelSet::ProjectPointsToSurface(std::vector<Particle*>& particles, const float& pscale) {
    for (Particle* p : particles) {
        glm::vec3 w = p->m_p * pscale;
        for (size_t i = 0; i < m_owner->m_sphereCenters.size(); ++i) {
            glm::vec3 d = w - m_owner->m_sphereCenters[i];
            if (glm::dot(d, d) < m_owner->m_sphereRadii[i] * m_owner->m_sphereRadii[i]) {
                w = m_owner->m_sphereCenters[i] + glm::normalize(d) * m_owner->m_sphereRadii[i];
                break;
            }
        }
        p->m_p = w / pscale;
    }
}

float LevelSet::GetCell(const int&, const int&, const int&) { return 1.0f; }

}  // namespace fluidCore

// ---------------------------------------------------------------------------------------------
// C API (ctypes) -- stage numbers follow include/ariel.h's ARIEL_STAGE_* where the reference's
// functions allow the same cut; see ariel_pin_stage.
// ---------------------------------------------------------------------------------------------
struct ariel_pin {
    sceneCore::Scene scene;
    fluidCore::FlipSim* sim = nullptr;
    int n = 0;
    bool inited = false;
};

namespace {

fluidCore::Particle* NewParticle(const float* pos, const float* vel, float mass, int type) {
    fluidCore::Particle* p = new fluidCore::Particle;
    p->m_p = glm::vec3(pos[0], pos[1], pos[2]);
    p->m_u = glm::vec3(vel[0], vel[1], vel[2]);
    p->m_n = glm::vec3(0.0f);
    p->m_density = 10.0f;
    p->m_mass = mass;
    p->m_type = type;
    p->m_t = glm::vec3(0.0f);
    p->m_t2 = glm::vec3(0.0f);
    p->m_ut = glm::vec3(0.0f);
    p->m_pt = glm::vec3(0.0f);
    p->m_invalid = false;
    p->m_temp = false;
    p->m_temp2 = false;
    return p;
}

fluidCore::Grid<float>* FloatGrid(ariel_pin* h, int which, int& ex, int& ey, int& ez) {
    const int n = h->n;
    fluidCore::FlipSim* s = h->sim;
    ex = ey = ez = n;
    switch (which) {
        case 0: ex = n + 1; return s->m_mgrid.m_u_x;
        case 1: ey = n + 1; return s->m_mgrid.m_u_y;
        case 2: ez = n + 1; return s->m_mgrid.m_u_z;
        case 3: ex = n + 1; return s->m_mgrid_previous.m_u_x;
        case 4: ey = n + 1; return s->m_mgrid_previous.m_u_y;
        case 5: ez = n + 1; return s->m_mgrid_previous.m_u_z;
        case 6: return s->m_mgrid.m_D;
        case 7: return s->m_mgrid.m_P;
        case 8: return s->m_mgrid.m_L;
        default: return nullptr;
    }
}

}  // namespace

extern "C" {

// n: cubic grid; density, dt: FlipSim's constructor arguments (src/sim/flip.hpp:22-23);
// forces: nforces xyz triples; spheres: nspheres (cx, cy, cz, r) in unit coordinates;
// rng_seed: the resampling jitter's Philox key.
ariel_pin* ariel_pin_create(int32_t n, float density, float dt, const float* forces, int32_t nforces,
                            const float* spheres, int32_t nspheres, uint64_t rng_seed) {
    if (n < 2 || density <= 0.0f || nforces < 0 || nspheres < 0) return nullptr;
    ariel_pin* h = new ariel_pin();
    h->n = n;
    const float maxd = (float)n;
    for (int i = 0; i < nforces; ++i)
        h->scene.m_externalForces.push_back(glm::vec3(forces[3 * i], forces[3 * i + 1], forces[3 * i + 2]));
    for (int i = 0; i < nspheres; ++i) {
        h->scene.m_sphereCenters.push_back(glm::vec3(spheres[4 * i], spheres[4 * i + 1], spheres[4 * i + 2]) * maxd);
        h->scene.m_sphereRadii.push_back(spheres[4 * i + 3] * maxd);
    }
    h->scene.m_solidLevelSet.m_owner = &h->scene;
    h->scene.m_liquidLevelSet.m_owner = &h->scene;
    g_rand = RandState();
    g_rand_seed = rng_seed;
    Quiet q;
    h->sim = new fluidCore::FlipSim(glm::vec3(n, n, n), density, dt, &h->scene, false);
    return h;
}

void ariel_pin_destroy(ariel_pin* h) {
    if (!h) return;
    for (fluidCore::Particle* p : h->scene.m_initialParticles) delete p;
    delete h->sim;
    delete h;
}

// The particle list Scene::GenerateParticles hands over at frame 0 (call before ariel_pin_init).
int32_t ariel_pin_set_scene_particles(ariel_pin* h, int64_t np, const float* pos, const float* vel,
                                      const float* mass, const int32_t* type) {
    if (!h || np < 0 || h->inited) return 1;
    for (fluidCore::Particle* p : h->scene.m_initialParticles) delete p;
    h->scene.m_initialParticles.clear();
    for (int64_t i = 0; i < np; ++i)
        h->scene.m_initialParticles.push_back(NewParticle(pos + 3 * i, vel + 3 * i, mass[i], type[i]));
    return 0;
}

// FlipSim::Init (src/sim/flip.cpp:42-77).
int32_t ariel_pin_init(ariel_pin* h) {
    if (!h || h->inited) return 1;
    Quiet q;
    h->sim->Init();
    h->inited = true;
    return 0;
}

// FlipSim::Step(false, false, false) (src/sim/flip.cpp:92-128), nsteps times.
int32_t ariel_pin_step(ariel_pin* h, int32_t nsteps) {
    if (!h || !h->inited || nsteps < 0) return 1;
    Quiet q;
    for (int s = 0; s < nsteps; ++s) h->sim->Step(false, false, false);
    return 0;
}

// One cut of FlipSim::Step, numbered as include/ariel.h's ARIEL_STAGE_* (src/sim/flip.cpp:93-123):
//  0 BEGIN       m_frame++, GenerateParticles, BuildSolidGeomLevelSet,
//                AdjustParticlesStuckInSolids, StoreTempParticleVelocities      (:93-103)
//  1 SORT        ParticleGrid::Sort                                              (:104)
//  2 DENSITY     ComputeDensity                                                  (:105)
//  3 FORCES      ApplyExternalForces                                             (:106)
//  4 P2G         SplatParticlesToMACGrid                                         (:107)
//  5 CLASSIFY    MarkCellTypes, then ParticleGrid::BuildSDF (called inside Project, :440; it reads
//                only the particle lists and densities, so running it here changes nothing)
//  6 BOUNDARY    StorePreviousGrid, EnforceBoundaryVelocity                      (:109-110)
//                (the divergence is computed inside Project: see 12)
//  7 SOLVE       Solve (FlipGrid + BuildPreconditioner + SolveConjugateGradient, solver.inl:356-379):
//                D must hold the divergence BEFORE FlipGrid
//  8 GRADIENT    SubtractPressureGradient, EnforceBoundaryVelocity               (:449, :112)
//  9 EXTRAPOLATE ExtrapolateVelocity, SubtractPreviousGrid                       (:113-114)
// 10 G2P_ADVECT  SolvePicFlip, AdvectParticles, CheckParticleSolidConstraints    (:115-118)
// 11 RESAMPLE    StoreTempParticleVelocities, ResampleParticles,
//                CheckParticleSolidConstraints                                   (:119-123)
// 12 PROJECT     StorePreviousGrid, EnforceBoundaryVelocity, Project, EnforceBoundaryVelocity
//                (:109-112; = stages 6-8 of include/ariel.h)
int32_t ariel_pin_stage(ariel_pin* h, int32_t stage) {
    if (!h || !h->inited) return 1;
    fluidCore::FlipSim* s = h->sim;
    Quiet q;
    const float maxd = glm::max(glm::max(s->m_dimensions.x, s->m_dimensions.z), s->m_dimensions.y);
    switch (stage) {
        case 0:
            s->m_frame++;
            s->m_scene->GenerateParticles(s->m_particles, s->m_dimensions, s->m_density, s->m_pgrid, s->m_frame);
            s->m_scene->BuildSolidGeomLevelSet(s->m_frame);
            s->AdjustParticlesStuckInSolids();
            s->StoreTempParticleVelocities();
            break;
        case 1: s->m_pgrid->Sort(s->m_particles); break;
        case 2: s->ComputeDensity(); break;
        case 3: s->ApplyExternalForces(); break;
        case 4: fluidCore::SplatParticlesToMACGrid(s->m_pgrid, s->m_particles, &s->m_mgrid); break;
        case 5:
            s->m_pgrid->MarkCellTypes(s->m_particles, s->m_mgrid.m_A, s->m_density);
            s->m_pgrid->BuildSDF(s->m_mgrid, s->m_density);
            break;
        case 6:
            s->StorePreviousGrid();
            fluidCore::EnforceBoundaryVelocity(&s->m_mgrid);
            break;
        case 7: fluidCore::Solve(s->m_mgrid, s->m_subcell, s->m_verbose); break;
        case 8:
            s->SubtractPressureGradient();
            fluidCore::EnforceBoundaryVelocity(&s->m_mgrid);
            break;
        case 9:
            s->ExtrapolateVelocity();
            s->SubtractPreviousGrid();
            break;
        case 10:
            s->SolvePicFlip();
            s->AdvectParticles();
            s->CheckParticleSolidConstraints();
            break;
        case 11: {
            s->StoreTempParticleVelocities();
            float h2 = s->m_density / maxd;
            fluidCore::ResampleParticles(s->m_pgrid, s->m_particles, s->m_scene, s->m_frame, s->m_stepsize, h2,
                                         s->m_dimensions);
            s->CheckParticleSolidConstraints();
            break;
        }
        case 12:
            s->StorePreviousGrid();
            fluidCore::EnforceBoundaryVelocity(&s->m_mgrid);
            s->Project();
            fluidCore::EnforceBoundaryVelocity(&s->m_mgrid);
            break;
        default: return 1;
    }
    return 0;
}

int64_t ariel_pin_particle_count(ariel_pin* h) { return h && h->sim ? (int64_t)h->sim->m_particles.size() : -1; }

int32_t ariel_pin_get_particles(ariel_pin* h, float* pos, float* vel, float* density, float* mass, int32_t* type) {
    if (!h) return 1;
    const std::vector<fluidCore::Particle*>& ps = h->sim->m_particles;
    for (size_t i = 0; i < ps.size(); ++i) {
        const fluidCore::Particle* p = ps[i];
        if (pos) {
            pos[3 * i] = p->m_p.x;
            pos[3 * i + 1] = p->m_p.y;
            pos[3 * i + 2] = p->m_p.z;
        }
        if (vel) {
            vel[3 * i] = p->m_u.x;
            vel[3 * i + 1] = p->m_u.y;
            vel[3 * i + 2] = p->m_u.z;
        }
        if (density) density[i] = p->m_density;
        if (mass) mass[i] = p->m_mass;
        if (type) type[i] = p->m_type;
    }
    return 0;
}

// Replaces the particle vector (new particles as the oracle's ariel_ref_set_particles makes them).
// Before ariel_pin_init this runs Init on an empty scene first, which computes the density
// normaliser m_max_density (src/sim/flip.cpp:42-70) as the oracle does.
int32_t ariel_pin_set_particles(ariel_pin* h, int64_t np, const float* pos, const float* vel, const float* mass,
                                const int32_t* type) {
    if (!h || np < 0) return 1;
    if (!h->inited) {
        for (fluidCore::Particle* p : h->scene.m_initialParticles) delete p;
        h->scene.m_initialParticles.clear();
        if (ariel_pin_init(h)) return 1;
    }
    std::vector<fluidCore::Particle*>& ps = h->sim->m_particles;
    for (fluidCore::Particle* p : ps) delete p;
    ps.clear();
    for (int64_t i = 0; i < np; ++i) ps.push_back(NewParticle(pos + 3 * i, vel + 3 * i, mass[i], type[i]));
    return 0;
}

// Per particle, the linear cell (i*n + j)*n + k of the list that holds it after the last Sort;
// per cell, the length of its list (ParticleGrid::m_grid / m_cells, src/grid/particlegrid.hpp:44-46).
int32_t ariel_pin_get_cells(ariel_pin* h, int32_t* particle_cell, int32_t* cell_count) {
    if (!h) return 1;
    const int n = h->n;
    fluidCore::ParticleGrid* g = h->sim->m_pgrid;
    std::unordered_map<const fluidCore::Particle*, int64_t> index;
    const std::vector<fluidCore::Particle*>& ps = h->sim->m_particles;
    for (size_t i = 0; i < ps.size(); ++i) index[ps[i]] = (int64_t)i;
    if (particle_cell)
        for (size_t i = 0; i < ps.size(); ++i) particle_cell[i] = -1;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                const int32_t c = (i * n + j) * n + k;
                int ci = g->m_grid->GetCell(i, j, k);
                int32_t cnt = 0;
                if (ci >= 0 && ci < (int)g->m_cells.size()) {
                    cnt = (int32_t)g->m_cells[ci].size();
                    if (particle_cell)
                        for (const fluidCore::Particle* p : g->m_cells[ci]) {
                            auto it = index.find(p);
                            if (it != index.end()) particle_cell[it->second] = c;
                        }
                }
                if (cell_count) cell_count[c] = cnt;
            }
    return 0;
}

// Grids, selected as include/ariel.h's ARIEL_GRID_* (0-8 f32, 9 the int32 cell types), laid out
// with the first index slowest.
int32_t ariel_pin_get_grid(ariel_pin* h, int32_t which, void* buf) {
    if (!h || !buf) return 1;
    const int n = h->n;
    if (which == 9) {
        int32_t* o = (int32_t*)buf;
        size_t t = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) o[t++] = h->sim->m_mgrid.m_A->GetCell(i, j, k);
        return 0;
    }
    int ex, ey, ez;
    fluidCore::Grid<float>* g = FloatGrid(h, which, ex, ey, ez);
    if (!g) return 1;
    float* o = (float*)buf;
    size_t t = 0;
    for (int i = 0; i < ex; ++i)
        for (int j = 0; j < ey; ++j)
            for (int k = 0; k < ez; ++k) o[t++] = g->GetCell(i, j, k);
    return 0;
}

int32_t ariel_pin_set_grid(ariel_pin* h, int32_t which, const void* buf) {
    if (!h || !buf) return 1;
    const int n = h->n;
    if (which == 9) {
        const int32_t* v = (const int32_t*)buf;
        size_t t = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) h->sim->m_mgrid.m_A->SetCell(i, j, k, v[t++]);
        return 0;
    }
    int ex, ey, ez;
    fluidCore::Grid<float>* g = FloatGrid(h, which, ex, ey, ez);
    if (!g) return 1;
    const float* v = (const float*)buf;
    size_t t = 0;
    for (int i = 0; i < ex; ++i)
        for (int j = 0; j < ey; ++j)
            for (int k = 0; k < ez; ++k) g->SetCell(i, j, k, v[t++]);
    return 0;
}

// Host threads the timing build's parallel_for uses (1 for the serial builds).
int32_t ariel_pin_threads(void) {
#if defined(ARIEL_TBB_OPENMP) && defined(_OPENMP)
    return omp_get_max_threads();
#else
    return 1;
#endif
}

float ariel_pin_max_density(ariel_pin* h) { return h ? h->sim->m_max_density : 0.0f; }
int32_t ariel_pin_frame(ariel_pin* h) { return h ? h->sim->m_frame : -1; }

// Philox4x32-10 of the driver's rand() stand-in, exposed for known-answer tests.
void ariel_pin_philox4x32_10(const uint32_t* c, const uint32_t* k, uint32_t* out) {
    uint32_t v[4] = {c[0], c[1], c[2], c[3]};
    philox4x32_10(v, k[0], k[1]);
    std::memcpy(out, v, sizeof v);
}

}  // extern "C"
