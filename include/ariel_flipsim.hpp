// ariel_flipsim.hpp -- header-only C++ host class over the C ABI (include/ariel.h) with the
// interface of the reference's fluidCore::FlipSim (src/sim/flip.hpp:20-66):
//   FlipSim(maxres, density, stepsize, scene, verbose), Init(), Step(saveVDB, saveOBJ,
//   savePARTIO), GetParticles(), GetDimensions(), GetScene(), m_frame.
// Two ways to construct it:
//  * from the reference's own scene object -- FlipSim(const glm::vec3& maxres, const float&
//    density, const float& stepsize, sceneCore::Scene* scene, const bool& verbose), the
//    reference constructor's exact shape.  Init() then seeds through that scene's own
//    GenerateParticles (src/scene/scene.cpp:257-360) and Step()'s export flags call its own
//    ExportParticles (src/sim/flip.cpp:125-126), so the host keeps its Partio/VDB/OBJ writers;
//  * from an AsimSceneDesc (boxes, spheres, forces), for hosts without the reference's Scene;
//    Init() seeds on the library's side and savePARTIO writes ariel_export_particles' format.
// Failures raise ariel::Error carrying the ariel_status (the reference prints and exits).
#ifndef ARIEL_FLIPSIM_HPP
#define ARIEL_FLIPSIM_HPP

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "ariel.h"

namespace ariel {

class Error : public std::runtime_error {
   public:
    Error(ariel_status code, const std::string& what)
        : std::runtime_error(what + ": " + ariel_status_string(code)), code_(code) {}
    ariel_status code() const { return code_; }

   private:
    ariel_status code_;
};

inline void check(ariel_status st, const char* what) {
    if (st != ARIEL_OK) throw Error(st, what);
}

// A reference scene file (SceneLoader's JSON) read by the library (ariel_scene_load): the scene
// description, with the settings' grid size, density, step size and output paths in *info when
// given.  Box and OBJ solids are registered meshes listed in the description; release them with
// ariel_mesh_destroy once no handle is to be created from it.  Throws Error with the loader's
// reason for what the path cannot represent.
inline AsimSceneDesc LoadScene(const std::string& path, AsimSceneInfo* info = nullptr, float jitter = 0.0f,
                               uint64_t seed = 1) {
    AsimSceneDesc d;
    AsimSceneInfo in;
    char why[512];
    const ariel_status st = ariel_scene_load(path.c_str(), jitter, seed, &d, &in, why, (int32_t)sizeof why);
    if (st != ARIEL_OK) throw Error(st, std::string("LoadScene(") + path + "): " + why);
    if (info) *info = in;
    return d;
}

// Host copy of the particle state, id order, xyz-interleaved vectors.
struct Particles {
    std::vector<float> pos, vel, density, mass;
    std::vector<int32_t> type;
    size_t size() const { return mass.size(); }
};

namespace detail {
// Type of a member function's first parameter (the particle vector of Scene::GenerateParticles).
template <class C, class R, class A0, class... As>
A0 first_param(R (C::*)(A0, As...));
template <class T>
using bare = typename std::remove_cv<typename std::remove_reference<T>::type>::type;
}  // namespace detail

// AsimSceneDesc of a reference scene (sceneCore::Scene, src/scene/scene.hpp:25-101), read through
// its public queries: GetExternalForces, GetLiquidGeoms / GetSolidGeoms with each geom's frame-0
// AABB (geomCore::GeomInterface::GetAabb, src/geom/geom.hpp), and CheckPointInsideSolidGeom --
// the query FlipSim::Step itself uses (flip.cpp:145) -- to tell a sphere from other solids: a
// solid geom whose AABB centre is inside it and whose AABB corner region is not is a sphere of
// the AABB's half width.  Geoms are in world (grid) units; the description is in unit
// coordinates.  Liquids become their AABBs (the scene files' mesh_gen cubes); the starting
// velocity is private to the Scene, so boxes get zero here -- FlipSim's Scene-pointer
// constructor takes the particles, velocities included, from the scene itself.  Throws for
// dynamic geoms, for solids that are not spheres and for more forces, liquids or solids than the
// ABI holds.
template <class SceneT>
AsimSceneDesc SceneFrom(SceneT& scene, int maxres, float density, float stepsize) {
    AsimSceneDesc d;
    ariel_scene_dambreak(&d, maxres);
    d.density = density;
    d.stepsize = stepsize;
    d.jitter = 0.0f;  // the reference seeds sub-cell centres (scene.cpp:283-297)
    const float maxd = (float)maxres;
    auto& forces = scene.GetExternalForces();
    if (forces.size() > (size_t)ARIEL_MAX_FORCES) throw Error(ARIEL_ERR_INVALID_ARG, "SceneFrom: too many forces");
    d.n_forces = (int32_t)forces.size();
    for (size_t i = 0; i < forces.size(); ++i) {
        d.forces[i][0] = forces[i].x;
        d.forces[i][1] = forces[i].y;
        d.forces[i][2] = forces[i].z;
    }
    auto& liquids = scene.GetLiquidGeoms();
    if (liquids.size() > (size_t)ARIEL_MAX_BOXES) throw Error(ARIEL_ERR_INVALID_ARG, "SceneFrom: too many liquids");
    d.n_liquid = (int32_t)liquids.size();
    for (size_t i = 0; i < liquids.size(); ++i) {
        if (liquids[i]->m_geom->IsDynamic()) throw Error(ARIEL_ERR_INVALID_ARG, "SceneFrom: animated liquid");
        auto box = liquids[i]->m_geom->GetAabb(0.0f);
        const float lo[3] = {box.m_min.x, box.m_min.y, box.m_min.z};
        const float hi[3] = {box.m_max.x, box.m_max.y, box.m_max.z};
        for (int a = 0; a < 3; ++a) {
            d.liquid[i].lo[a] = lo[a] / maxd;
            d.liquid[i].hi[a] = hi[a] / maxd;
            d.liquid[i].vel[a] = 0.0f;
        }
    }
    auto& solids = scene.GetSolidGeoms();
    if (solids.size() > (size_t)ARIEL_MAX_SPHERES) throw Error(ARIEL_ERR_INVALID_ARG, "SceneFrom: too many solids");
    d.n_solid = (int32_t)solids.size();
    for (size_t i = 0; i < solids.size(); ++i) {
        if (solids[i]->m_geom->IsDynamic()) throw Error(ARIEL_ERR_INVALID_ARG, "SceneFrom: animated solid");
        auto box = solids[i]->m_geom->GetAabb(0.0f);
        auto centre = box.m_min;
        centre.x = 0.5f * (box.m_min.x + box.m_max.x);
        centre.y = 0.5f * (box.m_min.y + box.m_max.y);
        centre.z = 0.5f * (box.m_min.z + box.m_max.z);
        auto corner = box.m_min;
        corner.x = box.m_min.x + 0.1f * (box.m_max.x - box.m_min.x);
        corner.y = box.m_min.y + 0.1f * (box.m_max.y - box.m_min.y);
        corner.z = box.m_min.z + 0.1f * (box.m_max.z - box.m_min.z);
        unsigned int id = 0;
        const bool sphere = scene.CheckPointInsideSolidGeom(centre, 0.0f, id) &&
                            !scene.CheckPointInsideSolidGeom(corner, 0.0f, id);
        if (!sphere) throw Error(ARIEL_ERR_INVALID_ARG, "SceneFrom: only sphere solids are supported");
        d.solid[i].center[0] = centre.x / maxd;
        d.solid[i].center[1] = centre.y / maxd;
        d.solid[i].center[2] = centre.z / maxd;
        d.solid[i].radius = 0.5f * (box.m_max.x - box.m_min.x) / maxd;
    }
    return d;
}

class FlipSim {
   public:
    // maxres/density/stepsize override the scene's grid size, lattice density and time step,
    // as the reference constructor's arguments do (flip.cpp:15-30).
    FlipSim(int maxres, float density, float stepsize, const AsimSceneDesc& scene, bool verbose = false,
            const AsimParams* params = nullptr)
        : m_frame(0), scene_(scene), verbose_(verbose) {
        scene_.dim = maxres;
        scene_.density = density;
        scene_.stepsize = stepsize;
        create(params);
    }

    // The reference constructor's shape (flip.hpp:22-23) over the host's own scene object.  The
    // grid must be cubic (the reference's G2P treats every axis as the largest,
    // particlegridoperations.inl:121-124).  The scene is read by SceneFrom; Init() seeds through
    // scene->GenerateParticles and Step() exports through scene->ExportParticles.
    template <class Vec3, class SceneT>
    FlipSim(const Vec3& maxres, const float& density, const float& stepsize, SceneT* scene, const bool& verbose,
            const AsimParams* params = nullptr)
        : m_frame(0), verbose_(verbose) {
        if (!scene) throw Error(ARIEL_ERR_INVALID_ARG, "FlipSim: null scene");
        if (!(maxres.x == maxres.y && maxres.y == maxres.z) || maxres.x < 2.0f)
            throw Error(ARIEL_ERR_INVALID_ARG, "FlipSim: the grid must be cubic");
        const int n = (int)maxres.x;
        scene_ = SceneFrom(*scene, n, density, stepsize);
        create(params);
        using PVec = detail::bare<decltype(detail::first_param(&SceneT::GenerateParticles))>;
        auto host = std::make_shared<PVec>();
        const Vec3 dims = maxres;
        const float dens = density;
        seed_ = [scene, host, dims, dens](Particles& out) {
            host->clear();
            // FlipSim::Init's call (flip.cpp:74): frame 0 builds the liquid and static solid sets
            scene->GenerateParticles(*host, dims, dens, nullptr, 0);
            const size_t np = host->size();
            out.pos.resize(3 * np);
            out.vel.resize(3 * np);
            out.mass.resize(np);
            out.type.resize(np);
            for (size_t i = 0; i < np; ++i) {
                const auto* p = (*host)[i];
                out.pos[3 * i] = p->m_p.x;
                out.pos[3 * i + 1] = p->m_p.y;
                out.pos[3 * i + 2] = p->m_p.z;
                out.vel[3 * i] = p->m_u.x;
                out.vel[3 * i + 1] = p->m_u.y;
                out.vel[3 * i + 2] = p->m_u.z;
                out.mass[i] = p->m_mass;
                out.type[i] = p->m_type;
            }
        };
        const float maxd = maxres.x;
        export_ = [scene, host, maxd](const Particles& cur, int frame, bool vdb, bool obj, bool partio) {
            // the GPU state goes back into the scene's own particle objects, then the scene's own
            // writer runs, as FlipSim::Step does (flip.cpp:125-126)
            for (size_t i = 0; i < host->size() && i < cur.size(); ++i) {
                auto* p = (*host)[i];
                p->m_p.x = cur.pos[3 * i];
                p->m_p.y = cur.pos[3 * i + 1];
                p->m_p.z = cur.pos[3 * i + 2];
                p->m_u.x = cur.vel[3 * i];
                p->m_u.y = cur.vel[3 * i + 1];
                p->m_u.z = cur.vel[3 * i + 2];
            }
            scene->ExportParticles(*host, maxd, frame, vdb, obj, partio);
        };
    }

    ~FlipSim() {
        if (sim_) ariel_destroy(sim_);
    }
    FlipSim(const FlipSim&) = delete;
    FlipSim& operator=(const FlipSim&) = delete;

    // FlipSim::Init (flip.cpp:42-77): the density normaliser, seeding, first sort and cell types.
    void Init() {
        if (seed_) {
            Particles p;
            seed_(p);
            check(ariel_set_particles(sim_, 0, (int64_t)p.size(), p.pos.data(), p.vel.data(), p.mass.data(),
                                      p.type.data()),
                  "ariel_set_particles");
        } else {
            check(ariel_init(sim_), "ariel_init");
        }
        m_frame = 0;
    }

    // FlipSim::Step (flip.cpp:92-128).  With any export flag set the particles are written after
    // the step: through the host scene's ExportParticles when constructed from one; otherwise
    // savePARTIO writes ariel_export_particles' Houdini ASCII geometry to the path given by
    // SetPartioPath, saveOBJ the liquid surface (ariel_export_surface) to the path given by
    // SetMeshPath, and saveVDB (an OpenVDB file) is refused.
    void Step(bool saveVDB = false, bool saveOBJ = false, bool savePARTIO = false) {
        check(ariel_step(sim_, 1), "ariel_step");
        ++m_frame;
        if (verbose_) {
            AsimStats st;
            check(ariel_stats(sim_, 0, &st), "ariel_stats");
            std::fprintf(stderr, "Simulating Step: %d... PCG %d iterations, residual %.3e\n", m_frame,
                         st.pcg_iterations, st.pcg_rel_residual);
        }
        if (!(saveVDB || saveOBJ || savePARTIO)) return;
        if (export_) {
            export_(GetParticles(), m_frame, saveVDB, saveOBJ, savePARTIO);
            return;
        }
        if (saveVDB) throw Error(ARIEL_ERR_INVALID_ARG, "Step: VDB export needs the host scene's writers");
        if (savePARTIO) {
            if (partio_path_.empty()) throw Error(ARIEL_ERR_INVALID_ARG, "Step: savePARTIO without SetPartioPath");
            check(ariel_export_particles(sim_, 0, partio_path_.c_str(), m_frame), "ariel_export_particles");
        }
        if (saveOBJ) {
            if (mesh_path_.empty()) throw Error(ARIEL_ERR_INVALID_ARG, "Step: saveOBJ without SetMeshPath");
            check(ariel_export_surface(sim_, 0, mesh_path_.c_str(), m_frame), "ariel_export_surface");
        }
    }

    // Target of savePARTIO without a host scene (Scene::SetPaths' partio path, scene.cpp:26-33);
    // must end in ".geo", the frame number is inserted before the extension.
    void SetPartioPath(const std::string& path) { partio_path_ = path; }
    // Target of saveOBJ without a host scene (Scene::SetPaths' mesh path): must end in ".obj".
    void SetMeshPath(const std::string& path) { mesh_path_ = path; }

    // FlipSim::GetParticles (flip.hpp:29): a host copy, refreshed on each call.
    const Particles& GetParticles() {
        int64_t n = 0;
        check(ariel_particle_count(sim_, 0, &n), "ariel_particle_count");
        parts_.pos.resize(3 * n);
        parts_.vel.resize(3 * n);
        parts_.density.resize(n);
        parts_.mass.resize(n);
        parts_.type.resize(n);
        check(ariel_get_particles(sim_, 0, parts_.pos.data(), parts_.vel.data(), parts_.density.data(),
                                  parts_.mass.data(), parts_.type.data()),
              "ariel_get_particles");
        return parts_;
    }

    // FlipSim::GetDimensions (flip.hpp:30)
    std::array<int, 3> GetDimensions() const { return {scene_.dim, scene_.dim, scene_.dim}; }
    // FlipSim::GetScene (flip.hpp:31): the scene as the library holds it
    const AsimSceneDesc& GetScene() const { return scene_; }
    ariel_sim* handle() { return sim_; }

    int m_frame;

   private:
    void create(const AsimParams* params) {
        AsimParams p;
        if (params)
            p = *params;
        else
            ariel_params_default(&p);
        check(ariel_create(&scene_, &p, &sim_), "ariel_create");
    }

    AsimSceneDesc scene_;
    bool verbose_;
    ariel_sim* sim_ = nullptr;
    Particles parts_;
    std::string partio_path_, mesh_path_;
    std::function<void(Particles&)> seed_;
    std::function<void(const Particles&, int, bool, bool, bool)> export_;
};

// Request server (ariel_server_*): scenes of any size submitted from any thread are stepped
// together; results are fetched by request id.  No counterpart in the reference.
class Server {
   public:
    explicit Server(const AsimParams* params = nullptr, const AsimServerConfig* config = nullptr) {
        AsimParams p;
        if (params)
            p = *params;
        else
            ariel_params_default(&p);
        AsimServerConfig c;
        if (config)
            c = *config;
        else
            ariel_server_config_default(&c);
        check(ariel_server_create(&p, &c, &srv_), "ariel_server_create");
    }
    ~Server() {
        if (srv_) ariel_server_shutdown(srv_);
    }
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    int64_t Submit(const AsimSceneDesc& scene, int32_t nsteps) {
        int64_t id = 0;
        check(ariel_server_submit(srv_, &scene, nsteps, &id), "ariel_server_submit");
        return id;
    }
    AsimRequestInfo Poll(int64_t id) {
        AsimRequestInfo info;
        check(ariel_server_poll(srv_, id, &info), "ariel_server_poll");
        return info;
    }
    void Wait(int64_t id, double timeout_ms = 1.0e9) { check(ariel_server_wait(srv_, id, timeout_ms), "ariel_server_wait"); }
    void Drain(double timeout_ms = 1.0e9) { check(ariel_server_drain(srv_, timeout_ms), "ariel_server_drain"); }
    // Positions and velocities of a finished request, id order, xyz-interleaved.
    void Fetch(int64_t id, std::vector<float>& pos, std::vector<float>& vel) {
        const AsimRequestInfo info = Poll(id);
        pos.resize(3 * (size_t)info.n_particles);
        vel.resize(3 * (size_t)info.n_particles);
        check(ariel_server_fetch(srv_, id, pos.data(), vel.data()), "ariel_server_fetch");
    }
    AsimServerStats Stats() {
        AsimServerStats st;
        check(ariel_server_stats(srv_, &st), "ariel_server_stats");
        return st;
    }

   private:
    ariel_server* srv_ = nullptr;
};

}  // namespace ariel

#endif
