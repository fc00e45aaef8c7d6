// ariel_flipsim.hpp -- header-only C++ host class over the C ABI (include/ariel.h) with the
// interface of the reference's fluidCore::FlipSim (src/sim/flip.hpp:20-66):
//   FlipSim(maxres, density, stepsize, scene, verbose), Init(), Step(saveVDB, saveOBJ,
//   savePARTIO), GetParticles(), GetDimensions(), GetScene(), m_frame.
// Failures raise ariel::Error carrying the ariel_status (the reference prints and exits).
#ifndef ARIEL_FLIPSIM_HPP
#define ARIEL_FLIPSIM_HPP

#include <array>
#include <cstdio>
#include <cstdint>
#include <stdexcept>
#include <string>
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

// Host copy of the particle state, id order, xyz-interleaved vectors.
struct Particles {
    std::vector<float> pos, vel, density, mass;
    std::vector<int32_t> type;
    size_t size() const { return mass.size(); }
};

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
        AsimParams p;
        if (params)
            p = *params;
        else
            ariel_params_default(&p);
        check(ariel_create(&scene_, &p, &sim_), "ariel_create");
    }
    ~FlipSim() {
        if (sim_) ariel_destroy(sim_);
    }
    FlipSim(const FlipSim&) = delete;
    FlipSim& operator=(const FlipSim&) = delete;

    // FlipSim::Init (flip.cpp:42-77)
    void Init() {
        check(ariel_init(sim_), "ariel_init");
        m_frame = 0;
    }

    // FlipSim::Step (flip.cpp:92-128).  The export flags are accepted for interface parity;
    // exporting is done by the caller from GetParticles().
    void Step(bool /*saveVDB*/ = false, bool /*saveOBJ*/ = false, bool /*savePARTIO*/ = false) {
        check(ariel_step(sim_, 1), "ariel_step");
        ++m_frame;
        if (verbose_) {
            AsimStats st;
            check(ariel_stats(sim_, 0, &st), "ariel_stats");
            std::fprintf(stderr, "Simulating Step: %d... PCG %d iterations, residual %.3e\n", m_frame,
                         st.pcg_iterations, st.pcg_rel_residual);
        }
    }

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
    // FlipSim::GetScene (flip.hpp:31)
    const AsimSceneDesc& GetScene() const { return scene_; }
    ariel_sim* handle() { return sim_; }

    int m_frame;

   private:
    AsimSceneDesc scene_;
    bool verbose_;
    ariel_sim* sim_ = nullptr;
    Particles parts_;
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
