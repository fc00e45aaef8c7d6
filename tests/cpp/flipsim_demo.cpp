// Host program driving the B200 FLIP step through the
// C++ FlipSim wrapper.  Exit codes: 0 ran on a GPU, 3 the library reported no sm_100 device.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ariel_flipsim.hpp"

int main(int argc, char** argv) {
    int n = argc > 1 ? std::atoi(argv[1]) : 16;
    int steps = argc > 2 ? std::atoi(argv[2]) : 2;
    AsimSceneDesc scene;
    ariel_scene_dambreak(&scene, n);
    try {
        ariel::FlipSim sim(n, 0.5f, 1.0f / 240.0f, scene, false);
        sim.Init();
        for (int i = 0; i < steps; ++i) sim.Step(false, false, false);
        const ariel::Particles& p = sim.GetParticles();
        double vy = 0;
        for (size_t i = 0; i < p.size(); ++i) vy += p.vel[3 * i + 1];
        std::printf("frame %d particles %zu mean vy %.6f dims %d\n", sim.m_frame, p.size(), vy / p.size(),
                    sim.GetDimensions()[0]);
        // the same scene through the request server, beside a second one, gives the same particles
        ariel::Server server;
        AsimSceneDesc other;
        ariel_scene_dambreak(&other, n + 4);
        const int64_t a = server.Submit(scene, steps);
        const int64_t b = server.Submit(other, steps + 1);
        server.Drain();
        std::vector<float> pos, vel;
        server.Fetch(a, pos, vel);
        bool same = pos.size() == p.pos.size();
        for (size_t i = 0; same && i < pos.size(); ++i) same = pos[i] == p.pos[i] && vel[i] == p.vel[i];
        std::printf("served %s, second request %d steps\n", same ? "identical" : "different",
                    server.Poll(b).steps_done);
        if (!same) return 1;
    } catch (const ariel::Error& e) {
        std::printf("error %d: %s\n", (int)e.code(), e.what());
        return e.code() == ARIEL_ERR_NO_DEVICE ? 3 : 1;
    }
    return 0;
}
