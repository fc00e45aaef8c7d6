// Host code shaped like the reference's src/main.cpp:50-54 and Viewer::SimLoopThread
// (src/viewer/viewer.cpp:66-87), with the two edits a maintainer makes to bind the B200 library:
// `fluidCore::FlipSim` becomes `ariel::FlipSim` (same constructor arguments) and the particles
// the loop reads become the library's host copy.  Built against the stand-in Scene of
// reference_scene_mock.hpp.  The loop runs `steps` times instead of forever.
// Exit codes: 0 stepped on a GPU, 3 the library reported no sm_100 device, 1 any other failure.
#include <cstdio>
#include <cstdlib>

#include "reference_scene_mock.hpp"
#include "ariel_flipsim.hpp"

int main(int argc, char** argv) {
    const int n = argc > 1 ? std::atoi(argv[1]) : 16;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 3;
    const float fn = (float)n;
    sceneCore::Scene* scene = new sceneCore::Scene();
    scene->AddLiquidBox(glm::vec3(0.0f), glm::vec3(0.35f * fn, 0.5f * fn, fn), glm::vec3(0.0f));
    scene->AddSolid(new geomCore::SphereGen(glm::vec3(0.6f * fn, 0.3f * fn, 0.5f * fn), 0.15f * fn));
    scene->AddExternalForce(glm::vec3(0.0f, -9.8f, 0.0f));
    sceneCore::SceneLoader* sloader = new sceneCore::SceneLoader(scene, glm::vec3(fn), 0.5f, 1.0f / 240.0f);
    const bool verbose = false;
    bool m_dumpVDB = false, m_dumpOBJ = false, m_dumpPARTIO = true;

    const AsimSceneDesc d = ariel::SceneFrom(*scene, n, 0.5f, 1.0f / 240.0f);
    std::printf("SceneFrom: liquids %d solids %d forces %d box %.3f %.3f %.3f sphere %.4f %.4f %.4f r %.4f\n",
                d.n_liquid, d.n_solid, d.n_forces, d.liquid[0].hi[0], d.liquid[0].hi[1], d.liquid[0].hi[2],
                d.solid[0].center[0], d.solid[0].center[1], d.solid[0].center[2], d.solid[0].radius);
    try {
        // src/main.cpp:50-54, with the namespace changed
        ariel::FlipSim* f = new ariel::FlipSim(sloader->GetDimensions(), sloader->GetDensity(),
                                               sloader->GetStepsize(), sloader->GetScene(),
                                               verbose);
        ariel::FlipSim* m_sim = f;
        const ariel::Particles* m_particles = nullptr;
        // Viewer::SimLoopThread (src/viewer/viewer.cpp:66-87)
        if (m_sim->m_frame == 0) {
            m_sim->Init();
            m_particles = &m_sim->GetParticles();
        }
        const size_t seeded = m_particles->size();
        for (int s = 0; s < steps; ++s) {
            m_sim->Step(m_dumpVDB, m_dumpOBJ, m_dumpPARTIO);
            m_particles = &m_sim->GetParticles();
        }
        int fluid = 0;
        for (size_t i = 0; i < m_particles->size(); ++i) fluid += m_particles->type[i] == FLUID;
        std::printf("frame %d particles %zu (seeded %zu) fluid %d exports %d last export frame %d fluid %d flags %d\n",
                    m_sim->m_frame, m_particles->size(), seeded, fluid, scene->m_exports, scene->m_lastExportFrame,
                    scene->m_lastExportFluid, scene->m_lastExportFlags);
        const bool ok = scene->m_exports == steps && scene->m_lastExportFrame == steps &&
                        scene->m_lastExportFluid == fluid && scene->m_lastExportFlags == 1 && seeded > 0;
        delete f;
        if (!ok) return 1;
    } catch (const ariel::Error& e) {
        std::printf("error %d: %s\n", (int)e.code(), e.what());
        return e.code() == ARIEL_ERR_NO_DEVICE ? 3 : 1;
    }
    delete sloader;
    delete scene;
    return 0;
}
