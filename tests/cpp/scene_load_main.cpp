// A C++ host reading a reference scene file through the library's loader (ariel::LoadScene),
// as a host without the reference's SceneLoader would: prints what the description holds, then
// shows a refused scene's reason.  Needs no GPU.
#include <cstdio>

#include "ariel_flipsim.hpp"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    AsimSceneInfo info;
    const AsimSceneDesc d = ariel::LoadScene(argv[1], &info);
    std::printf("dim %d density %.3f step %.6f partio %s\n", d.dim, info.density, info.step_size, info.partio_output);
    std::printf("liquids %d box %.3f %.3f %.3f solids %d sphere %.4f %.4f %.4f r %.4f meshes %d forces %d\n",
                d.n_liquid, d.liquid[0].hi[0], d.liquid[0].hi[1], d.liquid[0].hi[2], d.n_solid, d.solid[0].center[0],
                d.solid[0].center[1], d.solid[0].center[2], d.solid[0].radius, d.n_mesh, d.n_forces);
    for (int i = 0; i < d.n_mesh; ++i) {
        int32_t nv = 0, nt = 0;
        float t[3], s = 0.0f;
        ariel::check(ariel_mesh_info(d.mesh[i], &nv, &nt, t, &s), "ariel_mesh_info");
        std::printf("mesh %d vertices %d triangles %d scale %.6f\n", i, nv, nt, s);
        ariel::check(ariel_mesh_destroy(d.mesh[i]), "ariel_mesh_destroy");
    }
    try {
        ariel::LoadScene(argv[2]);
        std::printf("refused: no\n");
    } catch (const ariel::Error& e) {
        std::printf("refused: %s\n", e.what());
    }
    return 0;
}
