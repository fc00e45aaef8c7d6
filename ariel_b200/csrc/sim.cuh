// sim.cuh -- the simulation handle behind the C ABI and the host-side helpers that the step
// loop (host.cu) and the request server (server.cu) share.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "mesh.cuh"
#include "pcg.cuh"

namespace ariel {

// Named NVTX range for profilers (a no-op unless a tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

struct DeviceBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool keep = false;    // persistent state: survives a re-layout until the handle is deleted
    bool pooled = false;  // from the handle's stream-ordered memory pool
};

// One scene's static solid meshes in world (grid) coordinates behind one tree (mesh.cu), and
// each mesh's world bounding box (the seeding lattice's range).
struct SceneMeshes {
    std::vector<MeshNode> nodes;
    std::vector<MeshTri> tris;
    std::vector<float3> lo, hi;
};

// Host copy of one scene's particles (id order) used while (re)building packed state.
struct HostParticles {
    std::vector<float4> pos4;  // x y z mass
    std::vector<float4> vel4;  // u v w type-bits
    // The scene's SOLID particles binned by scene-local cell, id order inside a cell, and the
    // cell -> first solid offsets (n^3 + 1 entries; empty when the scene has none).
    std::vector<float4> solid_pos;
    std::vector<uint32_t> solid_start;
    bool binned = false;
};

// One scene's particles and solid bins already in device memory (uploaded ahead of a
// re-layout by the request server); solid_start is scene-local (n^3 + 1 entries) or null.
struct DeviceParticles {
    bool valid = false;
    float4* pos4 = nullptr;
    float4* vel4 = nullptr;
    float4* solid_pos = nullptr;
    uint32_t* solid_start = nullptr;
    long long np = 0, ns = 0;
};

inline float4 pack_vel(float u, float v, float w, int type) {
    float4 r;
    r.x = u;
    r.y = v;
    r.z = w;
    int t = type;
    std::memcpy(&r.w, &t, 4);
    return r;
}
inline int type_bits(const float4& v) {
    int t;
    std::memcpy(&t, &v.w, 4);
    return t;
}

constexpr int kEvSolveKernel = ARIEL_STAGE_COUNT + 1;
constexpr int kEvCount = ARIEL_STAGE_COUNT + 2;

}  // namespace ariel

struct ariel_sim {
    int device = 0;
    int k = 0;
    std::vector<AsimSceneDesc> descs;
    AsimParams prm{};
    std::vector<ariel::SceneDev> sh;  // host mirror of the scene table
    std::vector<std::shared_ptr<ariel::SceneMeshes>> meshes;  // per scene (empty without meshes)
    ariel::MeshNode* d_mesh_nodes = nullptr;
    ariel::MeshTri* d_mesh_tris = nullptr;
    std::vector<long long> ppref, cpref, fpref, spref;
    long long np = 0, nc = 0, nf = 0;
    bool any_solid = false;
    bool inited = false;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    cudaMemPool_t pool = nullptr;  // set: every buffer comes from this stream-ordered pool
    std::vector<ariel::DeviceBuf> bufs;
    // device pointers
    ariel::SceneDev* d_scenes = nullptr;
    long long *d_ppref = nullptr, *d_cpref = nullptr, *d_fpref = nullptr;
    ariel::DevState S{};
    ariel::PcgArgs PA{};
    void* scan_tmp = nullptr;
    uint32_t *flpred = nullptr, *flscan = nullptr;
    float* d_dens_id = nullptr;
    int pcg_blocks = 0;
    int mode = ariel::kRef32;
    // graphs of one whole step: [0] plain, [1],[2] with the two stage-event sets
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
    bool graph_tried[3] = {false, false, false};
    long long graph_kernels[3] = {0, 0, 0};
    // timing: two event sets (stage boundaries + solve-kernel start), used alternately so that
    // one step's events are read while the next step runs
    cudaEvent_t ev[2][ariel::kEvCount] = {};
    bool ev_pending[2] = {false, false};
    int ev_slot = 0;
    double acc_stage[ARIEL_STAGE_COUNT] = {};
    double acc_solve_kernel = 0;
    std::vector<double> step_hist;
    cudaEvent_t tb = nullptr, te = nullptr;
    double stage_ms[ARIEL_STAGE_COUNT] = {};
    double step_ms = 0;
    float* d_stage = nullptr;  // xyz staging for host-buffer particle I/O
    int last_status = ARIEL_OK;
    std::vector<int64_t> frames;
    double graph_ms = 0;  // host time spent capturing and instantiating step graphs
};

namespace ariel {
namespace hostimpl {

ariel_status map_cuda_error(cudaError_t e, const char* what = "");
cudaError_t copy_sync(cudaStream_t st, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind);

ariel_status validate(const AsimSceneDesc& d);
SceneDev make_scene(const AsimSceneDesc& d, const AsimParams& p);
// Scene::GenerateParticles for one scene, then bin_solids.
void generate_particles(const AsimSceneDesc& d, HostParticles& out);
// Solid meshes (mesh.cu): every id of d registered; node and triangle counts of d's tree; the
// tree itself.
bool meshes_valid(const AsimSceneDesc& d);
void mesh_counts(const AsimSceneDesc& d, long long& nodes, long long& tris);
ariel_status scene_meshes(const AsimSceneDesc& d, std::shared_ptr<SceneMeshes>& out);
void bin_solids(const AsimSceneDesc& d, HostParticles& hp);

// A handle with its stream and events but no device state.  `stream`/`pool` may be null (own
// stream, plain cudaMalloc).
ariel_status new_sim(const AsimSceneDesc* descs, int k, const AsimParams& prm, cudaStream_t stream,
                     cudaMemPool_t pool, ariel_sim** out);
void delete_sim(ariel_sim* s);

// (Re)allocates every buffer for s->descs and uploads the particles.  With `src`, scene i for
// which (*src_idx)[i] >= 0 takes its particles, pressure warm start, solid bins and solver
// record from scene (*src_idx)[i] of `src` by device copies instead of from hp[i].
// With `staged`, scene i whose (*staged)[i].valid takes its particles and solid bins from
// there by device copies.
ariel_status build_state(ariel_sim* s, std::vector<HostParticles>& hp, const ariel_sim* src = nullptr,
                         const std::vector<int>* src_idx = nullptr,
                         const std::vector<DeviceParticles>* staged = nullptr);
// Device bytes build_state allocates for these scenes with these particle/solid counts.
long long state_bytes(const std::vector<AsimSceneDesc>& descs, const std::vector<long long>& particles,
                      const std::vector<long long>& solids, const AsimParams& prm);
// Frees everything but the persistent buffers (particles, pressure, solid bins, scene and
// solver records), so that a re-layout holds at most those twice.
void free_scratch(ariel_sim* s);
// m_max_density of every scene (flip.cpp:42-70), into the device table and the host mirror.
ariel_status compute_max_density(ariel_sim* s);
// Reads the device scene table (frame counters, normalisers) into the host mirror.
ariel_status refresh_scene_table(ariel_sim* s);
// Sort, initial densities and flags after new particles (FlipSim::Init's state).
ariel_status sort_and_classify_init(ariel_sim* s);
// One step queued on the handle's stream (graph replay when enabled); with timing on, the
// other event set's step is collected first.  Does not wait for the step.
ariel_status step_async(ariel_sim* s);
// Collects every pending timing event set (waits for the steps that recorded them).
ariel_status collect_pending(ariel_sim* s);
ariel_status check_device_error(ariel_sim* s);

}  // namespace hostimpl
}  // namespace ariel
