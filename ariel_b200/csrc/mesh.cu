// mesh.cu -- host side of the static solid meshes: the registry behind ariel_mesh_create /
// ariel_mesh_destroy, and the per-scene world-space bounding volume hierarchy that the kernels
// and the host seeding traverse (mesh.cuh).  The reference builds one BVH per OBJ mesh in
// object space and transforms each ray (src/spatial/bvh.inl:110-260, src/geom/mesh.cpp:111-121);
// here every mesh of a scene is placed in world (grid) coordinates once and all of a scene's
// triangles share one tree, since the meshes are static.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>

#include "sim.cuh"

namespace {

struct MeshObj {
    std::vector<float> vertices;  // object space xyz
    std::vector<int32_t> triangles;
    float translate[3];
    float scale;
};

std::mutex g_mesh_mutex;
std::map<int32_t, std::shared_ptr<const MeshObj>> g_meshes;
int32_t g_next_mesh = 1;

std::shared_ptr<const MeshObj> find_mesh(int32_t id) {
    std::lock_guard<std::mutex> lock(g_mesh_mutex);
    auto it = g_meshes.find(id);
    return it == g_meshes.end() ? nullptr : it->second;
}

// Nodes of the tree over t triangles: halves until at most kMeshLeaf remain (memoised: only two
// distinct sizes occur per level).
long long node_count(long long t, std::map<long long, long long>& memo) {
    if (t <= ariel::kMeshLeaf) return 1;
    auto it = memo.find(t);
    if (it != memo.end()) return it->second;
    const long long v = 1 + node_count(t / 2, memo) + node_count(t - t / 2, memo);
    memo[t] = v;
    return v;
}

struct Builder {
    std::vector<ariel::MeshTri>& tris;
    std::vector<ariel::MeshNode>& nodes;
    std::vector<float3> cen;
    std::vector<int> order;

    // The node for triangles order[b, e); returns its index.  Children are split at the middle
    // of the triangles sorted by centroid along the widest axis (ties by index), so the shape of
    // the tree depends only on the triangle count.
    int build(int b, int e) {
        const int id = (int)nodes.size();
        nodes.push_back(ariel::MeshNode{});
        float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
        float clo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, chi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
        for (int i = b; i < e; ++i) {
            const ariel::MeshTri& T = tris[order[i]];
            const float4 vs[3] = {T.v0, T.v1, T.v2};
            for (const float4& v : vs) {
                const float c[3] = {v.x, v.y, v.z};
                for (int a = 0; a < 3; ++a) {
                    lo[a] = std::min(lo[a], c[a]);
                    hi[a] = std::max(hi[a], c[a]);
                }
            }
            const float cc[3] = {cen[order[i]].x, cen[order[i]].y, cen[order[i]].z};
            for (int a = 0; a < 3; ++a) {
                clo[a] = std::min(clo[a], cc[a]);
                chi[a] = std::max(chi[a], cc[a]);
            }
        }
        ariel::MeshNode N;
        for (int a = 0; a < 3; ++a) {
            // widened so that no hit the triangle test reports, nor any rounding of the traversal
            // tests, falls outside
            const float m = std::max(std::fabs(lo[a]), std::fabs(hi[a]));
            const float eps = 1.0e-3f + 1.0e-5f * m;
            N.lo[a] = lo[a] - eps;
            N.hi[a] = hi[a] + eps;
        }
        if (e - b <= ariel::kMeshLeaf) {
            N.a = b;
            N.b = -(e - b);
            nodes[id] = N;
            return id;
        }
        int ax = 0;
        for (int a = 1; a < 3; ++a)
            if (chi[a] - clo[a] > chi[ax] - clo[ax]) ax = a;
        auto key = [&](int t) { return ax == 0 ? cen[t].x : (ax == 1 ? cen[t].y : cen[t].z); };
        std::stable_sort(order.begin() + b, order.begin() + e, [&](int x, int y) {
            const float kx = key(x), ky = key(y);
            return kx < ky || (kx == ky && x < y);
        });
        const int mid = b + (e - b) / 2;
        N.a = build(b, mid);
        N.b = build(mid, e);
        nodes[id] = N;
        return id;
    }
};

}  // namespace

namespace ariel {
namespace hostimpl {

bool meshes_valid(const AsimSceneDesc& d) {
    if (d.n_mesh < 0 || d.n_mesh > ARIEL_MAX_MESHES) return false;
    for (int i = 0; i < d.n_mesh; ++i)
        if (!find_mesh(d.mesh[i])) return false;
    return true;
}

void mesh_counts(const AsimSceneDesc& d, long long& nodes, long long& tris) {
    nodes = tris = 0;
    for (int i = 0; i < d.n_mesh && i < ARIEL_MAX_MESHES; ++i) {
        auto m = find_mesh(d.mesh[i]);
        if (m) tris += (long long)m->triangles.size() / 3;
    }
    std::map<long long, long long> memo;
    if (tris > 0) nodes = node_count(tris, memo);
}

ariel_status scene_meshes(const AsimSceneDesc& d, std::shared_ptr<SceneMeshes>& out) {
    out = std::make_shared<SceneMeshes>();
    if (d.n_mesh <= 0) return ARIEL_OK;
    const float maxd = (float)d.dim;
    SceneMeshes& M = *out;
    int key = 0;  // a triangle's index across the scene's meshes, in mesh order
    for (int i = 0; i < d.n_mesh; ++i) {
        auto m = find_mesh(d.mesh[i]);
        if (!m) return ARIEL_ERR_INVALID_ARG;
        const std::vector<float>& v = m->vertices;
        auto world = [&](int vi, int a) { return (v[3 * vi + a] * m->scale + m->translate[a]) * maxd; };
        float3 lo = make_float3(3.0e38f, 3.0e38f, 3.0e38f), hi = make_float3(-3.0e38f, -3.0e38f, -3.0e38f);
        const int nt = (int)m->triangles.size() / 3;
        for (int t = 0; t < nt; ++t) {
            MeshTri T;
            float4* vs[3] = {&T.v0, &T.v1, &T.v2};
            for (int c = 0; c < 3; ++c) {
                const int vi = m->triangles[3 * t + c];
                *vs[c] = make_float4(world(vi, 0), world(vi, 1), world(vi, 2), 0.0f);
                lo.x = std::min(lo.x, vs[c]->x);
                lo.y = std::min(lo.y, vs[c]->y);
                lo.z = std::min(lo.z, vs[c]->z);
                hi.x = std::max(hi.x, vs[c]->x);
                hi.y = std::max(hi.y, vs[c]->y);
                hi.z = std::max(hi.z, vs[c]->z);
            }
            const int mesh = i, k = key++;
            std::memcpy(&T.v0.w, &mesh, 4);
            std::memcpy(&T.v1.w, &k, 4);
            M.tris.push_back(T);
        }
        M.lo.push_back(lo);
        M.hi.push_back(hi);
    }
    if (M.tris.empty()) return ARIEL_OK;
    std::vector<MeshTri> src = M.tris;
    Builder B{src, M.nodes, {}, {}};
    B.cen.resize(src.size());
    B.order.resize(src.size());
    for (size_t t = 0; t < src.size(); ++t) {
        const MeshTri& T = src[t];
        B.cen[t] = make_float3((T.v0.x + T.v1.x + T.v2.x) / 3.0f, (T.v0.y + T.v1.y + T.v2.y) / 3.0f,
                               (T.v0.z + T.v1.z + T.v2.z) / 3.0f);
        B.order[t] = (int)t;
    }
    M.nodes.reserve(2 * src.size());
    B.build(0, (int)src.size());
    // triangles in leaf order, so that a leaf's triangles are consecutive
    for (size_t t = 0; t < src.size(); ++t) M.tris[t] = src[B.order[t]];
    return ARIEL_OK;
}

}  // namespace hostimpl
}  // namespace ariel

extern "C" {

ariel_status ariel_mesh_create(const float* vertices, int32_t n_vertices, const int32_t* triangles,
                               int32_t n_triangles, const float* translate, float scale, int32_t* mesh_id) {
    if (!vertices || !triangles || !translate || !mesh_id || n_vertices < 3 || n_triangles < 1 ||
        n_triangles > (1 << 24) || !(scale > 0.0f) || !std::isfinite(scale))
        return ARIEL_ERR_INVALID_ARG;
    auto m = std::make_shared<MeshObj>();
    m->vertices.assign(vertices, vertices + 3 * (size_t)n_vertices);
    m->triangles.assign(triangles, triangles + 3 * (size_t)n_triangles);
    for (float x : m->vertices)
        if (!std::isfinite(x)) return ARIEL_ERR_NAN;
    for (int32_t t : m->triangles)
        if (t < 0 || t >= n_vertices) return ARIEL_ERR_INVALID_ARG;
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(translate[a])) return ARIEL_ERR_NAN;
        m->translate[a] = translate[a];
    }
    m->scale = scale;
    std::lock_guard<std::mutex> lock(g_mesh_mutex);
    const int32_t id = g_next_mesh++;
    g_meshes[id] = m;
    *mesh_id = id;
    return ARIEL_OK;
}

ariel_status ariel_mesh_destroy(int32_t mesh_id) {
    std::lock_guard<std::mutex> lock(g_mesh_mutex);
    return g_meshes.erase(mesh_id) ? ARIEL_OK : ARIEL_ERR_INVALID_ARG;
}

ariel_status ariel_mesh_info(int32_t mesh_id, int32_t* n_vertices, int32_t* n_triangles, float* translate,
                             float* scale) {
    std::lock_guard<std::mutex> lock(g_mesh_mutex);
    auto it = g_meshes.find(mesh_id);
    if (it == g_meshes.end()) return ARIEL_ERR_INVALID_ARG;
    const MeshObj& m = *it->second;
    if (n_vertices) *n_vertices = (int32_t)(m.vertices.size() / 3);
    if (n_triangles) *n_triangles = (int32_t)(m.triangles.size() / 3);
    if (translate)
        for (int a = 0; a < 3; ++a) translate[a] = m.translate[a];
    if (scale) *scale = m.scale;
    return ARIEL_OK;
}

}  // extern "C"
