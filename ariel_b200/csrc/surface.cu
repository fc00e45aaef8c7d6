// surface.cu -- the liquid surface of a scene for output: the reference's LevelSet(particles)
// (src/grid/levelset.cpp:101-111, OpenVDB ParticlesToLevelSet) and LevelSet::WriteObjToFile
// (levelset.cpp:113-172, OpenVDB VolumeToMesh), called by Scene::ExportParticles' OBJ branch
// (src/scene/scene.cpp:84-100).
//
// Level set: the FLUID particles as spheres of radius 0.5 cells (ParticleList::getPosRad,
// src/grid/levelset.hpp:44-57) rasterised on the integer points of the grid, padded kPad cells
// beyond each wall so that the surface closes outside the domain; a sample holds the smallest
// (distance to a particle centre - radius) over the particles within radius + kBand, else kBand.
// One thread per particle lowers the samples it reaches with an integer atomicMin on an
// order-preserving encoding of the float, so the result does not depend on the order.
// (OpenVDB's rasterizeTrails adds a tail of shrinking spheres behind each particle along its
// velocity and keeps a 3-cell band; those are not reproduced -- the zero crossing of the plain
// spheres' union is the surface here.)
//
// Mesh: surface nets at level 0, a dual method like VolumeToMesh: every grid cube whose corners
// change sign gets one vertex, the mean of the zero crossings on its sign-changing edges (in a
// fixed edge order), and every sign-changing grid edge gets a quad joining the vertices of its
// four cubes, wound so that its normal points from negative to positive.  Vertices are numbered
// in cube order and quads in edge order (axis x, y, z; samples in grid order).
#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "sim.cuh"
#include "state.cuh"

namespace ariel {
namespace {

constexpr int kPad = 2;
constexpr float kRadius = 0.5f;
constexpr float kBand = 1.5f;

__device__ __forceinline__ int f_ord(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : (i ^ 0x7FFFFFFF);
}
__device__ __forceinline__ float f_unord(int i) { return __int_as_float(i >= 0 ? i : (i ^ 0x7FFFFFFF)); }

__global__ void k_ls_fill(int* phi, long long m) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) phi[i] = f_ord(kBand);
}

__global__ void k_ls_scatter(const float4* __restrict__ pos4, const float4* __restrict__ vel4, long long n, float maxd,
                             int N, int* phi) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    if (type_of(vel4[g]) != ARIEL_FLUID) return;
    const float4 q = pos4[g];
    const float px = q.x * maxd, py = q.y * maxd, pz = q.z * maxd;
    const float R = kRadius + kBand;
    const float R2 = R * R;
    int lo[3], hi[3];
    const float pp[3] = {px, py, pz};
    for (int a = 0; a < 3; ++a) {
        lo[a] = max((int)ceilf(pp[a] - R), -kPad);
        hi[a] = min((int)floorf(pp[a] + R), N - 1 - kPad);
    }
    for (int i = lo[0]; i <= hi[0]; ++i) {
        const float dx = (float)i - px;
        for (int j = lo[1]; j <= hi[1]; ++j) {
            const float dy = (float)j - py;
            for (int k = lo[2]; k <= hi[2]; ++k) {
                const float dz = (float)k - pz;
                const float d2 = (dx * dx + dy * dy) + dz * dz;
                if (!(d2 < R2)) continue;
                const float v = sqrtf(d2) - kRadius;
                atomicMin(&phi[((long long)(i + kPad) * N + (j + kPad)) * N + (k + kPad)], f_ord(v));
            }
        }
    }
}

__global__ void k_ls_decode(int* phi, long long m) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) reinterpret_cast<float*>(phi)[i] = f_unord(phi[i]);
}

// The cube at (i, j, k) (corner samples i..i+1, ...): its vertex, if its corners change sign.
__device__ __forceinline__ bool cube_vertex(const float* __restrict__ phi, int N, int i, int j, int k, float3* out) {
    float c[8];
    int inside = 0;
    for (int b = 0; b < 8; ++b) {
        c[b] = phi[((long long)(i + (b & 1)) * N + (j + ((b >> 1) & 1))) * N + (k + ((b >> 2) & 1))];
        inside += c[b] < 0.0f ? 1 : 0;
    }
    if (inside == 0 || inside == 8) return false;
    if (!out) return true;
    // edges as corner pairs: 4 along x, 4 along y, 4 along z
    const int E[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
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
    *out = make_float3(sx / fc - (float)kPad, sy / fc - (float)kPad, sz / fc - (float)kPad);
    return true;
}

__global__ void k_cube_flags(const float* __restrict__ phi, int N, uint32_t* flag) {
    const int M = N - 1;
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)M * M * M) return;
    const int i = (int)(c / ((long long)M * M)), j = (int)((c / M) % M), k = (int)(c % M);
    flag[c] = cube_vertex(phi, N, i, j, k, nullptr) ? 1u : 0u;
}

__global__ void k_cube_vertices(const float* __restrict__ phi, int N, const uint32_t* __restrict__ vidx,
                                float3* __restrict__ verts) {
    const int M = N - 1;
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)M * M * M) return;
    if (vidx[c + 1] == vidx[c]) return;
    const int i = (int)(c / ((long long)M * M)), j = (int)((c / M) % M), k = (int)(c % M);
    float3 v;
    cube_vertex(phi, N, i, j, k, &v);
    verts[vidx[c]] = v;
}

// Edge e = axis * N^3 + sample: from the sample to its +axis neighbour.  A quad when the two
// ends change sign and all four cubes around the edge exist.
__device__ __forceinline__ bool edge_quad(const float* __restrict__ phi, int N, long long e, int cube[4], bool* flip) {
    const long long N3 = (long long)N * N * N;
    const int axis = (int)(e / N3);
    const long long s = e % N3;
    const int i = (int)(s / ((long long)N * N)), j = (int)((s / N) % N), k = (int)(s % N);
    const int p[3] = {i, j, k};
    if (p[axis] >= N - 1) return false;
    const int u = (axis + 1) % 3, w = (axis + 2) % 3;  // the plane of the four cubes, (u, w) right-handed
    if (p[u] < 1 || p[u] > N - 2 || p[w] < 1 || p[w] > N - 2) return false;
    int q[3] = {i, j, k};
    q[axis] += 1;
    const float a = phi[s];
    const float b = phi[((long long)q[0] * N + q[1]) * N + q[2]];
    if ((a < 0.0f) == (b < 0.0f)) return false;
    *flip = !(a < 0.0f);
    const int M = N - 1;
    const int du[4] = {-1, 0, 0, -1}, dw[4] = {-1, -1, 0, 0};
    for (int c = 0; c < 4; ++c) {
        int r[3] = {i, j, k};
        r[u] += du[c];
        r[w] += dw[c];
        cube[c] = (int)(((long long)r[0] * M + r[1]) * M + r[2]);
    }
    return true;
}

__global__ void k_edge_flags(const float* __restrict__ phi, int N, uint32_t* flag) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3ll * N * N * N) return;
    int cube[4];
    bool flip;
    flag[e] = edge_quad(phi, N, e, cube, &flip) ? 1u : 0u;
}

__global__ void k_edge_quads(const float* __restrict__ phi, int N, const uint32_t* __restrict__ qidx,
                             const uint32_t* __restrict__ vidx, int4* __restrict__ quads) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3ll * N * N * N) return;
    if (qidx[e + 1] == qidx[e]) return;
    int cube[4];
    bool flip;
    edge_quad(phi, N, e, cube, &flip);
    int v[4];
    for (int c = 0; c < 4; ++c) v[c] = (int)vidx[cube[c]];
    quads[qidx[e]] = flip ? make_int4(v[0], v[3], v[2], v[1]) : make_int4(v[0], v[1], v[2], v[3]);
}

struct DevTmp {
    std::vector<void*> ptrs;
    ~DevTmp() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(1, count) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(q);
        *p = (T*)q;
        return e;
    }
};

// The scene's level set into phi (N^3 samples, N = n + 1 + 2 kPad) on the handle's stream.
cudaError_t level_set(ariel_sim* s, int scene, float* phi, int N) {
    const long long m = (long long)N * N * N;
    cudaStream_t st = s->stream;
    int* pi = reinterpret_cast<int*>(phi);
    k_ls_fill<<<grid_for(m), kBlock, 0, st>>>(pi, m);
    const long long b = s->ppref[scene], n = s->ppref[scene + 1] - b;
    if (n > 0) k_ls_scatter<<<grid_for(n), kBlock, 0, st>>>(s->S.pos4 + b, s->S.vel4 + b, n, s->sh[scene].maxd, N, pi);
    k_ls_decode<<<grid_for(m), kBlock, 0, st>>>(pi, m);
    count_launch(n > 0 ? 3 : 2);
    return cudaGetLastError();
}

}  // namespace
}  // namespace ariel

using namespace ariel;
using namespace ariel::hostimpl;

extern "C" {

ariel_status ariel_get_level_set(ariel_sim* s, int32_t scene, float* phi, int64_t nbytes) {
    if (!s || !phi || scene < 0 || scene >= s->k) return ARIEL_ERR_INVALID_ARG;
    if (!s->inited) return ARIEL_ERR_STATE;
    const int N = s->descs[scene].dim + 1 + 2 * kPad;
    const long long m = (long long)N * N * N;
    if (nbytes != m * (long long)sizeof(float)) return ARIEL_ERR_INVALID_ARG;
    DevTmp T;
    float* d_phi = nullptr;
    cudaError_t e = T.alloc(&d_phi, m);
    if (e == cudaSuccess) e = level_set(s, scene, d_phi, N);
    if (e == cudaSuccess) e = copy_sync(s->stream, phi, d_phi, m * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return map_cuda_error(e, "ariel_get_level_set");
    }
    return ARIEL_OK;
}

ariel_status ariel_surface_mesh(ariel_sim* s, int32_t scene, float* vertices, int64_t max_vertices, int32_t* quads,
                                int64_t max_quads, int64_t* n_vertices, int64_t* n_quads) {
    if (!s || !n_vertices || !n_quads || scene < 0 || scene >= s->k || max_vertices < 0 || max_quads < 0)
        return ARIEL_ERR_INVALID_ARG;
    if (!s->inited) return ARIEL_ERR_STATE;
    const int N = s->descs[scene].dim + 1 + 2 * kPad;
    const long long m = (long long)N * N * N, M = (long long)(N - 1) * (N - 1) * (N - 1), ne = 3 * m;
    DevTmp T;
    float* d_phi = nullptr;
    uint32_t *d_cf = nullptr, *d_vidx = nullptr, *d_ef = nullptr, *d_qidx = nullptr;
    void* d_tmp = nullptr;
    float3* d_v = nullptr;
    int4* d_q = nullptr;
    cudaStream_t st = s->stream;
    uint32_t nv = 0, nq = 0;
    cudaError_t e = T.alloc(&d_phi, m);
    if (e == cudaSuccess) e = T.alloc(&d_cf, M);
    if (e == cudaSuccess) e = T.alloc(&d_vidx, M + 1);
    if (e == cudaSuccess) e = T.alloc(&d_ef, ne);
    if (e == cudaSuccess) e = T.alloc(&d_qidx, ne + 1);
    if (e == cudaSuccess) e = T.alloc((unsigned char**)&d_tmp, scan_tmp_bytes(std::max(M, ne)));
    if (e == cudaSuccess) e = level_set(s, scene, d_phi, N);
    if (e == cudaSuccess) {
        k_cube_flags<<<grid_for(M), kBlock, 0, st>>>(d_phi, N, d_cf);
        e = launch_scan_u32(d_cf, d_vidx, M, d_tmp, st);
    }
    if (e == cudaSuccess) {
        k_edge_flags<<<grid_for(ne), kBlock, 0, st>>>(d_phi, N, d_ef);
        e = launch_scan_u32(d_ef, d_qidx, ne, d_tmp, st);
    }
    if (e == cudaSuccess) e = copy_sync(st, &nv, d_vidx + M, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = copy_sync(st, &nq, d_qidx + ne, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = T.alloc(&d_v, nv);
    if (e == cudaSuccess) e = T.alloc(&d_q, nq);
    if (e == cudaSuccess) {
        k_cube_vertices<<<grid_for(M), kBlock, 0, st>>>(d_phi, N, d_vidx, d_v);
        k_edge_quads<<<grid_for(ne), kBlock, 0, st>>>(d_phi, N, d_qidx, d_vidx, d_q);
        count_launch(4);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && vertices && (int64_t)nv <= max_vertices)
        e = copy_sync(st, vertices, d_v, (size_t)nv * sizeof(float3), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && quads && (int64_t)nq <= max_quads)
        e = copy_sync(st, quads, d_q, (size_t)nq * sizeof(int4), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return map_cuda_error(e, "ariel_surface_mesh");
    }
    *n_vertices = nv;
    *n_quads = nq;
    if ((vertices && (int64_t)nv > max_vertices) || (quads && (int64_t)nq > max_quads)) return ARIEL_ERR_INVALID_ARG;
    return ARIEL_OK;
}

ariel_status ariel_export_surface(ariel_sim* s, int32_t scene, const char* path, int32_t frame) {
    if (!s || !path || scene < 0 || scene >= s->k || frame < 0) return ARIEL_ERR_INVALID_ARG;
    std::string name(path);
    const std::string ext = ".obj";
    if (name.size() <= ext.size() || name.compare(name.size() - ext.size(), ext.size(), ext) != 0)
        return ARIEL_ERR_INVALID_ARG;
    char fr[16];
    std::snprintf(fr, sizeof(fr), ".%04d", frame);
    const std::string out = name.substr(0, name.size() - ext.size()) + fr + ext;
    int64_t nv = 0, nq = 0;
    ariel_status st = ariel_surface_mesh(s, scene, nullptr, 0, nullptr, 0, &nv, &nq);
    if (st != ARIEL_OK) return st;
    std::vector<float> v(3 * (size_t)nv);
    std::vector<int32_t> q(4 * (size_t)nq);
    st = ariel_surface_mesh(s, scene, v.data(), nv, q.data(), nq, &nv, &nq);
    if (st != ARIEL_OK) return st;
    FILE* f = std::fopen(out.c_str(), "w");
    if (!f) return ARIEL_ERR_INVALID_ARG;
    for (int64_t i = 0; i < nv; ++i) std::fprintf(f, "v %.9g %.9g %.9g\n", v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    for (int64_t i = 0; i < nq; ++i)
        std::fprintf(f, "f %d %d %d %d\n", q[4 * i] + 1, q[4 * i + 1] + 1, q[4 * i + 2] + 1, q[4 * i + 3] + 1);
    return std::fclose(f) == 0 ? ARIEL_OK : ARIEL_ERR_INVALID_ARG;
}

}  // extern "C"
