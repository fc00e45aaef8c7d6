// common.cuh -- device-side data layout and exact-arithmetic helpers shared by every kernel.
//
// Layout (one handle = k scenes over packed index spaces):
//   particles  : scene s owns packed ids [p_begin, p_end); state arrays are in id order,
//                pos4 = (x, y, z, mass), vel4 = (u, v, w, type-as-int-bits);
//   cells      : scene s owns packed cells [c_begin, c_begin + n^3); cell (i,j,k) of the
//                scene is c_begin + (i*n + j)*n + k (z fastest, the reference's loop order);
//   faces      : scene s owns [f_begin, f_begin + 3 n^2 (n+1)): x faces ((n+1),n,n), then
//                y faces (n,(n+1),n), then z faces (n,n,(n+1)), each z fastest.
// All float arithmetic is written in the reference's expression order; the library is built
// with --fmad=false so no multiply-add is contracted, which keeps every stage bit-exact
// against the CPU restatement on identical inputs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ariel.h"

namespace ariel {

constexpr int kMaxScenes = 1024;
constexpr int kBlock = 256;

struct SceneDev {
    int n;             // cells per axis
    int n_forces;
    int n_spheres;
    int frame;         // FlipSim::m_frame (advanced by the BEGIN stage)
    float maxd;        // (float)n
    float density;     // lattice spacing in cells (m_density)
    float dt;          // m_stepsize
    float picflip;     // m_picflipratio
    float max_density; // m_max_density (Init)
    float dens_h;      // 4*density/maxd, ComputeDensity's Smooth radius (flip.cpp:724)
    float sdf0;        // 0.2*(1/density^3), CellSDF's threshold (particlegrid.cpp:88-89)
    float h;           // 1/maxd, cell width (flip.cpp:417, 573)
    float ax_h;        // 1/(n*n), ComputeAx's divisor (solver.inl:199-200)
    float resample_re; // density/maxd (flip.cpp:120)
    float pushout_re;  // 1.5*density/maxd (flip.cpp:268)
    int subcell;
    float fdt[ARIEL_MAX_FORCES][3];  // force * dt, applied in order
    float4 sphere[ARIEL_MAX_SPHERES]; // world units: centre xyz, radius
    long long p_begin, p_end;
    long long c_begin;
    long long f_begin;
    unsigned long long rng_seed;
    int resample_every;  // resample on frames divisible by this (1: every step, flip.cpp:121)
    int reseed_every;    // reseed on frames divisible by this (0: never)
    int reseed_min, reseed_max;  // particle-count bounds of the reseeding pass
    // When a kernel radius squared (in float) is a power of two, r2 / (h*h) equals
    // r2 * (1 / (h*h)) exactly, so the division can be replaced by a multiplication.
    int dens_pow2;       // dens_h * dens_h is a power of two
    float dens_inv_hh;
    int re_pow2;         // resample_re^2 is a power of two
    float re_inv_hh;
    // reciprocals of the grid's index divisors (n, n + 1, n^2, n (n + 1)) for index decoding
    double inv_n, inv_n1, inv_nn, inv_nn1;
    // static solid meshes: the scene's tree and triangles (mesh.cuh), world coordinates
    int n_meshes;
    const struct MeshNode* mesh_nodes;
    const struct MeshTri* mesh_tris;
};

// ------------------------------------------------------------------------------------------
// glm restatement: glm::min/max are ternaries (NaN and signed-zero behaviour included).
// ------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ float gmin(float x, float y) { return (y < x) ? y : x; }
__host__ __device__ __forceinline__ float gmax(float x, float y) { return (x < y) ? y : x; }

// Cell coordinate of a unit-cube position (particlegrid.cpp:156-158, flip.cpp:711-713).
__device__ __forceinline__ int cell_coord(float maxd, float x) {
    return (int)gmax(0.0f, gmin((float)(int)maxd - 1.0f, (float)(int)maxd * x));
}

// kernels.inl:25-38
__device__ __forceinline__ float sqrlength(float ax, float ay, float az, float bx, float by, float bz) {
    float a = ax - bx;
    float b = ay - by;
    float c = az - bz;
    return a * a + b * b + c * c;
}
// sqrlength(q.x, q.y, q.z, p.x, p.y, p.z) with the x and y terms as one packed pair of IEEE
// round-to-nearest operations (sm_100 f32x2 add and multiply, each lane the same bits as the
// scalar operation); `nxy` holds (-p.x, -p.y), and q.x + (-p.x) is q.x - p.x exactly.  The
// square of a difference does not depend on its sign, so it also serves (p - q) . (p - q).
__device__ __forceinline__ float sqrlength_xy2(float4 q, float2 nxy, float pz) {
    const float2 d = __fadd2_rn(make_float2(q.x, q.y), nxy);
    const float2 s = __fmul2_rn(d, d);
    const float c = q.z - pz;
    return s.x + s.y + c * c;
}
__device__ __forceinline__ float smooth_k(float r2, float h) { return gmax(1.0f - r2 / (h * h), 0.0f); }
// smooth_k with the division replaced by an exact power-of-two reciprocal when pow2 is set.
__device__ __forceinline__ float smooth_fast(float r2, float h, int pow2, float inv_hh) {
    return pow2 ? gmax(1.0f - r2 * inv_hh, 0.0f) : smooth_k(r2, h);
}
// Squared distance from x to the interval [lo, hi] along one axis.
__device__ __forceinline__ float axis_gap2(float x, float lo, float hi) {
    float d = x < lo ? lo - x : (x > hi ? x - hi : 0.0f);
    return d * d;
}
__device__ __forceinline__ float sharpen_k(float r2, float h) {
    return gmax(h * h / gmax(r2, 1.0e-5f) - 1.0f, 0.0f);
}

// glm::dot / length / normalize as used by the solid-constraint paths.
__device__ __forceinline__ float gdot3(float3 a, float3 b) {
    float tx = a.x * b.x, ty = a.y * b.y, tz = a.z * b.z;
    return (tx + ty) + tz;
}
__device__ __forceinline__ float glength3(float3 v) { return sqrtf(gdot3(v, v)); }
__device__ __forceinline__ float3 gnormalize3(float3 v) {
    float s = 1.0f / sqrtf(gdot3(v, v));
    return make_float3(v.x * s, v.y * s, v.z * s);
}
__device__ __forceinline__ float3 f3add(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 f3sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 f3mul(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 f3smul(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 f3div(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }

__device__ __forceinline__ int type_of(float4 v) { return __float_as_int(v.w); }

// ------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): replaces rand() of the resampler.
// ------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        unsigned long long p0 = (unsigned long long)0xD2511F53u * c.x;
        unsigned long long p1 = (unsigned long long)0xCD9E8D57u * c.z;
        uint4 o;
        o.x = (uint32_t)(p1 >> 32) ^ c.y ^ k0;
        o.y = (uint32_t)p1;
        o.z = (uint32_t)(p0 >> 32) ^ c.w ^ k1;
        o.w = (uint32_t)p0;
        c = o;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}
constexpr uint32_t kTagSeed = 0x53454544u;      // "SEED"
constexpr uint32_t kTagResample = 0x5245534Du;  // "RESM"
constexpr uint32_t kTagReseed = 0x52534544u;    // "RSED"

// ------------------------------------------------------------------------------------------
// Grid index decoding without integer division (a 64-bit division is a long instruction
// sequence, several per thread in the stencil kernels).  floor(x / d) for 0 <= x < 2^40 from a
// double reciprocal r of d accurate to a few ulp: x * r is then within 2^-11 of the quotient,
// so its truncation is off by at most one, which the remainder test corrects.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ long long div_r(long long x, long long d, double r) {
    long long q = (long long)((double)x * r);
    const long long rem = x - q * d;
    q += rem < 0 ? -1 : (rem >= d ? 1 : 0);
    return q;
}
// Cell (i, j, k) of local cell index c = (i n + j) n + k.
__device__ __forceinline__ void cell_ijk(const SceneDev& D, long long c, int& i, int& j, int& k) {
    const long long n = D.n, nn = n * n;
    const long long a = div_r(c, nn, D.inv_nn);
    const long long r = c - a * nn;
    const long long b = div_r(r, n, D.inv_n);
    i = (int)a;
    j = (int)b;
    k = (int)(r - b * n);
}
// Axis and (i, j, k) of local face index f: x faces (n+1) x n x n, then y faces n x (n+1) x n,
// then z faces n x n x (n+1), each block in (i, j, k) order.
__device__ __forceinline__ void face_ijk(const SceneDev& D, long long f, int& axis, int& i, int& j, int& k) {
    const long long n = D.n, n1 = n + 1, per = n * n * n1;
    axis = (f >= per ? 1 : 0) + (f >= 2 * per ? 1 : 0);
    const long long r = f - axis * per;
    const long long rowd = axis == 0 ? n * n : n1 * n;  // faces per i plane
    const double rowr = axis == 0 ? D.inv_nn : D.inv_nn1;
    const long long kd = axis == 2 ? n1 : n;            // faces per (i, j) row
    const double kr = axis == 2 ? D.inv_n1 : D.inv_n;
    const long long a = div_r(r, rowd, rowr);
    const long long r2 = r - a * rowd;
    const long long b = div_r(r2, kd, kr);
    i = (int)a;
    j = (int)b;
    k = (int)(r2 - b * kd);
}

// ------------------------------------------------------------------------------------------
// Packed index -> scene.  `pref` holds k+1 ascending begins; a block copies it to shared
// memory once and every thread binary-searches it.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ int find_scene(const long long* __restrict__ pref_s, int k, long long g) {
    int lo = 0, hi = k - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pref_s[mid] <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <int MAXK>
__device__ __forceinline__ void load_prefix(long long* dst, const long long* __restrict__ src, int k) {
    for (int i = threadIdx.x; i <= k && i < MAXK + 1; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

}  // namespace ariel
