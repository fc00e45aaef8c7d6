// mesh.cuh -- static solid meshes: triangle sets in world (grid) coordinates behind a bounding
// volume hierarchy, with the three queries the FLIP step makes of its solid geometry:
//   inside   -- Scene::CheckPointInsideSolidGeom (src/scene/scene.cpp:382-402): a ray from the
//               point along +z, a solid contains the point when the ray hits it an odd number
//               of times (HitCountTraverseAccumulator, src/spatial/spatial.cpp:61-76);
//   nearest  -- Scene::IntersectSolidGeoms (scene.cpp:425-434): the nearest hit of a ray, with
//               the point and a normal;
//   closest  -- LevelSet::ProjectPointsToSurface (src/grid/levelset.cpp:175-193): the closest
//               point of the surface.  The reference asks an OpenVDB level set; here the exact
//               closest point of the triangles is used.
// The ray-triangle test restates Obj::RayTriangleTest (src/geom/obj/obj.cpp:354-398) in the
// same float expressions (glm::cross and glm::dot as glm writes them); the hit normal is the
// triangle's geometric normal (the reference interpolates the OBJ's vertex normals), which
// enters the step only through the reflection 2 (d.n) n - d, the same for n and -n.
//
// Results do not depend on the tree: a hit is any triangle the test reports (the boxes are
// widened so that the traversal never skips one), hit counts are per mesh, and ties between
// triangles go to the lower triangle key (its index in mesh and file order), so a brute-force loop over the triangles (the CPU
// oracle's) gives the same bits.  Everything here compiles for host and device: the host seeds
// solid particles with the same inside test.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

namespace ariel {

constexpr int kMeshLeaf = 4;     // triangles per leaf at most
constexpr int kMeshStack = 64;   // traversal stack (the tree's depth is log2 of its leaves)

// 32 bytes.  Internal node: children a and b.  Leaf: triangles [a, a - b) (b = -count).
struct MeshNode {
    float lo[3];
    int a;
    float hi[3];
    int b;
};
// 48 bytes: vertices in world (grid) coordinates; v0.w holds the mesh index and v1.w the
// triangle's index across the scene's meshes (int bits).
struct MeshTri {
    float4 v0, v1, v2;
};

__host__ __device__ __forceinline__ float3 m3(float4 v) { return make_float3(v.x, v.y, v.z); }
__host__ __device__ __forceinline__ float3 msub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ float3 madd(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ float3 mscale(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
// glm::dot: the product vector summed x + y + z
__host__ __device__ __forceinline__ float mdot(float3 a, float3 b) {
    float tx = a.x * b.x, ty = a.y * b.y, tz = a.z * b.z;
    return (tx + ty) + tz;
}
// glm::cross
__host__ __device__ __forceinline__ float3 mcross(float3 x, float3 y) {
    return make_float3(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
__host__ __device__ __forceinline__ float3 mnormalize(float3 v) { return mscale(v, 1.0f / sqrtf(mdot(v, v))); }

// Obj::RayTriangleTest (obj.cpp:354-398): on a hit, t is the distance along the (unit) ray.
__host__ __device__ __forceinline__ bool tri_ray(const MeshTri& T, float3 o, float3 d, float& t) {
    const float3 v0 = m3(T.v0);
    const float3 e1 = msub(m3(T.v1), v0);
    const float3 e2 = msub(m3(T.v2), v0);
    const float3 pvec = mcross(d, e2);
    const float det = mdot(e1, pvec);
    if (det == 0.0f) return false;
    const float inv_det = 1.0f / det;
    const float3 tvec = msub(o, v0);
    const float bx = mdot(tvec, pvec) * inv_det;
    const float3 qvec = mcross(tvec, e1);
    const float by = mdot(d, qvec) * inv_det;
    t = mdot(e2, qvec) * inv_det;
    return bx >= 0.0f && by >= 0.0f && (bx + by) <= 1.0f;
}

// Closest point of a triangle to p (the Voronoi-region method of Ericson, Real-Time Collision
// Detection, 2005, section 5.1.5).
__host__ __device__ __forceinline__ float3 tri_closest(const MeshTri& T, float3 p) {
    const float3 a = m3(T.v0), b = m3(T.v1), c = m3(T.v2);
    const float3 ab = msub(b, a), ac = msub(c, a), ap = msub(p, a);
    const float d1 = mdot(ab, ap), d2 = mdot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return a;
    const float3 bp = msub(p, b);
    const float d3 = mdot(ab, bp), d4 = mdot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return b;
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return madd(a, mscale(ab, d1 / (d1 - d3)));
    const float3 cp = msub(p, c);
    const float d5 = mdot(ab, cp), d6 = mdot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return c;
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return madd(a, mscale(ac, d2 / (d2 - d6)));
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f)
        return madd(b, mscale(msub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
    const float denom = 1.0f / ((va + vb) + vc);
    return madd(madd(a, mscale(ab, vb * denom)), mscale(ac, vc * denom));
}

// Does the ray (o, unit d) reach box B at a distance not beyond tmax?  Conservative: the boxes
// are widened when built, so a triangle the test hits is never skipped.
__host__ __device__ __forceinline__ bool box_ray(const MeshNode& B, float3 o, float3 d, float tmax) {
    float t0 = 0.0f, t1 = tmax;
    const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    for (int a = 0; a < 3; ++a) {
        if (dd[a] == 0.0f) {
            if (oo[a] < B.lo[a] || oo[a] > B.hi[a]) return false;
            continue;
        }
        const float inv = 1.0f / dd[a];
        float ta = (B.lo[a] - oo[a]) * inv, tb = (B.hi[a] - oo[a]) * inv;
        if (ta > tb) {
            const float s = ta;
            ta = tb;
            tb = s;
        }
        t0 = ta > t0 ? ta : t0;
        t1 = tb < t1 ? tb : t1;
        if (t0 > t1) return false;
    }
    return true;
}

__host__ __device__ __forceinline__ float box_dist2(const MeshNode& B, float3 p) {
    const float pp[3] = {p.x, p.y, p.z};
    float s = 0.0f;
    for (int a = 0; a < 3; ++a) {
        const float e = pp[a] < B.lo[a] ? B.lo[a] - pp[a] : (pp[a] > B.hi[a] ? pp[a] - B.hi[a] : 0.0f);
        s += e * e;
    }
    return s;
}

__host__ __device__ __forceinline__ int f_bits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_int(f);
#else
    int v;
    memcpy(&v, &f, 4);
    return v;
#endif
}
// The mesh a triangle belongs to (v0.w) and its index across the scene's meshes in mesh and
// file order (v1.w), the tie-break of the nearest-hit and closest-point queries.
__host__ __device__ __forceinline__ int tri_mesh(const MeshTri& T) { return f_bits(T.v0.w); }
__host__ __device__ __forceinline__ int tri_key(const MeshTri& T) { return f_bits(T.v1.w); }

// Parity of the hits of the ray from p along +z, one bit per mesh: p is inside a mesh when its
// bit is set.  Hits count at t > 0.
__host__ __device__ inline uint32_t mesh_inside_bits(const MeshNode* N, const MeshTri* T, float3 p) {
    if (!N) return 0u;
    const float3 d = make_float3(0.0f, 0.0f, 1.0f);
    uint32_t bits = 0u;
    int stack[kMeshStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const MeshNode& B = N[stack[--sp]];
        if (p.x < B.lo[0] || p.x > B.hi[0] || p.y < B.lo[1] || p.y > B.hi[1] || p.z > B.hi[2]) continue;
        if (B.b >= 0) {
            if (sp + 2 <= kMeshStack) {
                stack[sp++] = B.b;
                stack[sp++] = B.a;
            }
            continue;
        }
        for (int t = B.a; t < B.a - B.b; ++t) {
            float th;
            if (tri_ray(T[t], p, d, th) && th > 0.0f) bits ^= 1u << (tri_mesh(T[t]) & 31);
        }
    }
    return bits;
}

// Nearest hit (t > 0) of the ray (o, unit d): the smallest distance |hit - o|, ties to the
// lower triangle key.  Returns the triangle or -1; `point` is o + t d (Ray::GetPointAlongRay).
__host__ __device__ inline int mesh_nearest(const MeshNode* N, const MeshTri* T, float3 o, float3 d, float3& point,
                                            float& dist) {
    int best = -1;
    dist = 0.0f;
    if (!N) return -1;
    float reach = 3.0e38f;  // traversal bound along the ray, a little beyond the best distance
    int stack[kMeshStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const MeshNode& B = N[stack[--sp]];
        if (!box_ray(B, o, d, reach)) continue;
        if (B.b >= 0) {
            if (sp + 2 <= kMeshStack) {
                stack[sp++] = B.b;
                stack[sp++] = B.a;
            }
            continue;
        }
        for (int t = B.a; t < B.a - B.b; ++t) {
            float th;
            if (!tri_ray(T[t], o, d, th) || !(th > 0.0f)) continue;
            const float3 pt = madd(o, mscale(d, th));
            const float3 dv = msub(pt, o);
            const float dd = sqrtf(mdot(dv, dv));
            if (best < 0 || dd < dist || (dd == dist && tri_key(T[t]) < tri_key(T[best]))) {
                best = t;
                dist = dd;
                point = pt;
                reach = dd * 1.0001f + 1.0e-3f;
            }
        }
    }
    return best;
}

// Closest surface point to p: the smallest squared distance, ties to the lower triangle key.
__host__ __device__ inline int mesh_closest(const MeshNode* N, const MeshTri* T, float3 p, float3& q) {
    int best = -1;
    float bd = 0.0f;
    if (!N) return -1;
    int stack[kMeshStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const MeshNode& B = N[stack[--sp]];
        if (best >= 0 && box_dist2(B, p) > bd * 1.0001f + 1.0e-6f) continue;
        if (B.b >= 0) {
            if (sp + 2 <= kMeshStack) {
                stack[sp++] = B.b;
                stack[sp++] = B.a;
            }
            continue;
        }
        for (int t = B.a; t < B.a - B.b; ++t) {
            const float3 c = tri_closest(T[t], p);
            const float3 e = msub(p, c);
            const float d2 = mdot(e, e);
            if (best < 0 || d2 < bd || (d2 == bd && tri_key(T[t]) < tri_key(T[best]))) {
                best = t;
                bd = d2;
                q = c;
            }
        }
    }
    return best;
}

}  // namespace ariel
