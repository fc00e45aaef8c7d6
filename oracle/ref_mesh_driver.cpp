// TEST INFRASTRUCTURE ONLY: exposes betajippity/Ariel's own ray-triangle test for the parity
// tests.  The reference's src/spatial/aabb.cpp and src/geom/obj/obj.cpp are compiled here as
// they lie under the reference checkout (`make -C oracle reference`; the include path points
// at its src/), with refshim/prelude.hpp and refshim/mesh_prelude.hpp standing in for the
// libraries they need.  Obj::RayTriangleTest (obj.cpp:354-398) is a static inline member defined
// in obj.cpp, so it is called from this translation unit, which includes that file.
#include "spatial/aabb.cpp"
#include "geom/obj/obj.cpp"

extern "C" {

// Obj::RayTriangleTest for the triangle v[0..8] (three xyz vertices) and the ray (o, d) as
// given: returns 1 on a hit, with the reference's hit point (Ray::GetPointAlongRay of its
// distance) in point[0..2].  The normals and UVs that the test also interpolates are constants.
int32_t ariel_pin_ray_triangle(const float* v, const float* o, const float* d, float* point) {
    rayCore::Ray r;
    r.m_origin = glm::vec3(o[0], o[1], o[2]);
    r.m_direction = glm::vec3(d[0], d[1], d[2]);
    const glm::vec3 v0(v[0], v[1], v[2]), v1(v[3], v[4], v[5]), v2(v[6], v[7], v[8]);
    const glm::vec3 n(0.0f, 0.0f, 1.0f);
    const glm::vec2 uv(0.0f, 0.0f);
    const rayCore::Intersection x = objCore::Obj::RayTriangleTest(v0, v1, v2, n, n, n, uv, uv, uv, r);
    if (!x.m_hit) return 0;
    point[0] = x.m_point.x;
    point[1] = x.m_point.y;
    point[2] = x.m_point.z;
    return 1;
}

}  // extern "C"
