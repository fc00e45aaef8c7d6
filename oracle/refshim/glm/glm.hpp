// TEST INFRASTRUCTURE ONLY: stand-in for the glm header that betajippity/Ariel's FLIP step
// includes (src/utilities/utilities.h:19).  glm (OpenGL Mathematics) is third-party and absent
// here; the reference pins no version beyond the "Nuparu v0.1.15.03" bundle (README.md:6),
// which dates from the glm 0.9.6 series.
//
// Only what the FLIP step's sources use is restated, with glm's published semantics:
//  * vec2/vec3/vec4 of float, component constructors converting each argument with
//    static_cast<float> (so `glm::vec3(i-1, j, k)` with unsigned i wraps exactly as in glm);
//  * component-wise + - * / and compound assignment;
//  * dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z  (glm computes the product vector, then sums
//    x + y + z left to right);
//  * length(v) = sqrt(dot(v, v)); normalize(v) = v * inversesqrt(dot(v, v)) with
//    inversesqrt(x) = 1 / sqrt(x);
//  * min/max as ternaries.  glm 0.9.6 writes min as `x < y ? x : y` and max as `x > y ? x : y`;
//    later releases write `(y < x) ? y : x` and `(x < y) ? y : x`.  The two differ only for NaN
//    operands and for +0 against -0.  The default is the later form; -DARIEL_GLM_096_MINMAX
//    selects the 0.9.6 form (the oracle tests build both and hold both to the same results).
// For the mesh sources (src/geom/obj/obj.cpp, src/spatial/aabb.cpp, built by
// oracle/ref_mesh_driver.cpp) also: cross(x, y) as glm writes it, uvec4, vec2 arithmetic, and
// the vec3 <-> vec4 conversions and indexing those files use to compile.
#ifndef ARIEL_REFSHIM_GLM_HPP
#define ARIEL_REFSHIM_GLM_HPP

#include <cmath>

namespace glm {

template <typename T>
inline T min(T x, T y) {
#ifdef ARIEL_GLM_096_MINMAX
    return x < y ? x : y;
#else
    return (y < x) ? y : x;
#endif
}

template <typename T>
inline T max(T x, T y) {
#ifdef ARIEL_GLM_096_MINMAX
    return x > y ? x : y;
#else
    return (x < y) ? y : x;
#endif
}

struct vec4;

struct vec2 {
    float x, y;
    vec2() : x(0.0f), y(0.0f) {}
    template <typename S>
    explicit vec2(S s) : x(static_cast<float>(s)), y(static_cast<float>(s)) {}
    template <typename A, typename B>
    vec2(A a, B b) : x(static_cast<float>(a)), y(static_cast<float>(b)) {}
};

struct vec3 {
    float x, y, z;
    vec3() : x(0.0f), y(0.0f), z(0.0f) {}
    template <typename S>
    explicit vec3(S s) : x(static_cast<float>(s)), y(static_cast<float>(s)), z(static_cast<float>(s)) {}
    template <typename A, typename B, typename C>
    vec3(A a, B b, C c) : x(static_cast<float>(a)), y(static_cast<float>(b)), z(static_cast<float>(c)) {}
    explicit vec3(const vec4& v);

    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }

    vec3& operator+=(const vec3& v) { x += v.x; y += v.y; z += v.z; return *this; }
    vec3& operator-=(const vec3& v) { x -= v.x; y -= v.y; z -= v.z; return *this; }
    vec3& operator*=(const vec3& v) { x *= v.x; y *= v.y; z *= v.z; return *this; }
    vec3& operator/=(const vec3& v) { x /= v.x; y /= v.y; z /= v.z; return *this; }
    vec3& operator+=(float s) { x += s; y += s; z += s; return *this; }
    vec3& operator-=(float s) { x -= s; y -= s; z -= s; return *this; }
    vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
    vec3& operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
};

struct vec4 {
    float x, y, z, w;
    vec4() : x(0.0f), y(0.0f), z(0.0f), w(0.0f) {}
    template <typename S>
    explicit vec4(S s)
        : x(static_cast<float>(s)), y(static_cast<float>(s)), z(static_cast<float>(s)), w(static_cast<float>(s)) {}
    template <typename A, typename B, typename C, typename D>
    vec4(A a, B b, C c, D d)
        : x(static_cast<float>(a)), y(static_cast<float>(b)), z(static_cast<float>(c)), w(static_cast<float>(d)) {}
    template <typename W>
    vec4(const vec3& v, W w) : x(v.x), y(v.y), z(v.z), w(static_cast<float>(w)) {}
    float& operator[](unsigned i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    float operator[](unsigned i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};
inline vec3::vec3(const vec4& v) : x(v.x), y(v.y), z(v.z) {}

struct mat4 {
    vec4 c[4];
};

struct uvec4 {
    unsigned x, y, z, w;
    uvec4() : x(0u), y(0u), z(0u), w(0u) {}
    template <typename S>
    explicit uvec4(S s)
        : x(static_cast<unsigned>(s)), y(static_cast<unsigned>(s)), z(static_cast<unsigned>(s)), w(static_cast<unsigned>(s)) {}
    template <typename A, typename B, typename C, typename D>
    uvec4(A a, B b, C c, D d)
        : x(static_cast<unsigned>(a)), y(static_cast<unsigned>(b)), z(static_cast<unsigned>(c)), w(static_cast<unsigned>(d)) {}
    uvec4(const vec4& v)
        : x(static_cast<unsigned>(v.x)), y(static_cast<unsigned>(v.y)), z(static_cast<unsigned>(v.z)),
          w(static_cast<unsigned>(v.w)) {}
    unsigned& operator[](unsigned i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    unsigned operator[](unsigned i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

// column-major matrix times vector
inline vec4 operator*(const mat4& m, const vec4& v) {
    return vec4(m.c[0].x * v.x + m.c[1].x * v.y + m.c[2].x * v.z + m.c[3].x * v.w,
                m.c[0].y * v.x + m.c[1].y * v.y + m.c[2].y * v.z + m.c[3].y * v.w,
                m.c[0].z * v.x + m.c[1].z * v.y + m.c[2].z * v.z + m.c[3].z * v.w,
                m.c[0].w * v.x + m.c[1].w * v.y + m.c[2].w * v.z + m.c[3].w * v.w);
}

inline vec2 operator+(const vec2& a, const vec2& b) { return vec2(a.x + b.x, a.y + b.y); }
inline vec2 operator-(const vec2& a, const vec2& b) { return vec2(a.x - b.x, a.y - b.y); }
inline vec2 operator*(const vec2& a, float s) { return vec2(a.x * s, a.y * s); }
inline vec2 operator*(float s, const vec2& a) { return vec2(s * a.x, s * a.y); }


inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator/(const vec3& a, const vec3& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline vec3 operator+(const vec3& a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
inline vec3 operator-(const vec3& a, float s) { return vec3(a.x - s, a.y - s, a.z - s); }
inline vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec3 operator+(float s, const vec3& a) { return vec3(s + a.x, s + a.y, s + a.z); }
inline vec3 operator-(float s, const vec3& a) { return vec3(s - a.x, s - a.y, s - a.z); }
inline vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(float s, const vec3& a) { return vec3(s / a.x, s / a.y, s / a.z); }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline bool operator==(const vec3& a, const vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool operator!=(const vec3& a, const vec3& b) { return !(a == b); }

inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 min(const vec3& a, float s) { return vec3(min(a.x, s), min(a.y, s), min(a.z, s)); }
inline vec3 max(const vec3& a, float s) { return vec3(max(a.x, s), max(a.y, s), max(a.z, s)); }
inline vec3 floor(const vec3& a) { return vec3(std::floor(a.x), std::floor(a.y), std::floor(a.z)); }
inline vec3 ceil(const vec3& a) { return vec3(std::ceil(a.x), std::ceil(a.y), std::ceil(a.z)); }

inline float sqrt(float x) { return std::sqrt(x); }
inline float floor(float x) { return std::floor(x); }
inline float inversesqrt(float x) { return 1.0f / std::sqrt(x); }

inline float dot(const vec3& a, const vec3& b) {
    vec3 t(a * b);
    return t.x + t.y + t.z;
}
inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
inline vec3 cross(const vec3& x, const vec3& y) {
    return vec3(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
inline vec3 normalize(const vec3& v) { return v * inversesqrt(dot(v, v)); }

}  // namespace glm

#endif
