// Minimal stand-in for the subset of glm 0.9.9.8 that the reference's
// src/octree_cpu.cpp and src/renderer/octree.cpp use (written for this
// project; no glm source).  Test infrastructure only: it lets the oracle
// recipe compile the reference's own octree code in place.
//
// Semantics pinned to glm's documented behaviour:
//   min(x, y) = (y < x) ? y : x      max(x, y) = (x < y) ? y : x
//   distance(a, b) = sqrt(dot(a - b, a - b)),  dot = (x*x' + y*y') + z*z'
#pragma once
#include <cmath>
#include <cstdint>

namespace glm {

template <typename T> struct tvec2 {
    T x{}, y{};
    tvec2() = default;
    explicit tvec2(T s) : x(s), y(s) {}
    tvec2(T a, T b) : x(a), y(b) {}
    bool operator==(const tvec2& o) const { return x == o.x && y == o.y; }
    bool operator!=(const tvec2& o) const { return !(*this == o); }
};

template <typename T> struct tvec3 {
    T x{}, y{}, z{};
    tvec3() = default;
    explicit tvec3(T s) : x(s), y(s), z(s) {}
    tvec3(T a, T b, T c) : x(a), y(b), z(c) {}
    template <typename U> explicit tvec3(const tvec3<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    tvec3& operator+=(const tvec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    tvec3& operator-=(const tvec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    tvec3& operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
    bool operator==(const tvec3& o) const { return x == o.x && y == o.y && z == o.z; }
    bool operator!=(const tvec3& o) const { return !(*this == o); }
};

template <typename T> struct tvec4 {
    T x{}, y{}, z{}, w{};
    tvec4() = default;
    explicit tvec4(T s) : x(s), y(s), z(s), w(s) {}
    tvec4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    tvec4(const tvec3<T>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
};

#define GLM_SHIM_BINOP(OP)                                                                       \
    template <typename T> tvec3<T> operator OP(const tvec3<T>& a, const tvec3<T>& b) {          \
        return tvec3<T>(a.x OP b.x, a.y OP b.y, a.z OP b.z); }                                   \
    template <typename T> tvec3<T> operator OP(const tvec3<T>& a, T s) {                        \
        return tvec3<T>(a.x OP s, a.y OP s, a.z OP s); }                                         \
    template <typename T> tvec3<T> operator OP(T s, const tvec3<T>& a) {                        \
        return tvec3<T>(s OP a.x, s OP a.y, s OP a.z); }
GLM_SHIM_BINOP(+)
GLM_SHIM_BINOP(-)
GLM_SHIM_BINOP(*)
GLM_SHIM_BINOP(/)
#undef GLM_SHIM_BINOP

template <typename T> tvec3<T> operator-(const tvec3<T>& a) { return tvec3<T>(-a.x, -a.y, -a.z); }

typedef tvec2<float> vec2;
typedef tvec2<int> ivec2;
typedef tvec3<float> vec3;
typedef tvec3<int> ivec3;
typedef tvec3<uint32_t> uvec3;
typedef tvec4<float> vec4;

template <typename T> T min(T a, T b) { return (b < a) ? b : a; }
template <typename T> T max(T a, T b) { return (a < b) ? b : a; }
template <typename T> tvec3<T> min(const tvec3<T>& a, const tvec3<T>& b) {
    return tvec3<T>(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z));
}
template <typename T> tvec3<T> max(const tvec3<T>& a, const tvec3<T>& b) {
    return tvec3<T>(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z));
}
inline float floor(float v) { return std::floor(v); }
inline float ceil(float v) { return std::ceil(v); }
template <typename T> T dot(const tvec3<T>& a, const tvec3<T>& b) {
    return (a.x * b.x + a.y * b.y) + a.z * b.z;
}
inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
inline float distance(const vec3& a, const vec3& b) { return length(a - b); }
inline vec3 normalize(const vec3& v) { float l = length(v); return vec3(v.x / l, v.y / l, v.z / l); }
inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
inline float radians(float deg) { return deg * 0.01745329251994329576923690768489f; }

}  // namespace glm
