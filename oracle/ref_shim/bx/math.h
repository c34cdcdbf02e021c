/*
 * ORACLE (test infrastructure): the part of bx's math API that the
 * reference's src/bvh.cpp and src/lights.cpp use, so they compile here
 * unmodified (bx itself is fetched at the reference's configure time and is
 * not in this container). Written from bx's documented semantics: plain
 * component-wise float arithmetic.
 */
#pragma once
#include <cmath>

namespace bx
{
struct Vec3
{
	float x, y, z;
};

constexpr float kPi = 3.1415926535897932384626433832795f;

inline Vec3 min(const Vec3& a, const Vec3& b) { return { a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z }; }
inline Vec3 max(const Vec3& a, const Vec3& b) { return { a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z }; }
inline Vec3 add(const Vec3& a, const Vec3& b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline Vec3 sub(const Vec3& a, const Vec3& b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline Vec3 mul(const Vec3& a, float s) { return { a.x * s, a.y * s, a.z * s }; }
inline Vec3 cross(const Vec3& a, const Vec3& b) { return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }
inline float dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(const Vec3& a) { return std::sqrt(dot(a, a)); }
} // namespace bx
