/*
 * ORACLE (test infrastructure, never linked into the product).
 *
 * A small GLSL-semantics shim so that the CPU restatement of the reference's
 * shaders (oracle.cpp) reads line by line like the shader sources.
 * Every operation is one binary32 operation in source order, as the numeric
 * conventions of include/restir_numeric.h require (build with
 * -ffp-contract=off, never -ffast-math): dot is ((x*x + y*y) + z*z),
 * normalize multiplies by 1 / sqrt(dot), mix is a*(1-t) + b*t, min and max
 * are fmin and fmax, mul(M, v) sums the row's products left to right.
 */
#ifndef ORACLE_GLSL_H
#define ORACLE_GLSL_H

#include "../include/restir_numeric.h"

#include <cmath>
#include <cstdint>

namespace glsl
{

typedef uint32_t uint;

struct vec2
{
	float x, y;
	vec2() : x(0.0f), y(0.0f) {}
	vec2(float _x, float _y) : x(_x), y(_y) {}
	explicit vec2(float _s) : x(_s), y(_s) {}
};

struct vec3
{
	float x, y, z;
	vec3() : x(0.0f), y(0.0f), z(0.0f) {}
	vec3(float _x, float _y, float _z) : x(_x), y(_y), z(_z) {}
	explicit vec3(float _s) : x(_s), y(_s), z(_s) {}
};

struct vec4
{
	float x, y, z, w;
	vec4() : x(0.0f), y(0.0f), z(0.0f), w(0.0f) {}
	vec4(float _x, float _y, float _z, float _w) : x(_x), y(_y), z(_z), w(_w) {}
	vec4(const vec3& _v, float _w) : x(_v.x), y(_v.y), z(_v.z), w(_w) {}
	explicit vec4(float _s) : x(_s), y(_s), z(_s), w(_s) {}
	vec3 xyz() const { return vec3(x, y, z); }
	vec2 xy() const { return vec2(x, y); }
};

inline vec2 vec2_splat(float s) { return vec2(s, s); }
inline vec3 vec3_splat(float s) { return vec3(s, s, s); }
inline vec4 vec4_splat(float s) { return vec4(s, s, s, s); }

#define GLSL_VEC2_OP(op) \
	inline vec2 operator op(const vec2& a, const vec2& b) { return vec2(a.x op b.x, a.y op b.y); } \
	inline vec2 operator op(const vec2& a, float b) { return vec2(a.x op b, a.y op b); } \
	inline vec2 operator op(float a, const vec2& b) { return vec2(a op b.x, a op b.y); }
#define GLSL_VEC3_OP(op) \
	inline vec3 operator op(const vec3& a, const vec3& b) { return vec3(a.x op b.x, a.y op b.y, a.z op b.z); } \
	inline vec3 operator op(const vec3& a, float b) { return vec3(a.x op b, a.y op b, a.z op b); } \
	inline vec3 operator op(float a, const vec3& b) { return vec3(a op b.x, a op b.y, a op b.z); }
GLSL_VEC2_OP(+) GLSL_VEC2_OP(-) GLSL_VEC2_OP(*) GLSL_VEC2_OP(/)
GLSL_VEC3_OP(+) GLSL_VEC3_OP(-) GLSL_VEC3_OP(*) GLSL_VEC3_OP(/)
#undef GLSL_VEC2_OP
#undef GLSL_VEC3_OP

inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec3& operator+=(vec3& a, const vec3& b) { a = a + b; return a; }
inline vec3& operator*=(vec3& a, float b) { a = a * b; return a; }
inline vec3& operator/=(vec3& a, float b) { a = a / b; return a; }
inline vec2& operator+=(vec2& a, const vec2& b) { a = a + b; return a; }
inline vec2& operator/=(vec2& a, float b) { a = a / b; return a; }

inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b)
{
	return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float inversesqrt(float x) { return 1.0f / std::sqrt(x); }
inline float length(const vec3& a) { return std::sqrt(dot(a, a)); }
inline float distance(const vec3& a, const vec3& b) { return length(a - b); }
inline vec3 normalize(const vec3& a) { return a * inversesqrt(dot(a, a)); }

inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }
inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 min(const vec3& a, float b) { return min(a, vec3_splat(b)); }
inline vec3 max(const vec3& a, float b) { return max(a, vec3_splat(b)); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline uint min(uint a, uint b) { return a < b ? a : b; }
inline uint max(uint a, uint b) { return a > b ? a : b; }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline float abs(float x) { return std::fabs(x); }
inline vec3 abs(const vec3& a) { return vec3(abs(a.x), abs(a.y), abs(a.z)); }
inline float floor(float x) { return std::floor(x); }
inline vec2 floor(const vec2& a) { return vec2(floor(a.x), floor(a.y)); }
inline vec3 floor(const vec3& a) { return vec3(floor(a.x), floor(a.y), floor(a.z)); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline vec2 mix(const vec2& a, const vec2& b, float t) { return a * (1.0f - t) + b * t; }
inline vec3 mix(const vec3& a, const vec3& b, float t) { return a * (1.0f - t) + b * t; }
/* mix with a per-component selector (restir.sh reprojection weights). */
inline vec2 mix(const vec2& a, const vec2& b, const vec2& t)
{
	return vec2(mix(a.x, b.x, t.x), mix(a.y, b.y, t.y));
}
inline float step(float edge, float x) { return x < edge ? 0.0f : 1.0f; }
inline float exp(float x) { return rn_exp(x); }
inline float sin(float x) { return rn_sin(x); }
inline float cos(float x) { return rn_cos(x); }
inline uint floatBitsToUint(float x) { return rn_float_bits(x); }
inline bool isnan_(float x) { return x != x; }

/* Row-major 4x4, clip = M * v. */
struct mat4
{
	float m[16];
};

inline vec4 mul(const mat4& M, const vec4& v)
{
	const float* m = M.m;
	return vec4(
		  m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3] * v.w
		, m[4] * v.x + m[5] * v.y + m[6] * v.z + m[7] * v.w
		, m[8] * v.x + m[9] * v.y + m[10] * v.z + m[11] * v.w
		, m[12] * v.x + m[13] * v.y + m[14] * v.z + m[15] * v.w);
}

inline mat4 make_mat4(const float* p)
{
	mat4 M;
	for (int i = 0; i < 16; ++i)
	{
		M.m[i] = p[i];
	}
	return M;
}

} // namespace glsl

#endif // ORACLE_GLSL_H
