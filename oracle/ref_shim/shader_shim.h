/*
 * ORACLE (test infrastructure, never linked into the product).
 *
 * The GLSL / bgfx shader-language environment in C++, so that the
 * reference's own shader sources (pkonecki/restir, the .sh and .sc files of its shaders directory)
 * compile as C++ and run on the CPU. oracle/ref_shim/glsl_to_cpp.py turns
 * each shader file into C++ first, mechanically: float literals get an `f`
 * suffix (GLSL literals are single precision), `out`/`inout` parameters
 * become references, comments are blanked; nothing else changes. This
 * header supplies the rest:
 *
 *  - vec2/3/4, ivec2/3, uvec2/3 with the swizzles the shaders use (.xyz,
 *    .rgb, .xy, .zw), mat4 with bgfx's mul(M, v) (row-major storage, clip =
 *    M * v, as RestirParams holds the matrices);
 *  - the GLSL built-ins, one IEEE binary32 operation each in source order
 *    under the numeric conventions of include/restir_numeric.h (dot sums
 *    left to right, normalize multiplies by 1/sqrt, mix is a*(1-t) + b*t,
 *    min/max are fmin/fmax, exp/sin/cos/pow are the library's own, floor of
 *    log2 is exact), the same conventions the oracle restatement and the
 *    kernels follow;
 *  - bgfx's resource macros (SAMPLER2D, IMAGE2D_*, BUFFER_*, uniform,
 *    SHARED, NUM_THREADS) as globals the C interface binds, with point
 *    sampling at floor(uv * size) clamped to the image (the sampling rule of
 *    the C ABI), and the compute built-ins (gl_GlobalInvocationID, ...) as
 *    per-lane values the dispatcher sets (a group's lanes are coroutines that
 *    switch at barriers, groups run on all host threads, and SHARED memory is
 *    one copy per worker thread);
 *  - bgfx shaderlib's clip-space helpers with NDC depth in [0, 1]
 *    (toClipSpaceDepth(d) = d, toClipSpaceY(y) = y when the texture origin is
 *    bottom-left, else -y, clipToWorld divides by w).
 */
#ifndef ORACLE_SHADER_SHIM_H
#define ORACLE_SHADER_SHIM_H

#include "../../include/restir_numeric.h"

#include <cmath>
#include <cstdint>
#include <cstring>

namespace refsh
{

typedef uint32_t uint;

struct vec2;
struct vec3;
struct vec4;

// A swizzle view of N components of a vector's storage (read and write).
template <class V, class T, int S, int A, int B>
struct Swizzle2
{
	T e[S];
	operator V() const { return V(e[A], e[B]); }
	Swizzle2& operator=(const V& v)
	{
		e[A] = v.x;
		e[B] = v.y;
		return *this;
	}
};

template <class V, class T, int S, int A, int B, int C>
struct Swizzle3
{
	T e[S];
	operator V() const { return V(e[A], e[B], e[C]); }
	Swizzle3& operator=(const V& v)
	{
		e[A] = v.x;
		e[B] = v.y;
		e[C] = v.z;
		return *this;
	}
};

struct vec2
{
	float x, y;
	vec2() : x(0.0f), y(0.0f) {}
	vec2(float _x, float _y) : x(_x), y(_y) {}
	explicit vec2(float _s) : x(_s), y(_s) {}
	explicit vec2(const struct uvec2& _v);
	explicit vec2(const struct ivec2& _v);
};

struct vec3
{
	union
	{
		struct { float x, y, z; };
		struct { float r, g, b; };
		Swizzle2<vec2, float, 3, 0, 1> xy;
	};
	vec3() : x(0.0f), y(0.0f), z(0.0f) {}
	vec3(float _x, float _y, float _z) : x(_x), y(_y), z(_z) {}
	vec3(const vec2& _v, float _z) : x(_v.x), y(_v.y), z(_z) {}
	explicit vec3(float _s) : x(_s), y(_s), z(_s) {}
	vec3(const vec3& _v) : x(_v.x), y(_v.y), z(_v.z) {}
	vec3& operator=(const vec3& _v)
	{
		x = _v.x;
		y = _v.y;
		z = _v.z;
		return *this;
	}
};

struct vec4
{
	union
	{
		struct { float x, y, z, w; };
		struct { float r, g, b, a; };
		Swizzle3<vec3, float, 4, 0, 1, 2> xyz;
		Swizzle3<vec3, float, 4, 0, 1, 2> rgb;
		Swizzle2<vec2, float, 4, 0, 1> xy;
		Swizzle2<vec2, float, 4, 2, 3> zw;
	};
	vec4() : x(0.0f), y(0.0f), z(0.0f), w(0.0f) {}
	vec4(float _x, float _y, float _z, float _w) : x(_x), y(_y), z(_z), w(_w) {}
	vec4(const vec3& _v, float _w) : x(_v.x), y(_v.y), z(_v.z), w(_w) {}
	vec4(const vec2& _a, const vec2& _b) : x(_a.x), y(_a.y), z(_b.x), w(_b.y) {}
	vec4(const vec2& _a, float _z, float _w) : x(_a.x), y(_a.y), z(_z), w(_w) {}
	explicit vec4(float _s) : x(_s), y(_s), z(_s), w(_s) {}
	vec4(const vec4& _v) : x(_v.x), y(_v.y), z(_v.z), w(_v.w) {}
	vec4& operator=(const vec4& _v)
	{
		x = _v.x;
		y = _v.y;
		z = _v.z;
		w = _v.w;
		return *this;
	}
};

struct ivec2
{
	int x, y;
	ivec2() : x(0), y(0) {}
	ivec2(int _x, int _y) : x(_x), y(_y) {}
	explicit ivec2(const vec2& _v) : x(int(_v.x)), y(int(_v.y)) {}
};

struct ivec3
{
	int x, y, z;
	ivec3() : x(0), y(0), z(0) {}
	ivec3(int _x, int _y, int _z) : x(_x), y(_y), z(_z) {}
	explicit ivec3(const vec3& _v) : x(int(_v.x)), y(int(_v.y)), z(int(_v.z)) {}
};

struct uvec2
{
	uint x, y;
	uvec2() : x(0u), y(0u) {}
	uvec2(uint _x, uint _y) : x(_x), y(_y) {}
	explicit uvec2(const ivec2& _v) : x(uint(_v.x)), y(uint(_v.y)) {}
};

struct uvec3
{
	union
	{
		struct { uint x, y, z; };
		Swizzle2<uvec2, uint, 3, 0, 1> xy;
	};
	uvec3() : x(0u), y(0u), z(0u) {}
	uvec3(uint _x, uint _y, uint _z) : x(_x), y(_y), z(_z) {}
	uvec3(const uvec3& _v) : x(_v.x), y(_v.y), z(_v.z) {}
	uvec3& operator=(const uvec3& _v)
	{
		x = _v.x;
		y = _v.y;
		z = _v.z;
		return *this;
	}
};

inline vec2::vec2(const uvec2& _v) : x(float(_v.x)), y(float(_v.y)) {}
inline vec2::vec2(const ivec2& _v) : x(float(_v.x)), y(float(_v.y)) {}

// bgfx's splat constructors.
inline vec2 vec2_splat(float _s) { return vec2(_s, _s); }
inline vec3 vec3_splat(float _s) { return vec3(_s, _s, _s); }
inline vec4 vec4_splat(float _s) { return vec4(_s, _s, _s, _s); }

// Component-wise arithmetic (one binary32 operation per component).
#define REFSH_VEC2_OP(op) \
	inline vec2 operator op(const vec2& a, const vec2& b) { return vec2(a.x op b.x, a.y op b.y); } \
	inline vec2 operator op(const vec2& a, float b) { return vec2(a.x op b, a.y op b); } \
	inline vec2 operator op(float a, const vec2& b) { return vec2(a op b.x, a op b.y); } \
	inline vec2& operator op##=(vec2& a, const vec2& b) { a = a op b; return a; } \
	inline vec2& operator op##=(vec2& a, float b) { a = a op b; return a; }
#define REFSH_VEC3_OP(op) \
	inline vec3 operator op(const vec3& a, const vec3& b) { return vec3(a.x op b.x, a.y op b.y, a.z op b.z); } \
	inline vec3 operator op(const vec3& a, float b) { return vec3(a.x op b, a.y op b, a.z op b); } \
	inline vec3 operator op(float a, const vec3& b) { return vec3(a op b.x, a op b.y, a op b.z); } \
	inline vec3& operator op##=(vec3& a, const vec3& b) { a = a op b; return a; } \
	inline vec3& operator op##=(vec3& a, float b) { a = a op b; return a; }
#define REFSH_VEC4_OP(op) \
	inline vec4 operator op(const vec4& a, const vec4& b) { return vec4(a.x op b.x, a.y op b.y, a.z op b.z, a.w op b.w); } \
	inline vec4 operator op(const vec4& a, float b) { return vec4(a.x op b, a.y op b, a.z op b, a.w op b); } \
	inline vec4 operator op(float a, const vec4& b) { return vec4(a op b.x, a op b.y, a op b.z, a op b.w); } \
	inline vec4& operator op##=(vec4& a, const vec4& b) { a = a op b; return a; } \
	inline vec4& operator op##=(vec4& a, float b) { a = a op b; return a; }
REFSH_VEC2_OP(+) REFSH_VEC2_OP(-) REFSH_VEC2_OP(*) REFSH_VEC2_OP(/)
REFSH_VEC3_OP(+) REFSH_VEC3_OP(-) REFSH_VEC3_OP(*) REFSH_VEC3_OP(/)
REFSH_VEC4_OP(+) REFSH_VEC4_OP(-) REFSH_VEC4_OP(*) REFSH_VEC4_OP(/)
#undef REFSH_VEC2_OP
#undef REFSH_VEC3_OP
#undef REFSH_VEC4_OP

inline vec2 operator-(const vec2& a) { return vec2(-a.x, -a.y); }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec4 operator-(const vec4& a) { return vec4(-a.x, -a.y, -a.z, -a.w); }
inline ivec2 operator+(const ivec2& a, const ivec2& b) { return ivec2(a.x + b.x, a.y + b.y); }
inline ivec2 operator-(const ivec2& a, const ivec2& b) { return ivec2(a.x - b.x, a.y - b.y); }

// Geometry.
inline float dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(const vec4& a, const vec4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline vec3 cross(const vec3& a, const vec3& b)
{
	return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float inversesqrt(float x) { return 1.0f / std::sqrt(x); }
inline float length(const vec2& a) { return std::sqrt(dot(a, a)); }
inline float length(const vec3& a) { return std::sqrt(dot(a, a)); }
inline float distance(const vec2& a, const vec2& b) { return length(a - b); }
inline float distance(const vec3& a, const vec3& b) { return length(a - b); }
inline vec2 normalize(const vec2& a) { return a * inversesqrt(dot(a, a)); }
inline vec3 normalize(const vec3& a) { return a * inversesqrt(dot(a, a)); }
inline vec3 reflect(const vec3& i, const vec3& n) { return i - n * (2.0f * dot(n, i)); }

// Common functions.
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline uint min(uint a, uint b) { return a < b ? a : b; }
inline uint max(uint a, uint b) { return a > b ? a : b; }
inline vec2 min(const vec2& a, const vec2& b) { return vec2(min(a.x, b.x), min(a.y, b.y)); }
inline vec2 max(const vec2& a, const vec2& b) { return vec2(max(a.x, b.x), max(a.y, b.y)); }
inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec2 min(const vec2& a, float b) { return min(a, vec2_splat(b)); }
inline vec2 max(const vec2& a, float b) { return max(a, vec2_splat(b)); }
inline vec3 min(const vec3& a, float b) { return min(a, vec3_splat(b)); }
inline vec3 max(const vec3& a, float b) { return max(a, vec3_splat(b)); }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline int clamp(int x, int lo, int hi) { return min(max(x, lo), hi); }
inline vec2 clamp(const vec2& x, const vec2& lo, const vec2& hi) { return min(max(x, lo), hi); }
inline vec2 clamp(const vec2& x, float lo, float hi) { return min(max(x, lo), hi); }
inline vec3 clamp(const vec3& x, float lo, float hi) { return min(max(x, lo), hi); }
inline float saturate(float x) { return clamp(x, 0.0f, 1.0f); }
inline vec3 saturate(const vec3& x) { return clamp(x, 0.0f, 1.0f); }
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline vec2 abs(const vec2& a) { return vec2(abs(a.x), abs(a.y)); }
inline vec3 abs(const vec3& a) { return vec3(abs(a.x), abs(a.y), abs(a.z)); }
inline float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline float floor(float x) { return std::floor(x); }
inline vec2 floor(const vec2& a) { return vec2(floor(a.x), floor(a.y)); }
inline vec3 floor(const vec3& a) { return vec3(floor(a.x), floor(a.y), floor(a.z)); }
inline float ceil(float x) { return std::ceil(x); }
inline float fract(float x) { return x - std::floor(x); }
inline vec2 fract(const vec2& a) { return vec2(fract(a.x), fract(a.y)); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline vec2 mix(const vec2& a, const vec2& b, float t) { return a * (1.0f - t) + b * t; }
inline vec3 mix(const vec3& a, const vec3& b, float t) { return a * (1.0f - t) + b * t; }
inline vec4 mix(const vec4& a, const vec4& b, float t) { return a * (1.0f - t) + b * t; }
inline vec2 mix(const vec2& a, const vec2& b, const vec2& t) { return vec2(mix(a.x, b.x, t.x), mix(a.y, b.y, t.y)); }
inline vec3 mix(const vec3& a, const vec3& b, const vec3& t)
{
	return vec3(mix(a.x, b.x, t.x), mix(a.y, b.y, t.y), mix(a.z, b.z, t.z));
}
inline float step(float edge, float x) { return x < edge ? 0.0f : 1.0f; }
inline float smoothstep(float e0, float e1, float x)
{
	float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
	return t * t * (3.0f - 2.0f * t);
}

// Transcendentals: the library's own (include/restir_numeric.h).
inline float exp(float x) { return rn_exp(x); }
inline float sin(float x) { return rn_sin(x); }
inline float cos(float x) { return rn_cos(x); }
inline float exp2(float x) { return rn_exp2(x); }
// log2 whose floor is the exact floor(log2 x): the correctly rounded value,
// nudged below an integer it rounded up to. Only floor(log2 x) is used on
// the hot path (hashgrid.sh gridCellSize).
inline float log2(float x)
{
	double exact = std::log2(double(x));
	float rounded = float(exact);
	if (rounded == std::floor(rounded) && double(rounded) > exact)
	{
		rounded = std::nextafter(rounded, -INFINITY);
	}
	return rounded;
}
// pow(x, 5) and pow(x, 64) are fixed product chains (the only exponents the
// hot path's shaders use), anything else exp2(y log2 x).
inline float pow(float x, float y)
{
	return y == 5.0f ? rn_pow5(x) : (y == 64.0f ? rn_pow64(x) : rn_pow(x, y));
}

inline uint floatBitsToUint(float x) { return rn_float_bits(x); }
inline float uintBitsToFloat(uint u)
{
	float f;
	std::memcpy(&f, &u, sizeof(f));
	return f;
}
inline bool isnan(float x) { return x != x; }
inline bool isinf(float x) { return std::isinf(x); }

// bgfx mul(M, v): clip = M * v with M stored row-major (RestirParams' matrices).
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

// --- resources ---------------------------------------------------------------------------------

enum TexelFormat
{
	kFormatR32F,     // float
	kFormatRGBA32F,  // float4
	kFormatRGBA16F,  // half4
	kFormatBGRA8,    // unorm8, stored b, g, r, a
	kFormatRG32F,    // float2
};

// A bound 2D image: point sampling at floor(uv * size), clamped.
struct Texture
{
	const void* data = nullptr;
	int width = 0;
	int height = 0;
	TexelFormat format = kFormatRGBA32F;
	void* write = nullptr; // image targets: where imageStore writes

	vec4 fetch(int x, int y) const
	{
		x = x < 0 ? 0 : (x >= width ? width - 1 : x);
		y = y < 0 ? 0 : (y >= height ? height - 1 : y);
		const size_t i = size_t(y) * size_t(width) + size_t(x);
		switch (format)
		{
		case kFormatR32F:
		{
			float v = static_cast<const float*>(data)[i];
			return vec4(v, 0.0f, 0.0f, 1.0f);
		}
		case kFormatRG32F:
		{
			const float* p = static_cast<const float*>(data) + 2 * i;
			return vec4(p[0], p[1], 0.0f, 1.0f);
		}
		case kFormatRGBA32F:
		{
			const float* p = static_cast<const float*>(data) + 4 * i;
			return vec4(p[0], p[1], p[2], p[3]);
		}
		case kFormatRGBA16F:
		{
			const uint16_t* p = static_cast<const uint16_t*>(data) + 4 * i;
			return vec4(rn_half_to_float(p[0]), rn_half_to_float(p[1]), rn_half_to_float(p[2]),
				rn_half_to_float(p[3]));
		}
		case kFormatBGRA8:
		{
			const uint8_t* p = static_cast<const uint8_t*>(data) + 4 * i;
			return vec4(rn_unorm8_to_float(p[2]), rn_unorm8_to_float(p[1]), rn_unorm8_to_float(p[0]),
				rn_unorm8_to_float(p[3]));
		}
		}
		return vec4();
	}

	void store(int x, int y, const vec4& v) const
	{
		if (x < 0 || y < 0 || x >= width || y >= height || write == nullptr)
		{
			return;
		}
		const size_t i = size_t(y) * size_t(width) + size_t(x);
		switch (format)
		{
		case kFormatR32F:
			static_cast<float*>(write)[i] = v.x;
			break;
		case kFormatRG32F:
			static_cast<float*>(write)[2 * i] = v.x;
			static_cast<float*>(write)[2 * i + 1] = v.y;
			break;
		case kFormatRGBA32F:
		{
			float* p = static_cast<float*>(write) + 4 * i;
			p[0] = v.x;
			p[1] = v.y;
			p[2] = v.z;
			p[3] = v.w;
			break;
		}
		case kFormatRGBA16F:
		{
			uint16_t* p = static_cast<uint16_t*>(write) + 4 * i;
			p[0] = rn_float_to_half(v.x);
			p[1] = rn_float_to_half(v.y);
			p[2] = rn_float_to_half(v.z);
			p[3] = rn_float_to_half(v.w);
			break;
		}
		case kFormatBGRA8:
		{
			uint8_t* p = static_cast<uint8_t*>(write) + 4 * i;
			p[2] = rn_unorm8(v.x);
			p[1] = rn_unorm8(v.y);
			p[0] = rn_unorm8(v.z);
			p[3] = rn_unorm8(v.w);
			break;
		}
		}
	}
};

inline int texelCoordinate(float uv, int size)
{
	float t = std::floor(uv * float(size));
	if (!(t >= 0.0f))
	{
		return 0;
	}
	return t >= float(size) ? size - 1 : int(t);
}

inline vec4 texture2DLod(const Texture& t, const vec2& uv, float)
{
	return t.fetch(texelCoordinate(uv.x, t.width), texelCoordinate(uv.y, t.height));
}
inline vec4 texture2D(const Texture& t, const vec2& uv) { return texture2DLod(t, uv, 0.0f); }
inline vec4 texelFetch(const Texture& t, const ivec2& p, int) { return t.fetch(p.x, p.y); }
inline vec4 imageLoad(const Texture& t, const ivec2& p) { return t.fetch(p.x, p.y); }
inline void imageStore(const Texture& t, const ivec2& p, const vec4& v) { t.store(p.x, p.y, v); }
inline ivec2 imageSize(const Texture& t) { return ivec2(t.width, t.height); }

// Storage buffers: the bound pointer and its element count (bounds-checked).
template <class T>
struct Buffer
{
	T* data = nullptr;
	size_t count = 0;
	static T s_dummy;
	T& operator[](int i) const { return (i >= 0 && size_t(i) < count) ? data[i] : (s_dummy = T()); }
	T& operator[](uint i) const { return size_t(i) < count ? data[i] : (s_dummy = T()); }
};
template <class T>
T Buffer<T>::s_dummy;

// Shared-memory and buffer atomics. The dispatcher runs one invocation at a
// time, or the lanes of one group under a lock (GroupLanes below).
void atomicLock();
void atomicUnlock();
inline void atomicFetchAndAdd(uint& _memory, uint _value, uint& _original)
{
	atomicLock();
	_original = _memory;
	_memory += _value;
	atomicUnlock();
}
inline void atomicFetchAndAdd(int& _memory, int _value, int& _original)
{
	atomicLock();
	_original = _memory;
	_memory += _value;
	atomicUnlock();
}
inline void atomicFetchCompareExchange(uint& _memory, uint _compare, uint _value, uint& _original)
{
	atomicLock();
	_original = _memory;
	if (_memory == _compare)
	{
		_memory = _value;
	}
	atomicUnlock();
}
inline uint atomicAdd(uint& _memory, uint _value)
{
	atomicLock();
	uint original = _memory;
	_memory += _value;
	atomicUnlock();
	return original;
}

// Compute built-ins, set per invocation by the dispatcher. The lanes of a
// compute group run as coroutines inside one worker thread (they switch at
// the shader's barriers), so everything private to an invocation lives in a
// per-lane slot of the worker's storage, indexed by the running lane.
constexpr int kMaxLanes = 64;
struct LaneBuiltins
{
	uvec3 globalId;
	uvec3 localId;
	uvec3 groupId;
	uint localIndex = 0u;
};
extern thread_local int t_lane;
extern thread_local LaneBuiltins t_builtins[kMaxLanes];
#define gl_GlobalInvocationID (refsh::t_builtins[refsh::t_lane].globalId)
#define gl_LocalInvocationID (refsh::t_builtins[refsh::t_lane].localId)
#define gl_WorkGroupID (refsh::t_builtins[refsh::t_lane].groupId)
#define gl_LocalInvocationIndex (refsh::t_builtins[refsh::t_lane].localIndex)
void barrier();
inline void memoryBarrierShared() {}
inline void GroupMemoryBarrierWithGroupSync() { barrier(); }

// Fragment built-ins and the full-screen pass's varying (the texel centre).
extern thread_local vec2 v_texcoord0;
extern thread_local vec4 gl_FragCoord;
extern thread_local vec4 gl_FragColor;
extern thread_local vec4 gl_FragData[4];

// bgfx shaderlib's clip-space helpers (texture origin from the bound frame).
extern bool g_originBottomLeft;
inline float toClipSpaceDepth(float _depth) { return _depth; }
inline float toClipSpaceY(float _y) { return g_originBottomLeft ? _y : -_y; }
inline vec3 clipToWorld(const mat4& _inverse, const vec3& _clip)
{
	vec4 world = mul(_inverse, vec4(_clip, 1.0f));
	return vec3(world.x, world.y, world.z) / world.w;
}

} // namespace refsh

// bgfx's declaration macros.
#define SAMPLER2D(_name, _stage) refsh::Texture _name
#define IMAGE2D_RO(_name, _format, _stage) refsh::Texture _name
#define IMAGE2D_WO(_name, _format, _stage) refsh::Texture _name
#define IMAGE2D_WR(_name, _format, _stage) refsh::Texture _name
#define IMAGE2D_RW(_name, _format, _stage) refsh::Texture _name
#define BUFFER_RO(_name, _type, _stage) refsh::Buffer<_type> _name
#define BUFFER_RW(_name, _type, _stage) refsh::Buffer<_type> _name
#define BUFFER_WO(_name, _type, _stage) refsh::Buffer<_type> _name
#define uniform
// Group-shared memory: one copy per worker thread, which runs one group at a time.
#define SHARED thread_local
#define NUM_THREADS(_x, _y, _z)
#define BGFX_SHADER_LANGUAGE_GLSL 0
#define BGFX_SHADER_LANGUAGE_HLSL 0
#define BGFX_SHADER_LANGUAGE_SPIRV 0

#endif // ORACLE_SHADER_SHIM_H
