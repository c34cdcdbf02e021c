// Device-side building blocks shared by every pass: vector arithmetic in the
// ABI's fixed order of operations (include/restir_numeric.h), texel fetches
// of the ABI's image formats, the reference's PCG stream, and the device
// status word.
//
// The kernels are compiled with --fmad=false and IEEE division and square
// root, so that each expression below is the same sequence of rounded
// binary32 operations the CPU restatement performs.
#pragma once

#include "../../include/restir_gpu.h"
#include "../../include/restir_numeric.h"

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace restir
{

// --- vectors -----------------------------------------------------------------

struct V2
{
	float x, y;
};

struct V3
{
	float x, y, z;
};

struct V4
{
	float x, y, z, w;
	__device__ __forceinline__ V3 xyz() const { return { x, y, z }; }
};

__device__ __forceinline__ V2 v2(float x, float y) { return { x, y }; }
__device__ __forceinline__ V3 v3(float x, float y, float z) { return { x, y, z }; }
__device__ __forceinline__ V3 v3s(float s) { return { s, s, s }; }
__device__ __forceinline__ V4 v4(float x, float y, float z, float w) { return { x, y, z, w }; }
__device__ __forceinline__ V4 v4(V3 a, float w) { return { a.x, a.y, a.z, w }; }

__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return { a.x * b.x, a.y * b.y, a.z * b.z }; }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return { a.x / b.x, a.y / b.y, a.z / b.z }; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return { a.x * s, a.y * s, a.z * s }; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return { a.x / s, a.y / s, a.z / s }; }
__device__ __forceinline__ V3 operator-(V3 a, float s) { return { a.x - s, a.y - s, a.z - s }; }
__device__ __forceinline__ V3 operator+(V3 a, float s) { return { a.x + s, a.y + s, a.z + s }; }
__device__ __forceinline__ V3 operator-(V3 a) { return { -a.x, -a.y, -a.z }; }

__device__ __forceinline__ V2 operator+(V2 a, V2 b) { return { a.x + b.x, a.y + b.y }; }
__device__ __forceinline__ V2 operator-(V2 a, V2 b) { return { a.x - b.x, a.y - b.y }; }
__device__ __forceinline__ V2 operator*(V2 a, V2 b) { return { a.x * b.x, a.y * b.y }; }
__device__ __forceinline__ V2 operator*(V2 a, float s) { return { a.x * s, a.y * s }; }
__device__ __forceinline__ V2 operator/(V2 a, float s) { return { a.x / s, a.y / s }; }
__device__ __forceinline__ V2 operator+(V2 a, float s) { return { a.x + s, a.y + s }; }
__device__ __forceinline__ V2 operator-(V2 a, float s) { return { a.x - s, a.y - s }; }

__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b)
{
	return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
}
__device__ __forceinline__ float inversesqrt(float x) { return 1.0f / sqrtf(x); }
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float distance(V3 a, V3 b) { return length(a - b); }
__device__ __forceinline__ V3 normalize(V3 a) { return a * inversesqrt(dot(a, a)); }
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return { fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z) }; }
__device__ __forceinline__ V3 vmax(V3 a, V3 b) { return { fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z) }; }
__device__ __forceinline__ V3 vabs(V3 a) { return { fabsf(a.x), fabsf(a.y), fabsf(a.z) }; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ V3 mix(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float stepf(float edge, float x) { return x < edge ? 0.0f : 1.0f; }

__device__ __forceinline__ float luminance(V3 c)
{
	return dot(c, v3(0.2126f, 0.7152f, 0.0722f));
}

// --- matrices (row-major, clip = M * v) --------------------------------------

__device__ __forceinline__ V4 mul(const float* m, V4 v)
{
	return {
		  m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3] * v.w
		, m[4] * v.x + m[5] * v.y + m[6] * v.z + m[7] * v.w
		, m[8] * v.x + m[9] * v.y + m[10] * v.z + m[11] * v.w
		, m[12] * v.x + m[13] * v.y + m[14] * v.z + m[15] * v.w };
}

// Only the w row (clip.w), with the same products and sums as mul().
__device__ __forceinline__ float mulW(const float* m, V3 p)
{
	return m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15] * 1.0f;
}

// --- random numbers (restir.sh:122-135) --------------------------------------

__device__ __forceinline__ uint32_t pcg(uint32_t v)
{
	uint32_t state = v * 747796405u + 2891336453u;
	uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
	return (word >> 22u) ^ word;
}

__device__ __forceinline__ float nextRandom(uint32_t& state)
{
	state = pcg(state);
	return float(state >> 8u) * (1.0f / 16777216.0f);
}

// --- image fetches (point sampling with clamp) -------------------------------

__device__ __forceinline__ int texelCoord(float uv, int size)
{
	float f = floorf(uv * float(size));
	if (!(f >= 0.0f))
	{
		return 0;
	}
	if (f > float(size - 1))
	{
		return size - 1;
	}
	return int(f);
}

__device__ __forceinline__ int texelIndex(V2 uv, int w, int h)
{
	return texelCoord(uv.y, h) * w + texelCoord(uv.x, w);
}

__device__ __forceinline__ V4 loadF4(const float* p, int i)
{
	float4 q = __ldg(reinterpret_cast<const float4*>(p) + i);
	return { q.x, q.y, q.z, q.w };
}

// A buffer this launch also writes: no read-only path.
__device__ __forceinline__ V4 loadF4rw(const float* p, int i)
{
	float4 q = reinterpret_cast<const float4*>(p)[i];
	return { q.x, q.y, q.z, q.w };
}

__device__ __forceinline__ void storeF4(float* p, int i, V4 v)
{
	reinterpret_cast<float4*>(p)[i] = make_float4(v.x, v.y, v.z, v.w);
}

__device__ __forceinline__ V4 loadH4(const uint16_t* p, int i)
{
	if (p == nullptr)
	{
		return { 0.0f, 0.0f, 0.0f, 0.0f };
	}
	uint2 q = __ldg(reinterpret_cast<const uint2*>(p) + i);
	__half2 lo = *reinterpret_cast<__half2*>(&q.x);
	__half2 hi = *reinterpret_cast<__half2*>(&q.y);
	float2 a = __half22float2(lo);
	float2 b = __half22float2(hi);
	return { a.x, a.y, b.x, b.y };
}

// The conversion rounds to nearest even like rn_float_to_half; a NaN becomes
// that function's quiet NaN (sign | 0x7e00) rather than the converter's
// canonical one, so that NaN passed through a target keeps the same bits.
__device__ __forceinline__ uint32_t halfPair(float a, float b)
{
	__half2 h = __floats2half2_rn(a, b);
	uint32_t q = *reinterpret_cast<uint32_t*>(&h);
	if (a != a)
	{
		q = (q & 0xffff0000u) | ((__float_as_uint(a) >> 16) & 0x8000u) | 0x7e00u;
	}
	if (b != b)
	{
		q = (q & 0x0000ffffu) | (((__float_as_uint(b) >> 16) & 0x8000u) | 0x7e00u) << 16;
	}
	return q;
}

__device__ __forceinline__ void storeH4(uint16_t* p, int i, V4 v)
{
	uint2 q;
	q.x = halfPair(v.x, v.y);
	q.y = halfPair(v.z, v.w);
	reinterpret_cast<uint2*>(p)[i] = q;
}

// BGRA8 bytes, read back as (r, g, b, a).
__device__ __forceinline__ V4 loadU8(const uint8_t* p, int i)
{
	uint32_t q = __ldg(reinterpret_cast<const uint32_t*>(p) + i);
	return {
		  float((q >> 16) & 0xffu) / 255.0f
		, float((q >> 8) & 0xffu) / 255.0f
		, float(q & 0xffu) / 255.0f
		, float(q >> 24) / 255.0f };
}

__device__ __forceinline__ void storeU8(uint8_t* p, int i, V4 v)
{
	uint32_t q = uint32_t(rn_unorm8(v.z)) | (uint32_t(rn_unorm8(v.y)) << 8)
		| (uint32_t(rn_unorm8(v.x)) << 16) | (uint32_t(rn_unorm8(v.w)) << 24);
	reinterpret_cast<uint32_t*>(p)[i] = q;
}

__device__ __forceinline__ float loadF1(const float* p, int i)
{
	return __ldg(p + i);
}

#define kPi 3.14159265359f
#define kSkyDepth 0.99999f
#define kSkySampleId 30000000.0f

// --- device status word ------------------------------------------------------

// Bit 0: a traversal reached its step cap; bit 1: a grid insertion found no
// free slot within its probes. Read and cleared by restir_status().
extern __device__ unsigned int g_restirStatus;

__device__ __forceinline__ void raiseStatus(unsigned int bit)
{
	atomicOr(&g_restirStatus, bit);
}

// --- work counters -----------------------------------------------------------

// Rays by kind, and the node fetches and triangle tests of every BVH ray,
// counted only while g_restirCounting is set (restir_counters), so that
// timed frames do none of this work.
#define RESTIR_COUNT_PRIMARY 0    // nearest-hit ray casts (G-buffer, shadow atlas, restir_trace)
#define RESTIR_COUNT_CLOSEST 1    // short-stack closest-hit rays (GI candidates)
#define RESTIR_COUNT_ANY 2        // stackless rays (visibility and shadow rays)
#define RESTIR_COUNT_SCREEN 3     // depth-buffer marches
#define RESTIR_COUNT_NODES 4
#define RESTIR_COUNT_TRIANGLES 5
#define RESTIR_COUNT_SCREEN_STEPS 6
#define RESTIR_COUNT_STEP_CAPPED 7  // rays cut short: the step cap, or a full traversal stack
#define RESTIR_COUNTERS 8

extern __device__ unsigned long long g_restirCounters[RESTIR_COUNTERS];
extern __device__ int g_restirCounting;

__device__ __forceinline__ void countWork(int kind, uint32_t nodes, uint32_t triangles)
{
	if (!g_restirCounting)
	{
		return;
	}
	const unsigned mask = __activemask();
	const unsigned n = __reduce_add_sync(mask, nodes);
	const unsigned t = __reduce_add_sync(mask, triangles);
	if (int(threadIdx.x & 31u) == __ffs(mask) - 1)
	{
		atomicAdd(&g_restirCounters[kind], static_cast<unsigned long long>(__popc(mask)));
		atomicAdd(&g_restirCounters[kind == RESTIR_COUNT_SCREEN ? RESTIR_COUNT_SCREEN_STEPS : RESTIR_COUNT_NODES],
			static_cast<unsigned long long>(n));
		if (kind != RESTIR_COUNT_SCREEN)
		{
			atomicAdd(&g_restirCounters[RESTIR_COUNT_TRIANGLES], static_cast<unsigned long long>(t));
		}
	}
}

// Bounds-checked builds (RESTIR_CHECKS=1: python -m restir_b200.build
// --checks, librestir_gpu_checked.so), the stand-in for a memory checker:
// every BVH row and light-list row index is tested before the load; one out
// of range raises status bit 4 and reads zeros instead, so a broken input is
// reported, not followed outside its buffer. Off in the product build.
#ifndef RESTIR_CHECKS
#define RESTIR_CHECKS 0
#endif

__device__ __forceinline__ bool checkedIndex(uint32_t index, uint32_t count)
{
#if RESTIR_CHECKS
	if (index >= count)
	{
		raiseStatus(16u);
		return false;
	}
#else
	(void)index;
	(void)count;
#endif
	return true;
}

// A traversal stopped short (the 2,048-visit cap, bvh.sh:23, or a full
// traversal stack): status bit 0, and one ray counted while counting is on.
__device__ __forceinline__ void reportTruncatedRay()
{
	raiseStatus(1u);
	if (g_restirCounting)
	{
		atomicAdd(&g_restirCounters[RESTIR_COUNT_STEP_CAPPED], 1ull);
	}
}

// --- launch helpers ----------------------------------------------------------

inline cudaStream_t asStream(void* s)
{
	return reinterpret_cast<cudaStream_t>(s);
}

inline int launchStatus()
{
	return cudaGetLastError() == cudaSuccess ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
}

} // namespace restir
