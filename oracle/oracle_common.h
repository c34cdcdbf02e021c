/*
 * ORACLE (test infrastructure, never linked into the product).
 *
 * CPU restatement of the reference's shader helpers, line by line in the
 * reference's own order of operations:
 *   shaders/bvh.sh      (traversal, lines 25-339)
 *   shaders/hashgrid.sh (grid keys, lookup and insertion, lines 61-200)
 *   shaders/restir.sh   (GI helpers and pairwise MIS, lines 117-931)
 *   shaders/shadow.sh   (atlas lookup, lines 31-133)
 *   shaders/sky.sh, shaders/brdf.sh, shaders/di.sh
 * with bgfx's shaderlib conventions fixed as the ABI fixes them: NDC depth in
 * [0, 1], texture row 0 at the top unless origin_bottom_left.
 *
 * Parity status: the reference has no tests, golden vectors or known-answer
 * tests for any of this (its CI only checks that a rendered PNG is not
 * blank), and its shaders need bgfx, which is absent, so this restatement is
 * pinned only where the reference's C++ can run here (the BVH and light-list
 * layouts, through oracle/_ref) and by its own known-answer tables
 * (tests/golden). Everything else is "parity unpinned" against the
 * reference itself.
 */
#ifndef ORACLE_COMMON_H
#define ORACLE_COMMON_H

#include "glsl.h"
#include "../include/restir_gpu.h"

#include <atomic>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle
{
using namespace glsl;

/* --- textures: point sampling with clamp -------------------------------- */

inline int texelCoord(float uv, int size)
{
	float f = floor(uv * float(size));
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

inline int texelIndex(vec2 uv, int w, int h)
{
	return texelCoord(uv.y, h) * w + texelCoord(uv.x, w);
}

struct TexF4 // RGBA32F
{
	const float* p = nullptr;
	int w = 0, h = 0;
	vec4 at(int i) const { const float* q = p + 4 * size_t(i); return vec4(q[0], q[1], q[2], q[3]); }
	vec4 sample(vec2 uv) const { return at(texelIndex(uv, w, h)); }
};

struct TexH4 // RGBA16F
{
	const uint16_t* p = nullptr;
	int w = 0, h = 0;
	vec4 at(int i) const
	{
		if (!p)
		{
			return vec4_splat(0.0f);
		}
		const uint16_t* q = p + 4 * size_t(i);
		return vec4(rn_half_to_float(q[0]), rn_half_to_float(q[1]), rn_half_to_float(q[2]), rn_half_to_float(q[3]));
	}
	vec4 sample(vec2 uv) const { return at(texelIndex(uv, w, h)); }
};

struct TexU8 // BGRA8, read back as rgba
{
	const uint8_t* p = nullptr;
	int w = 0, h = 0;
	vec4 at(int i) const
	{
		const uint8_t* q = p + 4 * size_t(i);
		return vec4(rn_unorm8_to_float(q[2]), rn_unorm8_to_float(q[1]), rn_unorm8_to_float(q[0]), rn_unorm8_to_float(q[3]));
	}
	vec4 sample(vec2 uv) const { return at(texelIndex(uv, w, h)); }
};

struct TexF1 // R32F / D32F
{
	const float* p = nullptr;
	int w = 0, h = 0;
	float at(int i) const { return p[i]; }
	float sample(vec2 uv) const { return at(texelIndex(uv, w, h)); }
};

inline void storeF4(float* p, int i, const vec4& v)
{
	float* q = p + 4 * size_t(i);
	q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
}

inline void storeH4(uint16_t* p, int i, const vec4& v)
{
	uint16_t* q = p + 4 * size_t(i);
	q[0] = rn_float_to_half(v.x); q[1] = rn_float_to_half(v.y);
	q[2] = rn_float_to_half(v.z); q[3] = rn_float_to_half(v.w);
}

inline void storeU8(uint8_t* p, int i, const vec4& v)
{
	uint8_t* q = p + 4 * size_t(i);
	q[2] = rn_unorm8(v.x); q[1] = rn_unorm8(v.y); q[0] = rn_unorm8(v.z); q[3] = rn_unorm8(v.w);
}

/* --- random numbers (restir.sh:122-135) --------------------------------- */

inline uint pcg(uint _value)
{
	uint state = _value * 747796405u + 2891336453u;
	uint word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
	return (word >> 22u) ^ word;
}

inline float nextRandom(uint& _state)
{
	_state = pcg(_state);
	return float(_state >> 8u) * (1.0f / 16777216.0f);
}

inline float luminance(vec3 _color)
{
	return dot(_color, vec3(0.2126f, 0.7152f, 0.0722f));
}

#define kPi 3.14159265359f
#define kSkyDepth 0.99999f

/* --- BVH traversal (bvh.sh) --------------------------------------------- */

struct Bvh
{
	const float* data = nullptr;
	int nodeCount = 0;
	int triangleOffset = 0;
	std::atomic<uint32_t>* status = nullptr; // bit 0: step cap reached
	/* Work counters (per thread copy): rays, node visits, triangle tests. */
	mutable uint64_t rays = 0, nodeVisits = 0, triangleTests = 0;

	vec4 row(int i) const { const float* q = data + 4 * size_t(i); return vec4(q[0], q[1], q[2], q[3]); }
	bool available() const { return nodeCount > 0; }
	vec3 vertex(int _triangle, int _corner) const { return row(triangleOffset + _triangle * 4 + _corner).xyz(); }
};

#define kBvhShortStack 8
#define kBvhMaxSteps 2048

inline float intersectBox(vec3 _origin, vec3 _inverseDirection, vec3 _min, vec3 _max, float _maxDistance)
{
	vec3 t0 = (_min - _origin) * _inverseDirection;
	vec3 t1 = (_max - _origin) * _inverseDirection;
	vec3 near_ = min(t0, t1);
	vec3 far_ = max(t0, t1);
	float enter = max(max(near_.x, near_.y), max(near_.z, 0.0f));
	float leave = min(min(far_.x, far_.y), min(far_.z, _maxDistance));
	return enter <= leave ? enter : -1.0f;
}

inline float intersectTriangle(vec3 _origin, vec3 _direction, vec3 _v0, vec3 _v1, vec3 _v2)
{
	vec3 edge1 = _v1 - _v0;
	vec3 edge2 = _v2 - _v0;
	vec3 p = cross(_direction, edge2);
	float determinant = dot(edge1, p);
	if (abs(determinant) < 1e-12f)
	{
		return -1.0f;
	}
	float inverse = 1.0f / determinant;
	vec3 s = _origin - _v0;
	float u = dot(s, p) * inverse;
	if (u < 0.0f || u > 1.0f)
	{
		return -1.0f;
	}
	vec3 q = cross(s, edge1);
	float v = dot(_direction, q) * inverse;
	if (v < 0.0f || u + v > 1.0f)
	{
		return -1.0f;
	}
	return dot(edge2, q) * inverse;
}

inline vec3 bvhInverseDirection(vec3 _direction)
{
	vec3 safe(
		  abs(_direction.x) > 1e-8f ? _direction.x : (_direction.x >= 0.0f ? 1e-8f : -1e-8f)
		, abs(_direction.y) > 1e-8f ? _direction.y : (_direction.y >= 0.0f ? 1e-8f : -1e-8f)
		, abs(_direction.z) > 1e-8f ? _direction.z : (_direction.z >= 0.0f ? 1e-8f : -1e-8f));
	return vec3_splat(1.0f) / safe;
}

inline int bvhIntersectLeaf(const Bvh& b, vec3 _origin, vec3 _direction, int _first, int _count, float& _distance, int _hit)
{
	int hit = _hit;
	b.triangleTests += uint64_t(_count > 0 ? _count : 0);
	for (int t = _first; t < _first + _count; ++t)
	{
		float d = intersectTriangle(_origin, _direction, b.vertex(t, 0), b.vertex(t, 1), b.vertex(t, 2));
		if (d > 0.0f && d < _distance)
		{
			_distance = d;
			hit = t;
		}
	}
	return hit;
}

inline int traceBvhStackless(const Bvh& b, vec3 _origin, vec3 _direction, bool _anyHit, float& _distance)
{
	vec3 inverseDirection = bvhInverseDirection(_direction);
	int hit = -1;
	int node = 0;
	int step = 0;
	for (; step < kBvhMaxSteps; ++step)
	{
		if (node >= b.nodeCount)
		{
			break;
		}
		++b.nodeVisits;
		vec4 node0 = b.row(node * 2);
		vec4 node1 = b.row(node * 2 + 1);
		bool leaf = node1.w >= 0.0f;
		if (intersectBox(_origin, inverseDirection, node0.xyz(), node1.xyz(), _distance) < 0.0f)
		{
			node = leaf ? node + 1 : int(-node1.w) - 1;
			continue;
		}
		if (leaf)
		{
			hit = bvhIntersectLeaf(b, _origin, _direction, int(node0.w), int(node1.w), _distance, hit);
			if (_anyHit && hit >= 0)
			{
				return hit;
			}
		}
		node = node + 1;
	}
	if (step == kBvhMaxSteps && b.status)
	{
		*b.status |= 1u;
	}
	return hit;
}

/* traceBvhWave (bvh.sh:177-212) for a wave of _count lanes: every step the
 * wave takes the smallest node a lane still needs (WaveActiveMin), the lanes
 * at that node test it; the step cap counts the wave's steps. */
inline void traceBvhWave(const Bvh& b, int _count, const vec3* _origin, const vec3* _direction, bool _anyHit,
	float* _distance, int* _hit)
{
	int node[32];
	vec3 inverseDirection[32];
	for (int lane = 0; lane < _count; ++lane)
	{
		inverseDirection[lane] = bvhInverseDirection(_direction[lane]);
		node[lane] = 0;
		_hit[lane] = -1;
	}
	int step = 0;
	for (; step < kBvhMaxSteps; ++step)
	{
		int waveNode = b.nodeCount;
		for (int lane = 0; lane < _count; ++lane)
		{
			waveNode = node[lane] < waveNode ? node[lane] : waveNode;
		}
		if (waveNode >= b.nodeCount)
		{
			break;
		}
		vec4 node0 = b.row(waveNode * 2);
		vec4 node1 = b.row(waveNode * 2 + 1);
		bool leaf = node1.w >= 0.0f;
		for (int lane = 0; lane < _count; ++lane)
		{
			if (node[lane] != waveNode)
			{
				continue;
			}
			++b.nodeVisits;
			if (intersectBox(_origin[lane], inverseDirection[lane], node0.xyz(), node1.xyz(), _distance[lane]) < 0.0f)
			{
				node[lane] = leaf ? node[lane] + 1 : int(-node1.w) - 1;
				continue;
			}
			if (leaf)
			{
				_hit[lane] = bvhIntersectLeaf(b, _origin[lane], _direction[lane], int(node0.w), int(node1.w), _distance[lane],
					_hit[lane]);
			}
			node[lane] = _anyHit && _hit[lane] >= 0 ? b.nodeCount : node[lane] + 1;
		}
	}
	if (step == kBvhMaxSteps && b.status)
	{
		*b.status |= 1u;
	}
}

inline int traceBvhSharedStack(const Bvh& b, vec3 _origin, vec3 _direction, float& _distance)
{
	vec3 inverseDirection = bvhInverseDirection(_direction);
	if (intersectBox(_origin, inverseDirection, b.row(0).xyz(), b.row(1).xyz(), _distance) < 0.0f)
	{
		return -1;
	}
	int stack[kBvhShortStack];
	int stackTop = 0;
	int stackCount = 0;
	bool dropped = false;
	int hit = -1;
	int node = 0;
	int step = 0;
	for (; step < kBvhMaxSteps; ++step)
	{
		vec4 node0 = b.row(node * 2);
		vec4 node1 = b.row(node * 2 + 1);
		b.nodeVisits += node1.w >= 0.0f ? 1 : 2; // an interior node reads both children
		if (node1.w >= 0.0f)
		{
			hit = bvhIntersectLeaf(b, _origin, _direction, int(node0.w), int(node1.w), _distance, hit);
		}
		else
		{
			int left = node + 1;
			int right = int(node0.w);
			float leftDistance = intersectBox(_origin, inverseDirection, b.row(left * 2).xyz(), b.row(left * 2 + 1).xyz(), _distance);
			float rightDistance = intersectBox(_origin, inverseDirection, b.row(right * 2).xyz(), b.row(right * 2 + 1).xyz(), _distance);
			bool visitLeft = leftDistance >= 0.0f;
			bool visitRight = rightDistance >= 0.0f;
			if (visitLeft && visitRight)
			{
				bool leftFirst = leftDistance <= rightDistance;
				stack[stackTop & (kBvhShortStack - 1)] = leftFirst ? right : left;
				++stackTop;
				if (stackCount == kBvhShortStack)
				{
					dropped = true;
				}
				else
				{
					++stackCount;
				}
				node = leftFirst ? left : right;
				continue;
			}
			if (visitLeft || visitRight)
			{
				node = visitLeft ? left : right;
				continue;
			}
		}
		if (stackCount == 0)
		{
			break;
		}
		--stackTop;
		--stackCount;
		node = stack[stackTop & (kBvhShortStack - 1)];
	}
	if (step == kBvhMaxSteps && b.status)
	{
		*b.status |= 1u;
	}
	if (dropped)
	{
		int stacklessHit = traceBvhStackless(b, _origin, _direction, false, _distance);
		if (stacklessHit >= 0)
		{
			hit = stacklessHit;
		}
	}
	return hit;
}

/* traceBvh with BVH_SHARED_STACK defined (the GI temporal pass) or not. */
inline int traceBvh(const Bvh& b, vec3 _origin, vec3 _direction, float _maxDistance, bool _anyHit, float& _distance, bool _sharedStack)
{
	_distance = _maxDistance;
	if (!b.available())
	{
		return -1;
	}
	++b.rays;
	if (_sharedStack && !_anyHit)
	{
		return traceBvhSharedStack(b, _origin, _direction, _distance);
	}
	return traceBvhStackless(b, _origin, _direction, _anyHit, _distance);
}

/* Watertight ray/triangle test (Woop, Benthin and Wald, JCGT 2(1), 2013),
 * the production alternative the ABI offers to bvh.sh's Moeller-Trumbore:
 * distance in (0, tmax] or -1. */
inline float component(vec3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

inline float intersectWatertight(vec3 _origin, vec3 _direction, vec3 _v0, vec3 _v1, vec3 _v2, float _tmax)
{
	vec3 a = abs(_direction);
	int kz = a.x > a.y ? (a.x > a.z ? 0 : 2) : (a.y > a.z ? 1 : 2);
	int kx = kz + 1 == 3 ? 0 : kz + 1;
	int ky = kx + 1 == 3 ? 0 : kx + 1;
	if (component(_direction, kz) < 0.0f)
	{
		int t = kx;
		kx = ky;
		ky = t;
	}
	float sx = component(_direction, kx) / component(_direction, kz);
	float sy = component(_direction, ky) / component(_direction, kz);
	float sz = 1.0f / component(_direction, kz);
	vec3 A = _v0 - _origin, B = _v1 - _origin, C = _v2 - _origin;
	float az = component(A, kz), bz = component(B, kz), cz = component(C, kz);
	float ax = component(A, kx) - sx * az;
	float ay = component(A, ky) - sy * az;
	float bx = component(B, kx) - sx * bz;
	float by = component(B, ky) - sy * bz;
	float cx = component(C, kx) - sx * cz;
	float cy = component(C, ky) - sy * cz;
	float u = cx * by - cy * bx;
	float v = ax * cy - ay * cx;
	float w = bx * ay - by * ax;
	if (u == 0.0f || v == 0.0f || w == 0.0f)
	{
		u = float(double(cx) * double(by) - double(cy) * double(bx));
		v = float(double(ax) * double(cy) - double(ay) * double(cx));
		w = float(double(bx) * double(ay) - double(by) * double(ax));
	}
	if ((u < 0.0f || v < 0.0f || w < 0.0f) && (u > 0.0f || v > 0.0f || w > 0.0f))
	{
		return -1.0f;
	}
	float det = u + v + w;
	if (det == 0.0f)
	{
		return -1.0f;
	}
	float t = u * (sz * az) + v * (sz * bz) + w * (sz * cz);
	float sign = det < 0.0f ? -1.0f : 1.0f;
	if (t * sign <= 0.0f || t * sign > _tmax * (det * sign))
	{
		return -1.0f;
	}
	return t / det;
}

/* Nearest hit in (0, distance) among the triangles _accept lets through,
 * ties to the lower triangle index, nearest child first with a full stack
 * (the order of the kernels' traversal, so that box culling decides alike).
 * _test(t, distance) is the triangle test; _conservative widens each box's
 * exit distance by 1 + 2 gamma_3 (Ize, "Robust BVH Ray Traversal", JCGT
 * 2(2), 2013) for the watertight mode. */
template<typename Test, typename Accept>
int traceNearestFirst(const Bvh& b, vec3 _origin, vec3 _direction, float& _distance, bool _conservative, Test _test,
	Accept _accept)
{
	vec3 inv = bvhInverseDirection(_direction);
	const float widen = _conservative ? 1.00000036f : 1.0f;
	auto box = [&](int node) -> float
	{
		vec3 t0 = (b.row(node * 2).xyz() - _origin) * inv;
		vec3 t1 = (b.row(node * 2 + 1).xyz() - _origin) * inv;
		vec3 n = min(t0, t1);
		vec3 f = max(t0, t1);
		float enter = max(max(n.x, n.y), max(n.z, 0.0f));
		float leave = min(min(f.x, f.y), f.z) * widen;
		leave = min(leave, _distance);
		return enter <= leave ? enter : -1.0f;
	};
	if (!b.available() || box(0) < 0.0f)
	{
		return -1;
	}
	std::vector<int> stack;
	int hit = -1;
	int node = 0;
	for (;;)
	{
		vec4 node0 = b.row(node * 2);
		vec4 node1 = b.row(node * 2 + 1);
		if (node1.w >= 0.0f)
		{
			int first = int(node0.w), count = int(node1.w);
			for (int t = first; t < first + count; ++t)
			{
				float h = _test(t, _distance);
				if (h > 0.0f && (h < _distance || (h == _distance && hit >= 0 && t < hit)) && _accept(t))
				{
					_distance = h;
					hit = t;
				}
			}
		}
		else
		{
			int left = node + 1;
			int right = int(node0.w);
			float leftDistance = box(left);
			float rightDistance = box(right);
			bool visitLeft = leftDistance >= 0.0f;
			bool visitRight = rightDistance >= 0.0f;
			if (visitLeft && visitRight)
			{
				bool leftFirst = leftDistance <= rightDistance;
				stack.push_back(leftFirst ? right : left);
				node = leftFirst ? left : right;
				continue;
			}
			if (visitLeft || visitRight)
			{
				node = visitLeft ? left : right;
				continue;
			}
		}
		bool found = false;
		while (!stack.empty())
		{
			int candidate = stack.back();
			stack.pop_back();
			if (box(candidate) >= 0.0f)
			{
				node = candidate;
				found = true;
				break;
			}
		}
		if (!found)
		{
			break;
		}
	}
	return hit;
}

/* Nearest watertight hit, ties to the lower triangle index. */
inline int traceWatertight(const Bvh& b, vec3 _origin, vec3 _direction, float& _distance)
{
	return traceNearestFirst(b, _origin, _direction, _distance, true,
		[&](int t, float tmax) { return intersectWatertight(_origin, _direction, b.vertex(t, 0), b.vertex(t, 1), b.vertex(t, 2), tmax); },
		[](int) { return true; });
}

inline vec3 bvhTriangleAlbedo(const Bvh& b, int _triangle)
{
	return b.row(b.triangleOffset + _triangle * 4 + 3).xyz();
}

inline vec3 bvhTriangleEmission(const Bvh& b, int _triangle)
{
	int base = b.triangleOffset + _triangle * 4;
	return vec3(b.row(base + 1).w, b.row(base + 2).w, b.row(base + 3).w);
}

/* --- hash grid (hashgrid.sh) -------------------------------------------- */

#define kGridInvalid 0xffffffffu
#define kGridMaxProbes 8u

inline uint gridHash(uint _value)
{
	uint state = _value * 747796405u + 2891336453u;
	uint word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
	return (word >> 22u) ^ word;
}

inline uint gridChecksumHash(uint _value)
{
	_value ^= _value >> 15u;
	_value *= 2246822519u;
	_value ^= _value >> 13u;
	_value *= 3266489917u;
	_value ^= _value >> 16u;
	return _value;
}

struct Grid
{
	float minCell = 0.0f;     // u_gridInfo.x
	float pixelSize = 0.0f;   // u_gridInfo.y
	float cellPixels = 0.0f;  // u_gridInfo.z
	bool worldSpace = true;   // u_gridInfo.w
	vec3 camera;              // u_gridCamera.xyz
	uint tableSize = 65536u;
	uint capacity = 32u;
	uint32_t* data = nullptr;

	uint mask() const { return tableSize - 1u; }

	/* floor(log2(...)) from the exponent and exp2 of an integer (exact), as
	 * the numeric conventions fix them. */
	float cellSize(vec3 _position) const
	{
		float target = distance(_position, camera) * pixelSize * cellPixels;
		float level = float(rn_floor_log2(max(target / minCell, 1.0f)));
		return minCell * rn_exp2i(int(level));
	}

	static uint normalBucket(vec3 _normal)
	{
		vec3 absolute = abs(_normal);
		uint bucket = _normal.z >= 0.0f ? 4u : 5u;
		if (absolute.x >= absolute.y && absolute.x >= absolute.z)
		{
			bucket = _normal.x >= 0.0f ? 0u : 1u;
		}
		else if (absolute.y >= absolute.z)
		{
			bucket = _normal.y >= 0.0f ? 2u : 3u;
		}
		return bucket;
	}

	static vec3 jitter(vec3 _position, vec3 _normal, float _cellSize, float _random0, float _random1)
	{
		vec3 tangent = normalize(abs(_normal.y) < 0.99f
			? cross(_normal, vec3(0.0f, 1.0f, 0.0f))
			: cross(_normal, vec3(1.0f, 0.0f, 0.0f)));
		vec3 bitangent = cross(_normal, tangent);
		return _position + (tangent * (_random0 - 0.5f) + bitangent * (_random1 - 0.5f)) * _cellSize;
	}

	void key(vec3 _position, vec3 _normal, float _cellSize, uint& _slot, uint& _checksum) const
	{
		vec3 c = floor(_position / _cellSize);
		int cx = int(c.x), cy = int(c.y), cz = int(c.z);
		uint level = floatBitsToUint(_cellSize);
		uint bucket = normalBucket(_normal);
		_slot = gridHash(level + gridHash(bucket + gridHash(uint(cx) + gridHash(uint(cy) + gridHash(uint(cz)))))) & mask();
		uint checksum = gridChecksumHash(level ^ gridChecksumHash(bucket ^ gridChecksumHash(
			uint(cx) ^ gridChecksumHash(uint(cy) ^ gridChecksumHash(uint(cz) + 0x9e3779b9u)))));
		_checksum = max(checksum, 1u);
	}

	uint findCell(uint _slot, uint _checksum) const
	{
		for (uint probe = 0u; probe < kGridMaxProbes; ++probe)
		{
			uint slot = (_slot + probe) & mask();
			uint stored = data[slot];
			if (stored == _checksum)
			{
				return slot;
			}
			if (stored == 0u)
			{
				break;
			}
		}
		return kGridInvalid;
	}

	uint pickEntry(vec3 _position, vec3 _normal, float _random0, float _random1, float _random2) const
	{
		float size = cellSize(_position);
		vec3 jittered = jitter(_position, _normal, size, _random0, _random1);
		uint slot, checksum;
		key(jittered, _normal, size, slot, checksum);
		uint cell = findCell(slot, checksum);
		if (cell == kGridInvalid)
		{
			return kGridInvalid;
		}
		uint count = min(data[tableSize + cell], capacity);
		if (count == 0u)
		{
			return kGridInvalid;
		}
		uint index = min(uint(_random2 * float(count)), count - 1u);
		return data[2u * tableSize + cell * capacity + index];
	}

	/* Sequential insertion, in the order of the calls: with calls in
	 * increasing pixel order a cell lists its lowest indices, sorted, which
	 * is the deterministic mode of the ABI. Returns false when the probes
	 * ran out. */
	bool insert(uint _slot, uint _checksum, uint _entry)
	{
		for (uint probe = 0u; probe < kGridMaxProbes; ++probe)
		{
			uint slot = (_slot + probe) & mask();
			uint previous = data[slot];
			if (previous == 0u)
			{
				data[slot] = _checksum;
			}
			if (previous == 0u || previous == _checksum)
			{
				uint index = data[tableSize + slot]++;
				if (index < capacity)
				{
					data[2u * tableSize + slot * capacity + index] = _entry;
				}
				return true;
			}
		}
		return false;
	}
};

} // namespace oracle

#endif // ORACLE_COMMON_H
