// BVH traversal over the reference's depth-first node layout (src/bvh.h:7-22):
// node i = float4 rows 2i, 2i+1: (min.xyz, a), (max.xyz, b); b >= 0 a leaf of
// triangles [a, a+b), b < 0 an interior node with right child a and skip
// link -b-1; triangle t = rows triangleOffset + 4t .. +3.
//
// Same algorithms and arithmetic as shaders/bvh.sh (slab test 32-41,
// Moeller-Trumbore 44-71, stackless walk 140-174, nearest-first short stack
// 216-295), so hit ids and distances are bit-identical to the CPU
// restatement. Every node and triangle row is one 16-byte read-only load.
#pragma once

#include "common.cuh"

namespace restir
{

#define kBvhShortStack 8
#define kBvhMaxSteps 2048

struct BvhView
{
	const float4* rows = nullptr;
	int nodeCount = 0;
	int triangleOffset = 0;
	int rowCount = 0;   // nodes x 2 + triangles x 4 (checked builds test indices against it)

	__device__ __forceinline__ bool available() const { return nodeCount > 0; }
	__device__ __forceinline__ V4 row(int i) const
	{
		if (!checkedIndex(uint32_t(i), uint32_t(rowCount)))
		{
			return { 0.0f, 0.0f, 0.0f, 0.0f };
		}
		float4 q = __ldg(rows + i);
		return { q.x, q.y, q.z, q.w };
	}
	__device__ __forceinline__ V3 vertex(int t, int corner) const { return row(triangleOffset + t * 4 + corner).xyz(); }
	__device__ __forceinline__ V3 albedo(int t) const { return row(triangleOffset + t * 4 + 3).xyz(); }
	__device__ __forceinline__ V3 emission(int t) const
	{
		int base = triangleOffset + t * 4;
		return v3(row(base + 1).w, row(base + 2).w, row(base + 3).w);
	}
};

__host__ __device__ inline BvhView makeBvhView(const RestirScene* s)
{
	BvhView b;
	if (s != nullptr && s->bvh != nullptr)
	{
		b.rows = reinterpret_cast<const float4*>(s->bvh);
		b.nodeCount = int(s->node_count);
		b.triangleOffset = int(s->triangle_offset);
		b.rowCount = int(s->triangle_offset + 4u * s->triangle_count);
	}
	return b;
}

// Node fetches and triangle tests of one ray, for the work counters.
struct TraceWork
{
	uint32_t nodes = 0;
	uint32_t triangles = 0;
};

__device__ __forceinline__ float intersectBox(V3 o, V3 inv, V3 bmin, V3 bmax, float maxDistance)
{
	V3 t0 = (bmin - o) * inv;
	V3 t1 = (bmax - o) * inv;
	V3 n = vmin(t0, t1);
	V3 f = vmax(t0, t1);
	float enter = fmaxf(fmaxf(n.x, n.y), fmaxf(n.z, 0.0f));
	float leave = fminf(fminf(f.x, f.y), fminf(f.z, maxDistance));
	return enter <= leave ? enter : -1.0f;
}

__device__ __forceinline__ float intersectTriangle(V3 o, V3 d, V3 v0, V3 v1, V3 v2)
{
	V3 edge1 = v1 - v0;
	V3 edge2 = v2 - v0;
	V3 p = cross(d, edge2);
	float determinant = dot(edge1, p);
	if (fabsf(determinant) < 1e-12f)
	{
		return -1.0f;
	}
	float inverse = 1.0f / determinant;
	V3 s = o - v0;
	float u = dot(s, p) * inverse;
	if (u < 0.0f || u > 1.0f)
	{
		return -1.0f;
	}
	V3 q = cross(s, edge1);
	float v = dot(d, q) * inverse;
	if (v < 0.0f || u + v > 1.0f)
	{
		return -1.0f;
	}
	return dot(edge2, q) * inverse;
}

__device__ __forceinline__ float safeInverse(float d)
{
	float s = fabsf(d) > 1e-8f ? d : (d >= 0.0f ? 1e-8f : -1e-8f);
	return 1.0f / s;
}

__device__ __forceinline__ V3 bvhInverseDirection(V3 d)
{
	return { safeInverse(d.x), safeInverse(d.y), safeInverse(d.z) };
}

__device__ __forceinline__ int intersectLeaf(const BvhView& b, V3 o, V3 d, int first, int count, float& distance, int hit,
	TraceWork& work)
{
	work.triangles += uint32_t(count);
	for (int t = first; t < first + count; ++t)
	{
		float h = intersectTriangle(o, d, b.vertex(t, 0), b.vertex(t, 1), b.vertex(t, 2));
		if (h > 0.0f && h < distance)
		{
			distance = h;
			hit = t;
		}
	}
	return hit;
}

// bvh.sh:140-174
__device__ inline int traceStacklessWalk(const BvhView& b, V3 o, V3 d, bool anyHit, float& distance, TraceWork& work)
{
	V3 inv = bvhInverseDirection(d);
	int hit = -1;
	int node = 0;
	int step = 0;
	for (; step < kBvhMaxSteps; ++step)
	{
		if (node >= b.nodeCount)
		{
			break;
		}
		++work.nodes;
		V4 node0 = b.row(node * 2);
		V4 node1 = b.row(node * 2 + 1);
		bool leaf = node1.w >= 0.0f;
		if (intersectBox(o, inv, node0.xyz(), node1.xyz(), distance) < 0.0f)
		{
			node = leaf ? node + 1 : int(-node1.w) - 1;
			continue;
		}
		if (leaf)
		{
			hit = intersectLeaf(b, o, d, int(node0.w), int(node1.w), distance, hit, work);
			if (anyHit && hit >= 0)
			{
				return hit;
			}
		}
		node = node + 1;
	}
	if (step == kBvhMaxSteps)
	{
		reportTruncatedRay();
	}
	return hit;
}

// traceBvhWave (bvh.sh:177-212), the visibility rays of the reference's
// Vulkan build: the lanes that call it walk the skip-link order in lock
// step. Each step the warp takes the smallest node any lane still needs
// (__reduce_min_sync; a finished lane asks for nodeCount), and the lanes at
// that node test it while the others wait, so lanes on the same part of the
// tree share every node fetch. A lane visits its nodes in the stackless
// walk's order, so its hit is the stackless walk's; only the step cap counts
// the warp's steps.
__device__ inline int traceStacklessWave(const BvhView& b, V3 o, V3 d, bool anyHit, float& distance, TraceWork& work)
{
	const unsigned mask = __activemask();
	V3 inv = bvhInverseDirection(d);
	const int nodeCount = b.nodeCount;
	int hit = -1;
	int node = 0;
	int step = 0;
	for (; step < kBvhMaxSteps; ++step)
	{
		const int waveNode = int(__reduce_min_sync(mask, unsigned(node)));
		if (waveNode >= nodeCount)
		{
			break;
		}
		if (node == waveNode)
		{
			++work.nodes;
			V4 node0 = b.row(waveNode * 2);
			V4 node1 = b.row(waveNode * 2 + 1);
			bool leaf = node1.w >= 0.0f;
			if (intersectBox(o, inv, node0.xyz(), node1.xyz(), distance) < 0.0f)
			{
				node = leaf ? node + 1 : int(-node1.w) - 1;
			}
			else
			{
				if (leaf)
				{
					hit = intersectLeaf(b, o, d, int(node0.w), int(node1.w), distance, hit, work);
				}
				node = anyHit && hit >= 0 ? nodeCount : node + 1;
			}
		}
	}
	if (step == kBvhMaxSteps)
	{
		reportTruncatedRay();
	}
	return hit;
}

// bvh.sh:216-295. stack: this thread's kBvhShortStack entries, stride apart
// (shared memory, interleaved across the block's threads).
__device__ inline int traceShortStack(const BvhView& b, V3 o, V3 d, float& distance, int* stack, int stride, TraceWork& work)
{
	V3 inv = bvhInverseDirection(d);
	++work.nodes;
	if (intersectBox(o, inv, b.row(0).xyz(), b.row(1).xyz(), distance) < 0.0f)
	{
		return -1;
	}
	int stackTop = 0;
	int stackCount = 0;
	bool dropped = false;
	int hit = -1;
	int node = 0;
	int step = 0;
	for (; step < kBvhMaxSteps; ++step)
	{
		V4 node0 = b.row(node * 2);
		V4 node1 = b.row(node * 2 + 1);
		if (node1.w >= 0.0f)
		{
			hit = intersectLeaf(b, o, d, int(node0.w), int(node1.w), distance, hit, work);
		}
		else
		{
			int left = node + 1;
			int right = int(node0.w);
			work.nodes += 2u;
			float leftDistance = intersectBox(o, inv, b.row(left * 2).xyz(), b.row(left * 2 + 1).xyz(), distance);
			float rightDistance = intersectBox(o, inv, b.row(right * 2).xyz(), b.row(right * 2 + 1).xyz(), distance);
			bool visitLeft = leftDistance >= 0.0f;
			bool visitRight = rightDistance >= 0.0f;
			if (visitLeft && visitRight)
			{
				bool leftFirst = leftDistance <= rightDistance;
				stack[(stackTop & (kBvhShortStack - 1)) * stride] = leftFirst ? right : left;
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
		node = stack[(stackTop & (kBvhShortStack - 1)) * stride];
	}
	if (step == kBvhMaxSteps)
	{
		reportTruncatedRay();
	}
	if (dropped)
	{
		int stacklessHit = traceStacklessWalk(b, o, d, false, distance, work);
		if (stacklessHit >= 0)
		{
			hit = stacklessHit;
		}
	}
	return hit;
}

// traceBvh (bvh.sh:298-319). stack == nullptr: stackless for every ray (the
// passes without BVH_SHARED_STACK).
__device__ __forceinline__ int traceBvh(const BvhView& b, V3 o, V3 d, float maxDistance, bool anyHit, float& distance,
	int* stack, int stride)
{
	distance = maxDistance;
	if (!b.available())
	{
		return -1;
	}
	TraceWork work;
	int hit;
	int kind;
	if (stack != nullptr && !anyHit)
	{
		hit = traceShortStack(b, o, d, distance, stack, stride, work);
		kind = RESTIR_COUNT_CLOSEST;
	}
	else
	{
		hit = traceStacklessWalk(b, o, d, anyHit, distance, work);
		kind = RESTIR_COUNT_ANY;
	}
	countWork(kind, work.nodes, work.triangles);
	return hit;
}

// A visibility (any-hit) ray: traceBvh's stackless walk, or with wave set
// the warp-lock-step walk of the reference's Vulkan build (same hits).
__device__ __forceinline__ int traceVisibility(const BvhView& b, V3 o, V3 d, float maxDistance, float& distance, bool wave)
{
	if (!wave)
	{
		return traceBvh(b, o, d, maxDistance, true, distance, nullptr, 0);
	}
	distance = maxDistance;
	if (!b.available())
	{
		return -1;
	}
	TraceWork work;
	const int hit = traceStacklessWave(b, o, d, true, distance, work);
	countWork(RESTIR_COUNT_ANY, work.nodes, work.triangles);
	return hit;
}

// Nearest hit in (0, distance) among the triangles accept() lets through,
// ties to the lower triangle index, nearest child first with a full stack of
// 64 entries in local memory (the layout's depth is at most 40, bvh.h:49).
// test(t, distance) is the triangle test. With conservative set, a box's exit
// distance is widened by 1 + 2 gamma_3 (Ize, "Robust BVH Ray Traversal",
// JCGT 2(2), 2013), so that rounding in the slab test never culls a box
// whose triangle the watertight test hits.
template<typename Test, typename Accept>
__device__ inline int traceNearestFirst(const BvhView& b, V3 o, V3 d, float& distance, bool conservative, Test test, Accept accept)
{
	V3 inv = bvhInverseDirection(d);
	const float widen = conservative ? 1.00000036f : 1.0f;
	TraceWork work;
	auto box = [&](int node) -> float
	{
		++work.nodes;
		V3 lo = b.row(node * 2).xyz();
		V3 hi = b.row(node * 2 + 1).xyz();
		V3 t0 = (lo - o) * inv;
		V3 t1 = (hi - o) * inv;
		V3 n = vmin(t0, t1);
		V3 f = vmax(t0, t1);
		float enter = fmaxf(fmaxf(n.x, n.y), fmaxf(n.z, 0.0f));
		float leave = fminf(fminf(f.x, f.y), f.z) * widen;
		leave = fminf(leave, distance);
		return enter <= leave ? enter : -1.0f;
	};
	if (!b.available() || box(0) < 0.0f)
	{
		countWork(RESTIR_COUNT_PRIMARY, work.nodes, work.triangles);
		return -1;
	}
	// Each entry keeps the box's entry distance: a box that passed its test
	// when pushed passes it again at the pop exactly when that distance is
	// still within the nearest hit (its own exit did not change), so the pop
	// needs no second fetch of the box.
	int stack[64];
	float stackEnter[64];
	int top = 0;
	int hit = -1;
	int node = 0;
	for (int step = 0; step < (1 << 24); ++step)
	{
		V4 node0 = b.row(node * 2);
		V4 node1 = b.row(node * 2 + 1);
		if (node1.w >= 0.0f)
		{
			int first = int(node0.w);
			int count = int(node1.w);
			work.triangles += uint32_t(count);
			for (int t = first; t < first + count; ++t)
			{
				float h = test(t, distance);
				if (h > 0.0f && (h < distance || (h == distance && hit >= 0 && t < hit)) && accept(t))
				{
					distance = h;
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
				if (top < 64)
				{
					stack[top] = leftFirst ? right : left;
					stackEnter[top] = leftFirst ? rightDistance : leftDistance;
					++top;
				}
				else
				{
					reportTruncatedRay();
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
		// Pop, skipping subtrees that the nearest hit found since rules out.
		bool found = false;
		while (top > 0)
		{
			--top;
			if (stackEnter[top] <= distance)
			{
				node = stack[top];
				found = true;
				break;
			}
		}
		if (!found)
		{
			break;
		}
	}
	countWork(RESTIR_COUNT_PRIMARY, work.nodes, work.triangles);
	return hit;
}

// Moeller-Trumbore nearest hit among accepted triangles (the raster
// passes' ray casts).
template<typename Accept>
__device__ inline int traceNearestFiltered(const BvhView& b, V3 o, V3 d, float& distance, Accept accept)
{
	return traceNearestFirst(b, o, d, distance, false,
		[&](int t, float) { return intersectTriangle(o, d, b.vertex(t, 0), b.vertex(t, 1), b.vertex(t, 2)); }, accept);
}

} // namespace restir
