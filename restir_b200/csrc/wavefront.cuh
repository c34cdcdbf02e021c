// Wavefront ray queues: a persistent traversal kernel that keeps every lane
// of a warp busy.
//
// A producer pass appends rays to a queue in global memory (a warp's lanes
// take consecutive slots: one __ballot_sync, one atomicAdd per warp). The
// tracer below runs one resident grid; each lane holds one ray and advances
// it one node per loop iteration, and as soon as its ray finishes it takes
// the next unclaimed ray (again one atomicAdd per warp for all lanes that
// need one). Lanes therefore stay in the same traversal loop instead of
// idling behind the longest ray of their warp.
//
// The per-ray algorithm is the reference's nearest-first short-stack
// traversal (bvh.sh:216-295) written as a resumable state machine: the same
// nodes in the same order, the same step cap, the same stackless fallback,
// so hit ids and distances are identical to traceShortStack's. The tracer's
// walk form runs the stackless walk (bvh.sh:140-174) the same way, for the
// rays of the fragment-shader passes.
#pragma once

#include "bvh.cuh"

namespace restir
{

// Queue layout: rays[2 * i] = (origin, tmax), rays[2 * i + 1] = (direction, 0)
// (restir_trace's ray format); results hitTriangle[i], hitDistance[i].
struct RayQueue
{
	float4* rays;
	int* hitTriangle;
	float* hitDistance;
	uint32_t* count;    // rays appended by the producer; null: capacity rays
	uint32_t* claimed;  // rays taken by the tracer
	uint32_t capacity;
};

// Appends this lane's ray when push is set; every lane of the warp must call
// it (it votes). Returns the slot, or -1.
__device__ __forceinline__ int queuePush(const RayQueue& q, bool push, V3 origin, float tmax, V3 direction)
{
	const unsigned lane = threadIdx.x & 31u;
	const unsigned mask = __ballot_sync(0xffffffffu, push);
	const int leader = mask != 0u ? __ffs(mask) - 1 : 0;
	uint32_t base = 0;
	if (mask != 0u && int(lane) == leader)
	{
		base = atomicAdd(q.count, uint32_t(__popc(mask)));
	}
	base = __shfl_sync(0xffffffffu, base, leader);
	if (!push)
	{
		return -1;
	}
	const uint32_t slot = base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
	if (slot >= q.capacity)
	{
		raiseStatus(4u);
		return -1;
	}
	q.rays[2 * slot] = make_float4(origin.x, origin.y, origin.z, tmax);
	q.rays[2 * slot + 1] = make_float4(direction.x, direction.y, direction.z, 0.0f);
	return int(slot);
}

// One lane's traversal state (registers), its short stack in shared memory.
struct ShortStackState
{
	V3 o, d, inv;
	float distance;
	int hit;          // nearest hit of the short-stack walk
	int fallbackHit;  // nearest hit of the stackless re-walk
	int node;
	int stackTop;
	int stackCount;
	int step;
	bool dropped;
	int phase;        // 0 short stack, 1 stackless re-walk, 2 done
	TraceWork work;
};

__device__ __forceinline__ void startShortStack(ShortStackState& s, const BvhView& b, V3 o, V3 d, float tmax)
{
	s.o = o;
	s.d = d;
	s.inv = bvhInverseDirection(d);
	s.distance = tmax;
	s.hit = -1;
	s.fallbackHit = -1;
	s.node = 0;
	s.stackTop = 0;
	s.stackCount = 0;
	s.step = 0;
	s.dropped = false;
	s.work = TraceWork();
	s.phase = 0;
	++s.work.nodes;
	if (!b.available() || intersectBox(o, s.inv, b.row(0).xyz(), b.row(1).xyz(), s.distance) < 0.0f)
	{
		s.phase = 2;
	}
}

// A ray of the stackless walk alone (the fragment-shader passes): phase 1
// from the root, whose box the walk tests in its first step.
__device__ __forceinline__ void startStacklessWalk(ShortStackState& s, V3 o, V3 d, float tmax)
{
	s.o = o;
	s.d = d;
	s.inv = bvhInverseDirection(d);
	s.distance = tmax;
	s.hit = -1;
	s.fallbackHit = -1;
	s.node = 0;
	s.stackTop = 0;
	s.stackCount = 0;
	s.step = 0;
	s.dropped = false;
	s.work = TraceWork();
	s.phase = 1;
}

// The end of the short-stack walk: the stackless re-walk if entries were dropped.
__device__ __forceinline__ void endShortStack(ShortStackState& s)
{
	if (s.step == kBvhMaxSteps)
	{
		reportTruncatedRay();
	}
	if (s.dropped)
	{
		s.phase = 1;
		s.node = 0;
		s.step = 0;
	}
	else
	{
		s.phase = 2;
	}
}

// traceStacklessWalk (bvh.sh:140-174), one node per call (the short stack's
// re-walk, phase 1) or, with kPair, one or two (a whole ray started by
// startStacklessWalk): the rows of the node after this one are fetched with
// this node's, and when the walk goes on to it (a box passed, or a leaf) it
// is visited in the same call, so that fetch's latency overlaps this node's
// test. Nodes, order and step count are the walk's.
template<bool kPair>
__device__ __forceinline__ void stepStacklessWalk(ShortStackState& s, const BvhView& b)
{
	if (s.step >= kBvhMaxSteps || s.node >= b.nodeCount)
	{
		if (s.step >= kBvhMaxSteps)
		{
			reportTruncatedRay();
		}
		if (s.fallbackHit >= 0)
		{
			s.hit = s.fallbackHit;
		}
		s.phase = 2;
		return;
	}
	const int following = s.node + 1;
	const bool fetched = kPair && following < b.nodeCount;
	const V4 node0 = b.row(s.node * 2);
	const V4 node1 = b.row(s.node * 2 + 1);
	V4 next0 = node0, next1 = node1;
	if (fetched)
	{
		next0 = b.row(following * 2);
		next1 = b.row(following * 2 + 1);
	}
	auto visit = [&](const V4& row0, const V4& row1)
	{
		++s.work.nodes;
		++s.step;
		const bool leaf = row1.w >= 0.0f;
		if (intersectBox(s.o, s.inv, row0.xyz(), row1.xyz(), s.distance) < 0.0f)
		{
			s.node = leaf ? s.node + 1 : int(-row1.w) - 1;
			return;
		}
		if (leaf)
		{
			s.fallbackHit = intersectLeaf(b, s.o, s.d, int(row0.w), int(row1.w), s.distance, s.fallbackHit, s.work);
		}
		s.node = s.node + 1;
	};
	visit(node0, node1);
	if (fetched && s.node == following && s.step < kBvhMaxSteps)
	{
		visit(next0, next1);
	}
}

// Advances the traversal by one node.
__device__ __forceinline__ void stepShortStack(ShortStackState& s, const BvhView& b, int* stack, int stride)
{
	if (s.phase == 0)
	{
		if (s.step >= kBvhMaxSteps)
		{
			endShortStack(s);
			return;
		}
		V4 node0 = b.row(s.node * 2);
		V4 node1 = b.row(s.node * 2 + 1);
		if (node1.w >= 0.0f)
		{
			s.hit = intersectLeaf(b, s.o, s.d, int(node0.w), int(node1.w), s.distance, s.hit, s.work);
		}
		else
		{
			int left = s.node + 1;
			int right = int(node0.w);
			s.work.nodes += 2u;
			float leftDistance = intersectBox(s.o, s.inv, b.row(left * 2).xyz(), b.row(left * 2 + 1).xyz(), s.distance);
			float rightDistance = intersectBox(s.o, s.inv, b.row(right * 2).xyz(), b.row(right * 2 + 1).xyz(), s.distance);
			bool visitLeft = leftDistance >= 0.0f;
			bool visitRight = rightDistance >= 0.0f;
			if (visitLeft && visitRight)
			{
				bool leftFirst = leftDistance <= rightDistance;
				stack[(s.stackTop & (kBvhShortStack - 1)) * stride] = leftFirst ? right : left;
				++s.stackTop;
				if (s.stackCount == kBvhShortStack)
				{
					s.dropped = true;
				}
				else
				{
					++s.stackCount;
				}
				s.node = leftFirst ? left : right;
				++s.step;
				return;
			}
			if (visitLeft || visitRight)
			{
				s.node = visitLeft ? left : right;
				++s.step;
				return;
			}
		}
		if (s.stackCount == 0)
		{
			endShortStack(s);
			return;
		}
		--s.stackTop;
		--s.stackCount;
		s.node = stack[(s.stackTop & (kBvhShortStack - 1)) * stride];
		++s.step;
		return;
	}
	if (s.phase == 1)
	{
		stepStacklessWalk<false>(s, b);
	}
}

// The persistent closest-hit tracer over a queue. Launch with a whole number
// of warps per block; stack: kBvhShortStack ints per thread of the block.
// kWalk: every ray takes the stackless walk instead (traceBvh without a
// stack, the fragment-shader passes; no stack storage).
template<int kThreads, bool kWalk = false>
__device__ inline void traceQueueClosest(const BvhView& b, const RayQueue& q, int* stackStorage)
{
	const unsigned lane = threadIdx.x & 31u;
	int* stack = kWalk ? nullptr : stackStorage + threadIdx.x;
	const uint32_t total = q.count != nullptr ? min(*q.count, q.capacity) : q.capacity;
	ShortStackState s;
	s.phase = 2;
	int ray = -1;
	bool exhausted = false;
	for (;;)
	{
		// Lanes without a ray take the next ones, one atomic per warp.
		const bool need = ray < 0 && !exhausted;
		const unsigned needMask = __ballot_sync(0xffffffffu, need);
		if (needMask != 0u)
		{
			uint32_t base = 0;
			if (lane == uint32_t(__ffs(needMask) - 1))
			{
				base = atomicAdd(q.claimed, uint32_t(__popc(needMask)));
			}
			base = __shfl_sync(0xffffffffu, base, __ffs(needMask) - 1);
			if (need)
			{
				const uint32_t index = base + uint32_t(__popc(needMask & ((1u << lane) - 1u)));
				if (index < total)
				{
					ray = int(index);
					float4 a = q.rays[2 * index];
					float4 c = q.rays[2 * index + 1];
					if (kWalk)
					{
						startStacklessWalk(s, v3(a.x, a.y, a.z), v3(c.x, c.y, c.z), a.w);
					}
					else
					{
						startShortStack(s, b, v3(a.x, a.y, a.z), v3(c.x, c.y, c.z), a.w);
					}
				}
				else
				{
					exhausted = true;
				}
			}
		}
		if (!__any_sync(0xffffffffu, ray >= 0))
		{
			break;
		}
		if (ray >= 0)
		{
			if (s.phase != 2)
			{
				if (kWalk)
				{
					stepStacklessWalk<true>(s, b);
				}
				else
				{
					stepShortStack(s, b, stack, kThreads);
				}
			}
			if (s.phase == 2)
			{
				q.hitTriangle[ray] = s.hit;
				q.hitDistance[ray] = s.distance;
				countWork(kWalk ? RESTIR_COUNT_ANY : RESTIR_COUNT_CLOSEST, s.work.nodes, s.work.triangles);
				ray = -1;
			}
		}
	}
}

} // namespace restir
