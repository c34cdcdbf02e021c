// BVH builder on the device: the host builder's split rule and output
// (src/bvh.cpp:96-199, 253-393; restir_b200/host/bvh_build.cpp), built
// breadth first.
//
// Large nodes (more than kSmallTask triangles) are split level by level over
// the whole device:
//   1. binning: one block per chunk of up to kChunk triangles of one node
//      bins them on the three axes in shared memory (count, triangle bounds,
//      centroid bounds per bin; float bounds as order-preserving integers for
//      atomicMin / atomicMax), then merges into the node's bins;
//   2. one thread per node evaluates the 12-bin SAH exactly as the host does
//      (same loops, same float operations, the same first minimum) and
//      creates the children, whose bounds and centroid bounds are the unions
//      of their bins (min and max are exact, so they equal the host's
//      triangle-by-triangle bounds);
//   3. the partition reproduces std::partition's permutation (the reference's
//      and the host builder's): its two-pointer sweep swaps the k-th element
//      of the left part that belongs right with the k-th element from the end
//      of the right part that belongs left, so with a prefix sum of the
//      predicate every element knows its partner.
// Nodes of at most kSmallTask triangles, and the rare node whose centroids
// all coincide (a median split), are finished by one thread each with the
// host's sequential code. The tree is then numbered depth first (subtree
// sizes bottom up, indices top down) and written in the host's layout, so
// the buffer is the host builder's, bit for bit.
#include "common.cuh"

#include "../host/bvh_build.h"

#include <cub/device/device_scan.cuh>

#include <cfloat>
#include <chrono>
#include <cstring>

namespace restir
{
namespace
{

constexpr int kBins = 12;
constexpr uint32_t kMaxLeafSize = 4;
constexpr uint32_t kForcedLeafSize = 16;
constexpr uint32_t kMaxDepth = 40;
constexpr uint32_t kSmallTask = 64;   // subtrees this small are built by one thread
constexpr uint32_t kChunk = 4096;     // triangles per binning block
constexpr int kBinValues = 13;        // count, triangle bounds (6), centroid bounds (6)
constexpr int kTaskBins = 3 * kBins * kBinValues;

// The triangles' bounds and centroids, nine arrays of n floats: lo xyz, hi xyz, centroid xyz.
struct Soup
{
	const float* v;
	uint32_t n;
	__device__ float lo(uint32_t t, int k) const { return v[size_t(k) * n + t]; }
	__device__ float hi(uint32_t t, int k) const { return v[size_t(3 + k) * n + t]; }
	__device__ float c(uint32_t t, int k) const { return v[size_t(6 + k) * n + t]; }
};

struct TreeNode
{
	float lo[3], hi[3];
	uint32_t begin, count, depth;
	int child[2]; // -1: a leaf
};

struct Task
{
	uint32_t node, begin, count, depth;
	float clo[3], chi[3]; // centroid bounds
	int axis, plane;      // the SAH split, axis -1 when the node is not partitioned here
	uint32_t middle;
};

struct Counters
{
	uint32_t nodes;
	uint32_t nextTasks;
	uint32_t smallTasks;
	uint32_t chunks;
	uint32_t maxDepth;
	uint32_t errors;   // partition partners out of range (never expected)
};

// std::min / std::max as the host builder calls them: the first argument on ties.
__device__ __forceinline__ float minStd(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float maxStd(float a, float b) { return a < b ? b : a; }

// Floats as unsigned integers in the same order (for atomicMin / atomicMax).
__device__ __forceinline__ uint32_t orderedBits(float f)
{
	const uint32_t b = __float_as_uint(f);
	return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ float fromOrdered(uint32_t u)
{
	return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ int binOf(float c, float low, float scale)
{
	return min(int((c - low) * scale), kBins - 1);
}

__device__ __forceinline__ float boxArea(const float* lo, const float* hi)
{
	if (lo[0] > hi[0])
	{
		return 0.0f;
	}
	const float x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
	return 2.0f * (x * y + y * z + z * x);
}

// --- triangle bounds and the root -------------------------------------------------------

__global__ void triangleBoundsKernel(const float* __restrict__ positions, uint32_t n, float* soup)
{
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n)
	{
		return;
	}
	const float* p = positions + size_t(t) * 9;
	for (int k = 0; k < 3; ++k)
	{
		float lo = FLT_MAX, hi = -FLT_MAX;
		for (int corner = 0; corner < 3; ++corner)
		{
			lo = minStd(lo, p[corner * 3 + k]);
			hi = maxStd(hi, p[corner * 3 + k]);
		}
		soup[size_t(k) * n + t] = lo;
		soup[size_t(3 + k) * n + t] = hi;
		soup[size_t(6 + k) * n + t] = (lo + hi) * 0.5f;
	}
}

// Root bounds and centroid bounds into 12 ordered words: lo3, hi3, clo3, chi3.
__global__ void rootBoundsKernel(Soup s, uint32_t* words)
{
	uint32_t local[12];
	for (int k = 0; k < 3; ++k)
	{
		local[k] = orderedBits(FLT_MAX);
		local[3 + k] = orderedBits(-FLT_MAX);
		local[6 + k] = orderedBits(FLT_MAX);
		local[9 + k] = orderedBits(-FLT_MAX);
	}
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < s.n; t += gridDim.x * blockDim.x)
	{
		for (int k = 0; k < 3; ++k)
		{
			local[k] = min(local[k], orderedBits(s.lo(t, k)));
			local[3 + k] = max(local[3 + k], orderedBits(s.hi(t, k)));
			local[6 + k] = min(local[6 + k], orderedBits(s.c(t, k)));
			local[9 + k] = max(local[9 + k], orderedBits(s.c(t, k)));
		}
	}
	for (int i = 0; i < 12; ++i)
	{
		uint32_t v = local[i];
		const bool isMin = (i % 6) < 3;
		for (int offset = 16; offset > 0; offset >>= 1)
		{
			const uint32_t other = __shfl_xor_sync(0xffffffffu, v, offset);
			v = isMin ? min(v, other) : max(v, other);
		}
		if ((threadIdx.x & 31u) == 0u)
		{
			if (isMin)
			{
				atomicMin(words + i, v);
			}
			else
			{
				atomicMax(words + i, v);
			}
		}
	}
}

__global__ void rootTaskKernel(const uint32_t* words, uint32_t n, TreeNode* nodes, Task* tasks, Counters* counters)
{
	TreeNode& root = nodes[0];
	Task& task = tasks[0];
	for (int k = 0; k < 3; ++k)
	{
		root.lo[k] = fromOrdered(words[k]);
		root.hi[k] = fromOrdered(words[3 + k]);
		task.clo[k] = fromOrdered(words[6 + k]);
		task.chi[k] = fromOrdered(words[9 + k]);
	}
	root.begin = 0;
	root.count = n;
	root.depth = 1;
	root.child[0] = root.child[1] = -1;
	task.node = 0;
	task.begin = 0;
	task.count = n;
	task.depth = 1;
	task.axis = -1;
	counters->nodes = 1;
	counters->maxDepth = 1;
}

// --- one level of large nodes ---------------------------------------------------------

// Chunks per task (for the binning grid), and a zero after the last task for
// the exclusive prefix in chunkStart.
__global__ void chunkCountKernel(const Task* tasks, uint32_t count, uint32_t* chunks)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i <= count)
	{
		chunks[i] = i < count ? (tasks[i].count + kChunk - 1) / kChunk : 0u;
	}
}

__global__ void binInitKernel(uint32_t* bins, uint32_t words)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x)
	{
		const int v = int(i % kBinValues);
		bins[i] = v == 0 ? 0u : ((v - 1) % 6 < 3 ? orderedBits(FLT_MAX) : orderedBits(-FLT_MAX));
	}
}

// The task of chunk b: the last task whose first chunk is <= b.
__device__ __forceinline__ uint32_t taskOfChunk(const uint32_t* chunkStart, uint32_t tasks, uint32_t b)
{
	uint32_t lo = 0, hi = tasks;
	while (hi - lo > 1)
	{
		const uint32_t mid = (lo + hi) / 2;
		if (chunkStart[mid] <= b)
		{
			lo = mid;
		}
		else
		{
			hi = mid;
		}
	}
	return lo;
}

__global__ void __launch_bounds__(256) binKernel(const Task* __restrict__ tasks, uint32_t taskCount,
	const uint32_t* __restrict__ chunkStart, const uint32_t* __restrict__ order, Soup s, uint32_t* bins)
{
	__shared__ uint32_t local[kTaskBins];
	const uint32_t ti = taskOfChunk(chunkStart, taskCount, blockIdx.x);
	const Task task = tasks[ti];
	for (int i = int(threadIdx.x); i < kTaskBins; i += int(blockDim.x))
	{
		const int v = i % kBinValues;
		local[i] = v == 0 ? 0u : ((v - 1) % 6 < 3 ? orderedBits(FLT_MAX) : orderedBits(-FLT_MAX));
	}
	__syncthreads();
	float low[3], scale[3];
	bool active[3];
	for (int a = 0; a < 3; ++a)
	{
		low[a] = task.clo[a];
		const float extent = task.chi[a] - low[a];
		active[a] = extent > 0.0f;
		scale[a] = active[a] ? float(kBins) / extent : 0.0f;
	}
	const uint32_t first = task.begin + (blockIdx.x - chunkStart[ti]) * kChunk;
	const uint32_t last = min(first + kChunk, task.begin + task.count);
	for (uint32_t slot = first + threadIdx.x; slot < last; slot += blockDim.x)
	{
		const uint32_t t = order[slot];
		uint32_t box[12];
		for (int k = 0; k < 3; ++k)
		{
			box[k] = orderedBits(s.lo(t, k));
			box[3 + k] = orderedBits(s.hi(t, k));
			box[6 + k] = orderedBits(s.c(t, k));
			box[9 + k] = box[6 + k];
		}
		for (int a = 0; a < 3; ++a)
		{
			if (!active[a])
			{
				continue;
			}
			uint32_t* b = local + (a * kBins + binOf(s.c(t, a), low[a], scale[a])) * kBinValues;
			atomicAdd(b, 1u);
			for (int k = 0; k < 12; ++k)
			{
				if (k % 6 < 3)
				{
					atomicMin(b + 1 + k, box[k]);
				}
				else
				{
					atomicMax(b + 1 + k, box[k]);
				}
			}
		}
	}
	__syncthreads();
	uint32_t* global = bins + size_t(ti) * kTaskBins;
	for (int i = int(threadIdx.x); i < kTaskBins; i += int(blockDim.x))
	{
		const int v = i % kBinValues;
		if (v == 0)
		{
			if (local[i] != 0u)
			{
				atomicAdd(global + i, local[i]);
			}
		}
		else if ((v - 1) % 6 < 3)
		{
			if (local[i] != orderedBits(FLT_MAX))
			{
				atomicMin(global + i, local[i]);
			}
		}
		else if (local[i] != orderedBits(-FLT_MAX))
		{
			atomicMax(global + i, local[i]);
		}
	}
}

struct BinBox
{
	float lo[3], hi[3], clo[3], chi[3];
	uint32_t count;
};

__device__ __forceinline__ void emptyBox(BinBox& b)
{
	for (int k = 0; k < 3; ++k)
	{
		b.lo[k] = FLT_MAX;
		b.hi[k] = -FLT_MAX;
		b.clo[k] = FLT_MAX;
		b.chi[k] = -FLT_MAX;
	}
	b.count = 0;
}

__device__ __forceinline__ void readBin(const uint32_t* bins, int axis, int bin, BinBox& b)
{
	const uint32_t* w = bins + (axis * kBins + bin) * kBinValues;
	b.count = w[0];
	for (int k = 0; k < 3; ++k)
	{
		b.lo[k] = fromOrdered(w[1 + k]);
		b.hi[k] = fromOrdered(w[4 + k]);
		b.clo[k] = fromOrdered(w[7 + k]);
		b.chi[k] = fromOrdered(w[10 + k]);
	}
}

__device__ __forceinline__ void growBox(BinBox& into, const BinBox& b)
{
	for (int k = 0; k < 3; ++k)
	{
		into.lo[k] = minStd(into.lo[k], b.lo[k]);
		into.hi[k] = maxStd(into.hi[k], b.hi[k]);
		into.clo[k] = minStd(into.clo[k], b.clo[k]);
		into.chi[k] = maxStd(into.chi[k], b.chi[k]);
	}
	into.count += b.count;
}

__device__ __forceinline__ void noteDepth(Counters* counters, uint32_t depth)
{
	atomicMax(&counters->maxDepth, depth);
}

// A new node (and its task for the next level, or for the one-thread builder).
__device__ void makeChild(const BinBox& b, uint32_t begin, uint32_t depth, int& id, TreeNode* nodes, Task* next,
	uint32_t* small, Counters* counters)
{
	id = int(atomicAdd(&counters->nodes, 1u));
	TreeNode& node = nodes[id];
	for (int k = 0; k < 3; ++k)
	{
		node.lo[k] = b.lo[k];
		node.hi[k] = b.hi[k];
	}
	node.begin = begin;
	node.count = b.count;
	node.depth = depth;
	node.child[0] = node.child[1] = -1;
	noteDepth(counters, depth);
	if (b.count > kSmallTask && depth < kMaxDepth)
	{
		Task& task = next[atomicAdd(&counters->nextTasks, 1u)];
		task.node = uint32_t(id);
		task.begin = begin;
		task.count = b.count;
		task.depth = depth;
		task.axis = -1;
		for (int k = 0; k < 3; ++k)
		{
			task.clo[k] = b.clo[k];
			task.chi[k] = b.chi[k];
		}
	}
	else if (b.count > 1 && depth < kMaxDepth)
	{
		small[atomicAdd(&counters->smallTasks, 1u)] = uint32_t(id);
	}
}

// The host builder's split decision for each large node (bvh_build.cpp split()).
__global__ void sahKernel(Task* tasks, uint32_t taskCount, const uint32_t* __restrict__ allBins, TreeNode* nodes,
	Task* next, uint32_t* small, Counters* counters)
{
	const uint32_t ti = blockIdx.x * blockDim.x + threadIdx.x;
	if (ti >= taskCount)
	{
		return;
	}
	Task& task = tasks[ti];
	TreeNode& node = nodes[task.node];
	const uint32_t* bins = allBins + size_t(ti) * kTaskBins;
	float bestCost = FLT_MAX;
	int bestAxis = -1, bestPlane = 0;
	for (int axis = 0; axis < 3; ++axis)
	{
		if (!(task.chi[axis] - task.clo[axis] > 0.0f))
		{
			continue;
		}
		float rightArea[kBins];
		uint32_t rightCount[kBins];
		BinBox right;
		emptyBox(right);
		for (int bin = kBins - 1; bin > 0; --bin)
		{
			BinBox b;
			readBin(bins, axis, bin, b);
			growBox(right, b);
			rightArea[bin] = boxArea(right.lo, right.hi);
			rightCount[bin] = right.count;
		}
		BinBox left;
		emptyBox(left);
		for (int plane = 1; plane < kBins; ++plane)
		{
			BinBox b;
			readBin(bins, axis, plane - 1, b);
			growBox(left, b);
			if (left.count == 0 || rightCount[plane] == 0)
			{
				continue;
			}
			const float cost = boxArea(left.lo, left.hi) * float(left.count) + rightArea[plane] * float(rightCount[plane]);
			if (cost < bestCost)
			{
				bestCost = cost;
				bestAxis = axis;
				bestPlane = plane;
			}
		}
	}
	const float leafCost = boxArea(node.lo, node.hi) * float(task.count);
	if (bestAxis >= 0 && (bestCost < leafCost || task.count > kMaxLeafSize))
	{
		BinBox left, right;
		emptyBox(left);
		emptyBox(right);
		for (int bin = 0; bin < kBins; ++bin)
		{
			BinBox b;
			readBin(bins, bestAxis, bin, b);
			growBox(bin < bestPlane ? left : right, b);
		}
		task.axis = bestAxis;
		task.plane = bestPlane;
		task.middle = task.begin + left.count;
		makeChild(left, task.begin, task.depth + 1, node.child[0], nodes, next, small, counters);
		makeChild(right, task.middle, task.depth + 1, node.child[1], nodes, next, small, counters);
	}
	else if (task.count > kForcedLeafSize)
	{
		// Every centroid coincides: the one-thread builder splits at the median.
		task.axis = -1;
		small[atomicAdd(&counters->smallTasks, 1u)] = task.node;
	}
	else
	{
		task.axis = -1;
	}
}

// std::partition of the split nodes: flags, then every misplaced element finds its partner.
__global__ void __launch_bounds__(256) flagKernel(const Task* __restrict__ tasks, uint32_t taskCount,
	const uint32_t* __restrict__ chunkStart, const uint32_t* __restrict__ order, Soup s, uint32_t* flags)
{
	const uint32_t ti = taskOfChunk(chunkStart, taskCount, blockIdx.x);
	const Task task = tasks[ti];
	const uint32_t first = task.begin + (blockIdx.x - chunkStart[ti]) * kChunk;
	const uint32_t last = min(first + kChunk, task.begin + task.count);
	const bool split = task.axis >= 0;
	float low = 0.0f, scale = 0.0f;
	if (split)
	{
		low = task.clo[task.axis];
		scale = float(kBins) / (task.chi[task.axis] - low);
	}
	for (uint32_t slot = first + threadIdx.x; slot < last; slot += blockDim.x)
	{
		flags[slot] = split && binOf(s.c(order[slot], task.axis), low, scale) < task.plane ? 1u : 0u;
	}
}

// prefix: exclusive sum of flags over all slots (n + 1 entries).
__global__ void __launch_bounds__(256) pairKernel(const Task* __restrict__ tasks, uint32_t taskCount,
	const uint32_t* __restrict__ chunkStart, const uint32_t* __restrict__ flags, const uint32_t* __restrict__ prefix,
	uint32_t* leftPos, uint32_t* rightPos)
{
	const uint32_t ti = taskOfChunk(chunkStart, taskCount, blockIdx.x);
	const Task task = tasks[ti];
	if (task.axis < 0)
	{
		return;
	}
	const uint32_t b = task.begin, e = task.begin + task.count, mid = task.middle;
	const uint32_t first = b + (blockIdx.x - chunkStart[ti]) * kChunk;
	const uint32_t last = min(first + kChunk, e);
	for (uint32_t p = first + threadIdx.x; p < last; p += blockDim.x)
	{
		const bool goesLeft = flags[p] != 0u;
		if (p < mid && !goesLeft)
		{
			leftPos[b + (p - b) - (prefix[p] - prefix[b])] = p;
		}
		else if (p >= mid && goesLeft)
		{
			rightPos[b + prefix[e] - prefix[p + 1]] = p;
		}
	}
}

__global__ void __launch_bounds__(256) swapKernel(const Task* __restrict__ tasks, uint32_t taskCount,
	const uint32_t* __restrict__ chunkStart, const uint32_t* __restrict__ flags, const uint32_t* __restrict__ prefix,
	const uint32_t* __restrict__ rightPos, uint32_t* order, Counters* counters)
{
	const uint32_t ti = taskOfChunk(chunkStart, taskCount, blockIdx.x);
	const Task task = tasks[ti];
	if (task.axis < 0)
	{
		return;
	}
	const uint32_t b = task.begin, mid = task.middle;
	const uint32_t first = b + (blockIdx.x - chunkStart[ti]) * kChunk;
	const uint32_t last = min(first + kChunk, mid);
	for (uint32_t p = first + threadIdx.x; p < last; p += blockDim.x)
	{
		if (flags[p] == 0u)
		{
			const uint32_t q = rightPos[b + (p - b) - (prefix[p] - prefix[b])];
			if (q < mid || q >= b + task.count)
			{
				atomicAdd(&counters->errors, 1u);
				continue;
			}
			const uint32_t t = order[p];
			order[p] = order[q];
			order[q] = t;
		}
	}
}

// --- small subtrees: the host builder's code, one thread per subtree --------------------

__global__ void smallKernel(const uint32_t* __restrict__ small, uint32_t count, Soup s, uint32_t* order,
	TreeNode* nodes, Counters* counters)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count)
	{
		return;
	}
	uint32_t stack[2 * kMaxDepth + 2];
	int top = 0;
	stack[top++] = small[i];
	while (top > 0)
	{
		const uint32_t id = stack[--top];
		TreeNode& node = nodes[id];
		const uint32_t begin = node.begin, count = node.count, depth = node.depth;
		const uint32_t end = begin + count;
		float lo[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, hi[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
		float clo[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, chi[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
		for (uint32_t slot = begin; slot < end; ++slot)
		{
			const uint32_t t = order[slot];
			for (int k = 0; k < 3; ++k)
			{
				lo[k] = minStd(lo[k], s.lo(t, k));
				hi[k] = maxStd(hi[k], s.hi(t, k));
				clo[k] = minStd(clo[k], s.c(t, k));
				chi[k] = maxStd(chi[k], s.c(t, k));
			}
		}
		for (int k = 0; k < 3; ++k)
		{
			node.lo[k] = lo[k];
			node.hi[k] = hi[k];
		}
		node.child[0] = node.child[1] = -1;
		noteDepth(counters, depth);
		if (count <= 1 || depth >= kMaxDepth)
		{
			continue;
		}
		float bestCost = FLT_MAX;
		int bestAxis = -1, bestPlane = 0;
		for (int axis = 0; axis < 3; ++axis)
		{
			const float low = clo[axis];
			const float extent = chi[axis] - low;
			if (extent <= 0.0f)
			{
				continue;
			}
			float binLo[kBins][3], binHi[kBins][3];
			uint32_t binCount[kBins];
			for (int bin = 0; bin < kBins; ++bin)
			{
				binCount[bin] = 0;
				for (int k = 0; k < 3; ++k)
				{
					binLo[bin][k] = FLT_MAX;
					binHi[bin][k] = -FLT_MAX;
				}
			}
			const float scale = float(kBins) / extent;
			for (uint32_t slot = begin; slot < end; ++slot)
			{
				const uint32_t t = order[slot];
				const int bin = binOf(s.c(t, axis), low, scale);
				for (int k = 0; k < 3; ++k)
				{
					binLo[bin][k] = minStd(binLo[bin][k], s.lo(t, k));
					binHi[bin][k] = maxStd(binHi[bin][k], s.hi(t, k));
				}
				++binCount[bin];
			}
			float rightArea[kBins];
			uint32_t rightCount[kBins];
			float rlo[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, rhi[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
			uint32_t rightTotal = 0;
			for (int bin = kBins - 1; bin > 0; --bin)
			{
				for (int k = 0; k < 3; ++k)
				{
					rlo[k] = minStd(rlo[k], binLo[bin][k]);
					rhi[k] = maxStd(rhi[k], binHi[bin][k]);
				}
				rightTotal += binCount[bin];
				rightArea[bin] = boxArea(rlo, rhi);
				rightCount[bin] = rightTotal;
			}
			float llo[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, lhi[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
			uint32_t leftTotal = 0;
			for (int plane = 1; plane < kBins; ++plane)
			{
				for (int k = 0; k < 3; ++k)
				{
					llo[k] = minStd(llo[k], binLo[plane - 1][k]);
					lhi[k] = maxStd(lhi[k], binHi[plane - 1][k]);
				}
				leftTotal += binCount[plane - 1];
				if (leftTotal == 0 || rightCount[plane] == 0)
				{
					continue;
				}
				const float cost = boxArea(llo, lhi) * float(leftTotal) + rightArea[plane] * float(rightCount[plane]);
				if (cost < bestCost)
				{
					bestCost = cost;
					bestAxis = axis;
					bestPlane = plane;
				}
			}
		}
		const float leafCost = boxArea(lo, hi) * float(count);
		uint32_t middle = begin;
		if (bestAxis >= 0 && (bestCost < leafCost || count > kMaxLeafSize))
		{
			// std::partition (two pointers, swapping the misplaced pair).
			const float low = clo[bestAxis];
			const float scale = float(kBins) / (chi[bestAxis] - low);
			uint32_t a = begin, b = end;
			for (;;)
			{
				while (a != b && binOf(s.c(order[a], bestAxis), low, scale) < bestPlane)
				{
					++a;
				}
				if (a == b)
				{
					break;
				}
				--b;
				while (a != b && !(binOf(s.c(order[b], bestAxis), low, scale) < bestPlane))
				{
					--b;
				}
				if (a == b)
				{
					break;
				}
				const uint32_t t = order[a];
				order[a] = order[b];
				order[b] = t;
				++a;
			}
			middle = a;
		}
		else if (count > kForcedLeafSize)
		{
			middle = begin + count / 2;
		}
		else
		{
			continue;
		}
		const int first = int(atomicAdd(&counters->nodes, 2u));
		node.child[0] = first;
		node.child[1] = first + 1;
		const uint32_t ranges[2][2] = { { begin, middle - begin }, { middle, end - middle } };
		for (int c = 0; c < 2; ++c)
		{
			TreeNode& child = nodes[first + c];
			child.begin = ranges[c][0];
			child.count = ranges[c][1];
			child.depth = depth + 1;
			child.child[0] = child.child[1] = -1;
			stack[top++] = uint32_t(first + c);
		}
	}
}

// --- depth-first numbering and the output ---------------------------------------------

__global__ void sizeKernel(const TreeNode* nodes, uint32_t count, uint32_t depth, uint32_t* size)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < count && nodes[i].depth == depth)
	{
		const TreeNode& n = nodes[i];
		size[i] = n.child[0] < 0 ? 1u : 1u + size[n.child[0]] + size[n.child[1]];
	}
}

__global__ void indexKernel(const TreeNode* nodes, uint32_t count, uint32_t depth, const uint32_t* size, uint32_t* index)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < count && nodes[i].depth == depth && nodes[i].child[0] >= 0)
	{
		const TreeNode& n = nodes[i];
		index[n.child[0]] = index[i] + 1u;
		index[n.child[1]] = index[i] + 1u + size[n.child[0]];
	}
}

__global__ void nodeRowsKernel(const TreeNode* nodes, uint32_t count, const uint32_t* size, const uint32_t* index,
	float4* rows)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count)
	{
		return;
	}
	const TreeNode& n = nodes[i];
	const uint32_t at = index[i];
	const bool leaf = n.child[0] < 0;
	rows[2 * at] = make_float4(n.lo[0], n.lo[1], n.lo[2], leaf ? float(n.begin) : float(index[n.child[1]]));
	rows[2 * at + 1] = make_float4(n.hi[0], n.hi[1], n.hi[2], leaf ? float(n.count) : -float(at + size[i] + 1u));
}

// The triangle records in leaf order (bvh_build.cpp buildBvh, bvh.cpp:306-390).
__global__ void triangleRowsKernel(const uint32_t* __restrict__ order, uint32_t n, const float* __restrict__ positions,
	const float* __restrict__ normals, const uint32_t* __restrict__ material, const uint8_t* __restrict__ twoSided,
	const float* __restrict__ materials, float4* rows, float4* triangleNormals, uint32_t* emissive)
{
	const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
	if (slot >= n)
	{
		return;
	}
	const uint32_t t = order[slot];
	const uint32_t m = material[t];
	const float* mat = materials + size_t(m) * 8; // base rgb, roughness, emission rgb, metallic
	const float* p = positions + size_t(t) * 9;
	float4* out = rows + size_t(slot) * 4;
	float metallic = 0.0f;
	float base[3] = { 0.0f, 0.0f, 0.0f };
	for (int corner = 0; corner < 3; ++corner)
	{
		for (int k = 0; k < 3; ++k)
		{
			base[k] += mat[k] / 3.0f;
		}
		metallic += mat[7] / 3.0f;
	}
	out[0] = make_float4(p[0], p[1], p[2], float(m));
	out[1] = make_float4(p[3], p[4], p[5], mat[4]);
	out[2] = make_float4(p[6], p[7], p[8], mat[5]);
	out[3] = make_float4(base[0] * 1.0f * (1.0f - metallic), base[1] * 1.0f * (1.0f - metallic),
		base[2] * 1.0f * (1.0f - metallic), mat[6]);
	triangleNormals[slot] = make_float4(normals[size_t(t) * 3], normals[size_t(t) * 3 + 1], normals[size_t(t) * 3 + 2],
		twoSided != nullptr ? float(twoSided[t]) : 0.0f);
	emissive[slot] = (mat[4] > 0.0f || mat[5] > 0.0f || mat[6] > 0.0f) ? 1u : 0u;
}

// The BVH slots of the emissive triangles, in slot order, with their mesh triangles.
__global__ void emitterListKernel(const uint32_t* __restrict__ emissive, const uint32_t* __restrict__ offsets,
	const uint32_t* __restrict__ order, uint32_t n, uint2* list)
{
	const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
	if (slot < n && emissive[slot] != 0u)
	{
		list[offsets[slot]] = make_uint2(slot, order[slot]);
	}
}

__global__ void identityKernel(uint32_t* order, uint32_t n)
{
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < n)
	{
		order[t] = t;
	}
}

// --- host side ----------------------------------------------------------------------------

// Temporary device memory from the stream-ordered pool, freed on the stream.
template<typename T>
struct DeviceArray
{
	T* p = nullptr;
	cudaStream_t stream = nullptr;
	bool allocate(size_t n, cudaStream_t s)
	{
		stream = s;
		return cudaMallocAsync(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T), s) == cudaSuccess;
	}
	~DeviceArray()
	{
		if (p != nullptr)
		{
			cudaFreeAsync(p, stream);
		}
	}
};

uint32_t blocksFor(uint64_t n, uint32_t threads)
{
	return uint32_t((n + threads - 1) / threads);
}

} // namespace

int buildBvhGpu(const Mesh& mesh, void* streamHandle, BvhResult& result, DeviceBvh* device)
{
	const cudaStream_t stream = static_cast<cudaStream_t>(streamHandle);
	const auto start = std::chrono::steady_clock::now();
	result = BvhResult();
	const uint32_t n = mesh.triangleCount();
	result.triangleCount = n;
	if (n == 0)
	{
		return RESTIR_OK;
	}
	if (mesh.materialData.size() < mesh.materials.size() * 8 || mesh.positions.size() < size_t(n) * 9
		|| mesh.normals.size() < size_t(n) * 3 || (!mesh.twoSided.empty() && mesh.twoSided.size() < n))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	for (uint32_t t = 0; t < n; ++t)
	{
		if (mesh.material[t] >= mesh.materials.size())
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
	}
	const uint32_t maxNodes = 2 * n;
	const uint32_t maxTasks = n / kSmallTask + 1;
	DeviceArray<float> positions, normals, materials, soup;
	DeviceArray<uint32_t> material, order, flags, prefix, leftPos, rightPos, small, bins, chunks, chunkStart, rootWords,
		size, index, emissive, emitterOffsets;
	DeviceArray<uint2> emitterList;
	DeviceArray<uint8_t> twoSided, scanScratch;
	DeviceArray<TreeNode> nodes;
	DeviceArray<Task> tasks[2];
	DeviceArray<Counters> counters;
	bool ok = positions.allocate(size_t(n) * 9, stream) && normals.allocate(size_t(n) * 3, stream)
		&& materials.allocate(mesh.materialData.size(), stream) && soup.allocate(size_t(n) * 9, stream)
		&& material.allocate(n, stream) && order.allocate(n, stream) && flags.allocate(n + 1, stream)
		&& prefix.allocate(n + 1, stream) && leftPos.allocate(n, stream) && rightPos.allocate(n, stream)
		&& small.allocate(n, stream) && nodes.allocate(maxNodes, stream) && tasks[0].allocate(maxTasks, stream)
		&& tasks[1].allocate(maxTasks, stream) && counters.allocate(1, stream) && rootWords.allocate(12, stream)
		&& size.allocate(maxNodes, stream) && index.allocate(maxNodes, stream) && emissive.allocate(n + 1, stream)
		&& emitterOffsets.allocate(n + 1, stream) && emitterList.allocate(n, stream)
		&& chunks.allocate(maxTasks + 1, stream) && chunkStart.allocate(maxTasks + 1, stream)
		&& bins.allocate(size_t(maxTasks) * kTaskBins, stream)
		&& (mesh.twoSided.empty() || twoSided.allocate(n, stream));
	// The outputs: node and triangle rows, shading normals (kept on the device or downloaded).
	float4* rows = nullptr;
	float4* triangleNormals = nullptr;
	ok = ok && cudaMalloc(&rows, (2 * size_t(maxNodes) + 4 * size_t(n)) * sizeof(float4)) == cudaSuccess;
	ok = ok && cudaMalloc(&triangleNormals, size_t(n) * sizeof(float4)) == cudaSuccess;
	size_t scanBytes = 0;
	cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, flags.p, prefix.p, n + 1, stream);
	ok = ok && scanScratch.allocate(scanBytes, stream);
	auto releaseOutputs = [&]()
	{
		cudaFree(rows);
		cudaFree(triangleNormals);
	};
	if (!ok)
	{
		cudaStreamSynchronize(stream);
		releaseOutputs();
		return RESTIR_ERROR_OUT_OF_MEMORY;
	}
	auto fail = [&](int status)
	{
		cudaStreamSynchronize(stream);
		releaseOutputs();
		return status;
	};
	cudaMemcpyAsync(positions.p, mesh.positions.data(), size_t(n) * 9 * sizeof(float), cudaMemcpyHostToDevice, stream);
	cudaMemcpyAsync(normals.p, mesh.normals.data(), size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice, stream);
	cudaMemcpyAsync(materials.p, mesh.materialData.data(), mesh.materialData.size() * sizeof(float), cudaMemcpyHostToDevice, stream);
	cudaMemcpyAsync(material.p, mesh.material.data(), size_t(n) * sizeof(uint32_t), cudaMemcpyHostToDevice, stream);
	if (!mesh.twoSided.empty())
	{
		cudaMemcpyAsync(twoSided.p, mesh.twoSided.data(), n, cudaMemcpyHostToDevice, stream);
	}
	identityKernel<<<blocksFor(n, 256), 256, 0, stream>>>(order.p, n);
	cudaMemsetAsync(counters.p, 0, sizeof(Counters), stream);
	cudaMemsetAsync(flags.p, 0, (n + 1) * sizeof(uint32_t), stream);

	const Soup s = { soup.p, n };
	triangleBoundsKernel<<<blocksFor(n, 256), 256, 0, stream>>>(positions.p, n, soup.p);
	{
		uint32_t init[12];
		for (int k = 0; k < 12; ++k)
		{
			const float v = (k % 6) < 3 ? FLT_MAX : -FLT_MAX;
			uint32_t b;
			std::memcpy(&b, &v, 4);
			init[k] = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
		}
		cudaMemcpyAsync(rootWords.p, init, sizeof(init), cudaMemcpyHostToDevice, stream);
		cudaStreamSynchronize(stream); // init lives on this stack frame
	}
	rootBoundsKernel<<<std::min<uint32_t>(blocksFor(n, 256), 1184), 256, 0, stream>>>(s, rootWords.p);
	rootTaskKernel<<<1, 1, 0, stream>>>(rootWords.p, n, nodes.p, tasks[0].p, counters.p);

	Counters host = {};
	uint32_t taskCount = 0;
	if (n > kSmallTask)
	{
		taskCount = 1;
	}
	else if (n > 1)
	{
		// The root is a small subtree: node 0, one small task.
		cudaMemsetAsync(small.p, 0, sizeof(uint32_t), stream);
		const uint32_t one = 1;
		cudaMemcpyAsync(&counters.p->smallTasks, &one, sizeof(uint32_t), cudaMemcpyHostToDevice, stream);
		cudaStreamSynchronize(stream);
	}
	int current = 0;
	uint32_t chunkTotal = 0;
	while (taskCount > 0)
	{
		Task* level = tasks[current].p;
		Task* next = tasks[1 - current].p;
		chunkCountKernel<<<blocksFor(taskCount + 1, 256), 256, 0, stream>>>(level, taskCount, chunks.p);
		size_t bytes = scanBytes;
		cub::DeviceScan::ExclusiveSum(scanScratch.p, bytes, chunks.p, chunkStart.p, taskCount + 1, stream);
		cudaMemcpyAsync(&chunkTotal, chunkStart.p + taskCount, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
		binInitKernel<<<std::min<uint32_t>(blocksFor(size_t(taskCount) * kTaskBins, 256), 4096), 256, 0, stream>>>(
			bins.p, taskCount * kTaskBins);
		cudaMemsetAsync(&counters.p->nextTasks, 0, sizeof(uint32_t), stream);
		if (cudaStreamSynchronize(stream) != cudaSuccess)
		{
			return fail(RESTIR_ERROR_LAUNCH);
		}
		binKernel<<<chunkTotal, 256, 0, stream>>>(level, taskCount, chunkStart.p, order.p, s, bins.p);
		sahKernel<<<blocksFor(taskCount, 128), 128, 0, stream>>>(level, taskCount, bins.p, nodes.p, next, small.p, counters.p);
		flagKernel<<<chunkTotal, 256, 0, stream>>>(level, taskCount, chunkStart.p, order.p, s, flags.p);
		bytes = scanBytes;
		cub::DeviceScan::ExclusiveSum(scanScratch.p, bytes, flags.p, prefix.p, n + 1, stream);
		pairKernel<<<chunkTotal, 256, 0, stream>>>(level, taskCount, chunkStart.p, flags.p, prefix.p, leftPos.p, rightPos.p);
		swapKernel<<<chunkTotal, 256, 0, stream>>>(level, taskCount, chunkStart.p, flags.p, prefix.p, rightPos.p, order.p,
			counters.p);
		// The flags of this level's ranges back to zero for the next scan.
		cudaMemsetAsync(flags.p, 0, (n + 1) * sizeof(uint32_t), stream);
		cudaMemcpyAsync(&host, counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, stream);
		if (cudaStreamSynchronize(stream) != cudaSuccess)
		{
			return fail(RESTIR_ERROR_LAUNCH);
		}
		if (host.errors != 0u)
		{
			return fail(RESTIR_ERROR_LAUNCH);
		}
		taskCount = host.nextTasks;
		current = 1 - current;
	}
	cudaMemcpyAsync(&host, counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, stream);
	if (cudaStreamSynchronize(stream) != cudaSuccess)
	{
		return fail(RESTIR_ERROR_LAUNCH);
	}
	if (host.smallTasks > 0)
	{
		smallKernel<<<blocksFor(host.smallTasks, 64), 64, 0, stream>>>(small.p, host.smallTasks, s, order.p, nodes.p,
			counters.p);
	}
	cudaMemcpyAsync(&host, counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, stream);
	if (cudaStreamSynchronize(stream) != cudaSuccess)
	{
		return fail(RESTIR_ERROR_LAUNCH);
	}
	const uint32_t nodeCount = host.nodes;
	const uint32_t depth = host.maxDepth;
	for (uint32_t d = depth; d >= 1; --d)
	{
		sizeKernel<<<blocksFor(nodeCount, 256), 256, 0, stream>>>(nodes.p, nodeCount, d, size.p);
	}
	cudaMemsetAsync(index.p, 0, sizeof(uint32_t), stream);
	for (uint32_t d = 1; d < depth; ++d)
	{
		indexKernel<<<blocksFor(nodeCount, 256), 256, 0, stream>>>(nodes.p, nodeCount, d, size.p, index.p);
	}
	nodeRowsKernel<<<blocksFor(nodeCount, 256), 256, 0, stream>>>(nodes.p, nodeCount, size.p, index.p, rows);
	cudaMemsetAsync(emissive.p + n, 0, sizeof(uint32_t), stream);
	triangleRowsKernel<<<blocksFor(n, 256), 256, 0, stream>>>(order.p, n, positions.p, normals.p, material.p,
		mesh.twoSided.empty() ? nullptr : twoSided.p, materials.p, rows + 2 * size_t(nodeCount), triangleNormals,
		emissive.p);
	size_t bytes = scanBytes;
	cub::DeviceScan::ExclusiveSum(scanScratch.p, bytes, emissive.p, emitterOffsets.p, n + 1, stream);
	emitterListKernel<<<blocksFor(n, 256), 256, 0, stream>>>(emissive.p, emitterOffsets.p, order.p, n, emitterList.p);
	uint32_t emitterCount = 0;
	cudaMemcpyAsync(&emitterCount, emitterOffsets.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
	if (cudaStreamSynchronize(stream) != cudaSuccess)
	{
		return fail(RESTIR_ERROR_LAUNCH);
	}
	std::vector<uint2> emitterPairs(emitterCount);
	cudaMemcpyAsync(emitterPairs.data(), emitterList.p, size_t(emitterCount) * sizeof(uint2), cudaMemcpyDeviceToHost, stream);

	result.nodeCount = nodeCount;
	result.depth = depth;
	result.triangleOffset = 2 * nodeCount;
	const size_t rowCount = size_t(result.triangleOffset) + 4 * size_t(n);
	if (device == nullptr)
	{
		result.data.resize(rowCount * 4);
		result.order.resize(n);
		result.triangleNormals.resize(size_t(n) * 4);
		cudaMemcpyAsync(result.data.data(), rows, rowCount * sizeof(float4), cudaMemcpyDeviceToHost, stream);
		cudaMemcpyAsync(result.order.data(), order.p, size_t(n) * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
		cudaMemcpyAsync(result.triangleNormals.data(), triangleNormals, size_t(n) * sizeof(float4), cudaMemcpyDeviceToHost,
			stream);
	}
	if (cudaStreamSynchronize(stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
	{
		return fail(RESTIR_ERROR_LAUNCH);
	}
	for (const uint2& e : emitterPairs)
	{
		const Material& m = mesh.materials[mesh.material[e.y]];
		Emitter emitter;
		emitter.triangle = e.x;
		std::memcpy(emitter.vertices, &mesh.positions[size_t(e.y) * 9], sizeof(emitter.vertices));
		std::memcpy(emitter.emission, m.emission, sizeof(emitter.emission));
		result.emitters.push_back(emitter);
	}
	if (device != nullptr)
	{
		device->rows = rows;
		device->rowsBytes = rowCount * sizeof(float4);
		device->normals = triangleNormals;
		device->normalsBytes = size_t(n) * sizeof(float4);
	}
	else
	{
		releaseOutputs();
	}
	result.buildMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
	return RESTIR_OK;
}

} // namespace restir
