// BVH builder for the reference's node layout (src/bvh.h:7-22).
//
// The split rule is the reference's (bvh.cpp:96-199): binned SAH over 12
// bins per axis on triangle-bound centroids, a leaf when the SAH says so and
// the node holds at most 4 triangles, a median split above 16 when the
// centroids coincide, depth at most 40. What differs is how it runs: the
// triangle bounds are kept in a structure-of-arrays, large subtrees are
// built on separate threads, and the tree is emitted once into the float4
// buffer in depth-first order with skip links, followed by the triangle
// records (v0, material), (v1, emission.r), (v2, emission.g),
// (diffuse albedo, emission.b) in leaf order (bvh.cpp:306-390, untextured).
#include "bvh_build.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>

namespace restir
{
namespace
{

constexpr int kBins = 12;
constexpr uint32_t kMaxLeafSize = 4;
constexpr uint32_t kForcedLeafSize = 16;
constexpr uint32_t kMaxDepth = 40;
constexpr uint32_t kParallelGrain = 1u << 15;

struct Box
{
	float lo[3] = { std::numeric_limits<float>::max(), std::numeric_limits<float>::max(), std::numeric_limits<float>::max() };
	float hi[3] = { -std::numeric_limits<float>::max(), -std::numeric_limits<float>::max(), -std::numeric_limits<float>::max() };

	void grow(const float* p)
	{
		for (int k = 0; k < 3; ++k)
		{
			lo[k] = std::min(lo[k], p[k]);
			hi[k] = std::max(hi[k], p[k]);
		}
	}
	void grow(const Box& b)
	{
		for (int k = 0; k < 3; ++k)
		{
			lo[k] = std::min(lo[k], b.lo[k]);
			hi[k] = std::max(hi[k], b.hi[k]);
		}
	}
	float area() const
	{
		if (lo[0] > hi[0])
		{
			return 0.0f;
		}
		float x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
		return 2.0f * (x * y + y * z + z * x);
	}
};

struct Node
{
	Box box;
	uint32_t first = 0, count = 0; // leaf range
	Node* child[2] = { nullptr, nullptr };
	bool leaf() const { return child[0] == nullptr; }
};

struct Context
{
	const std::vector<Box>* bounds;
	const std::vector<float>* centroids; // 3 per triangle
	std::vector<uint32_t>* order;
	int threads;
	std::atomic<uint32_t> depth{ 0 };
	std::atomic<uint32_t> nodes{ 0 };
};

int binOf(float c, float low, float scale)
{
	return std::min(int((c - low) * scale), kBins - 1);
}

Node* split(Context& ctx, uint32_t begin, uint32_t end, uint32_t depth, int spare)
{
	Node* node = new Node();
	ctx.nodes.fetch_add(1, std::memory_order_relaxed);
	std::vector<uint32_t>& order = *ctx.order;
	const std::vector<Box>& bounds = *ctx.bounds;
	const float* c = ctx.centroids->data();
	Box centroidBox;
	for (uint32_t i = begin; i < end; ++i)
	{
		node->box.grow(bounds[order[i]]);
		centroidBox.grow(c + 3 * size_t(order[i]));
	}
	const uint32_t count = end - begin;
	auto makeLeaf = [&]()
	{
		node->first = begin;
		node->count = count;
		uint32_t seen = ctx.depth.load(std::memory_order_relaxed);
		while (depth > seen && !ctx.depth.compare_exchange_weak(seen, depth))
		{
		}
		return node;
	};
	if (count <= 1 || depth >= kMaxDepth)
	{
		return makeLeaf();
	}
	float bestCost = std::numeric_limits<float>::max();
	int bestAxis = -1, bestPlane = 0;
	for (int axis = 0; axis < 3; ++axis)
	{
		const float low = centroidBox.lo[axis];
		const float extent = centroidBox.hi[axis] - low;
		if (extent <= 0.0f)
		{
			continue;
		}
		std::array<Box, kBins> binBox;
		std::array<uint32_t, kBins> binCount = {};
		const float scale = float(kBins) / extent;
		for (uint32_t i = begin; i < end; ++i)
		{
			const uint32_t t = order[i];
			const int bin = binOf(c[3 * size_t(t) + axis], low, scale);
			binBox[bin].grow(bounds[t]);
			++binCount[bin];
		}
		std::array<float, kBins> rightArea = {};
		std::array<uint32_t, kBins> rightCount = {};
		Box right;
		uint32_t rightTotal = 0;
		for (int bin = kBins - 1; bin > 0; --bin)
		{
			right.grow(binBox[bin]);
			rightTotal += binCount[bin];
			rightArea[bin] = right.area();
			rightCount[bin] = rightTotal;
		}
		Box left;
		uint32_t leftTotal = 0;
		for (int plane = 1; plane < kBins; ++plane)
		{
			left.grow(binBox[plane - 1]);
			leftTotal += binCount[plane - 1];
			if (leftTotal == 0 || rightCount[plane] == 0)
			{
				continue;
			}
			const float cost = left.area() * float(leftTotal) + rightArea[plane] * float(rightCount[plane]);
			if (cost < bestCost)
			{
				bestCost = cost;
				bestAxis = axis;
				bestPlane = plane;
			}
		}
	}
	const float leafCost = node->box.area() * float(count);
	uint32_t middle = begin;
	if (bestAxis >= 0 && (bestCost < leafCost || count > kMaxLeafSize))
	{
		const float low = centroidBox.lo[bestAxis];
		const float scale = float(kBins) / (centroidBox.hi[bestAxis] - low);
		middle = uint32_t(std::partition(order.begin() + begin, order.begin() + end, [&](uint32_t t)
		{
			return binOf(c[3 * size_t(t) + bestAxis], low, scale) < bestPlane;
		}) - order.begin());
	}
	else if (count > kForcedLeafSize)
	{
		middle = begin + count / 2;
	}
	else
	{
		return makeLeaf();
	}
	if (spare > 0 && count > kParallelGrain)
	{
		auto future = std::async(std::launch::async, [&ctx, begin, middle, depth, spare]()
		{
			return split(ctx, begin, middle, depth + 1, spare / 2 - 1 > 0 ? spare / 2 - 1 : 0);
		});
		node->child[1] = split(ctx, middle, end, depth + 1, spare / 2);
		node->child[0] = future.get();
	}
	else
	{
		node->child[0] = split(ctx, begin, middle, depth + 1, 0);
		node->child[1] = split(ctx, middle, end, depth + 1, 0);
	}
	return node;
}

// Depth-first, left child next, skip link to the node after the subtree.
void emit(const Node* node, float* out, uint32_t& written)
{
	float* values = out + size_t(written) * 8;
	++written;
	values[0] = node->box.lo[0];
	values[1] = node->box.lo[1];
	values[2] = node->box.lo[2];
	values[4] = node->box.hi[0];
	values[5] = node->box.hi[1];
	values[6] = node->box.hi[2];
	if (node->leaf())
	{
		values[3] = float(node->first);
		values[7] = float(node->count);
		return;
	}
	emit(node->child[0], out, written);
	const uint32_t right = written;
	emit(node->child[1], out, written);
	values[3] = float(right);
	values[7] = -float(written + 1);
}

void release(Node* node)
{
	if (node == nullptr)
	{
		return;
	}
	release(node->child[0]);
	release(node->child[1]);
	delete node;
}

} // namespace

BvhResult buildBvh(const Mesh& mesh, int threads)
{
	const auto start = std::chrono::steady_clock::now();
	BvhResult result;
	const uint32_t n = mesh.triangleCount();
	result.triangleCount = n;
	if (n == 0)
	{
		return result;
	}
	std::vector<Box> bounds(n);
	std::vector<float> centroids(size_t(n) * 3);
	for (uint32_t t = 0; t < n; ++t)
	{
		const float* p = &mesh.positions[size_t(t) * 9];
		Box b;
		b.grow(p);
		b.grow(p + 3);
		b.grow(p + 6);
		bounds[t] = b;
		for (int k = 0; k < 3; ++k)
		{
			centroids[size_t(t) * 3 + k] = (b.lo[k] + b.hi[k]) * 0.5f;
		}
	}
	result.order.resize(n);
	for (uint32_t t = 0; t < n; ++t)
	{
		result.order[t] = t;
	}
	Context ctx;
	ctx.bounds = &bounds;
	ctx.centroids = &centroids;
	ctx.order = &result.order;
	ctx.threads = std::max(1, threads);
	Node* root = split(ctx, 0, n, 1, ctx.threads > 1 ? 2 * ctx.threads : 0);

	result.nodeCount = ctx.nodes.load();
	result.depth = ctx.depth.load();
	result.triangleOffset = 2 * result.nodeCount;
	result.data.assign((size_t(result.triangleOffset) + 4 * size_t(n)) * 4, 0.0f);
	uint32_t written = 0;
	emit(root, result.data.data(), written);
	release(root);

	float* out = result.data.data() + size_t(written) * 8;
	result.triangleNormals.resize(size_t(n) * 4);
	for (uint32_t slot = 0; slot < n; ++slot)
	{
		const uint32_t t = result.order[slot];
		const uint32_t m = mesh.material[t];
		const Material& material = mesh.materials[m];
		const float* p = &mesh.positions[size_t(t) * 9];
		for (int corner = 0; corner < 3; ++corner)
		{
			out[corner * 4 + 0] = p[corner * 3 + 0];
			out[corner * 4 + 1] = p[corner * 3 + 1];
			out[corner * 4 + 2] = p[corner * 3 + 2];
		}
		out[3] = float(m);
		// The diffuse albedo as the reference derives it from per-vertex
		// attributes (bvh.cpp:392-421): each corner's colour and metallic
		// divided by three and summed, times (1 - metallic).
		float metallic = 0.0f;
		float base[3] = { 0.0f, 0.0f, 0.0f };
		for (int corner = 0; corner < 3; ++corner)
		{
			for (int k = 0; k < 3; ++k)
			{
				base[k] += material.base[k] / 3.0f;
			}
			metallic += material.metallic / 3.0f;
		}
		for (int k = 0; k < 3; ++k)
		{
			out[12 + k] = base[k] * 1.0f * (1.0f - metallic);
		}
		out[7] = material.emission[0];
		out[11] = material.emission[1];
		out[15] = material.emission[2];
		if (material.emission[0] > 0.0f || material.emission[1] > 0.0f || material.emission[2] > 0.0f)
		{
			Emitter e;
			e.triangle = slot;
			std::memcpy(e.vertices, p, sizeof(e.vertices));
			std::memcpy(e.emission, material.emission, sizeof(e.emission));
			result.emitters.push_back(e);
		}
		float* normal = &result.triangleNormals[size_t(slot) * 4];
		normal[0] = mesh.normals[size_t(t) * 3 + 0];
		normal[1] = mesh.normals[size_t(t) * 3 + 1];
		normal[2] = mesh.normals[size_t(t) * 3 + 2];
		normal[3] = mesh.twoSided.empty() ? 0.0f : float(mesh.twoSided[t]);
		out += 16;
	}
	result.buildMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
	return result;
}

} // namespace restir
