// restir_trace: a fixed ray set through the BVH (bvh.sh:298-319), one thread
// per ray. Closest-hit rays keep their short stack in shared memory,
// interleaved so that the 32 lanes of a warp touch 32 different banks.
// RESTIR_TRACE_CLOSEST_QUEUE runs the same closest-hit traversal through the
// persistent queue tracer (wavefront.cuh): the ray set is the queue.
#include "bvh.cuh"
#include "wavefront.cuh"
#include "watertight.cuh"

namespace restir
{
namespace
{

constexpr int kTraceBlock = 128;

__global__ void __launch_bounds__(kTraceBlock) traceKernel(BvhView bvh, const float4* __restrict__ rays,
	int32_t* __restrict__ hitTriangle, float* __restrict__ hitDistance, uint32_t n, int kind)
{
	__shared__ int stack[kBvhShortStack * kTraceBlock];
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	float4 a = __ldg(rays + 2 * i);
	float4 b = __ldg(rays + 2 * i + 1);
	V3 o = v3(a.x, a.y, a.z);
	V3 d = v3(b.x, b.y, b.z);
	float distance = a.w;
	int hit = -1;
	if (kind == RESTIR_TRACE_CLOSEST)
	{
		hit = traceBvh(bvh, o, d, a.w, false, distance, stack + threadIdx.x, kTraceBlock);
	}
	else if (kind == RESTIR_TRACE_ANY)
	{
		hit = traceBvh(bvh, o, d, a.w, true, distance, nullptr, 0);
	}
	else if (kind == RESTIR_TRACE_CLOSEST_STACKLESS)
	{
		hit = traceBvh(bvh, o, d, a.w, false, distance, nullptr, 0);
	}
	else if (kind == RESTIR_TRACE_ANY_WAVE)
	{
		hit = traceVisibility(bvh, o, d, a.w, distance, true);
	}
	else
	{
		hit = traceWatertight(bvh, o, d, distance);
	}
	hitTriangle[i] = hit;
	hitDistance[i] = distance;
}

__global__ void __launch_bounds__(kTraceBlock) traceQueueKernel(BvhView bvh, RayQueue queue)
{
	__shared__ int stack[kBvhShortStack * kTraceBlock];
	traceQueueClosest<kTraceBlock>(bvh, queue, stack);
}

int residentQueueBlocks()
{
	int device = 0, sms = 148, perSm = 0;
	if (cudaGetDevice(&device) == cudaSuccess)
	{
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	}
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, traceQueueKernel, kTraceBlock, 0) != cudaSuccess || perSm < 1)
	{
		perSm = 1;
	}
	return sms * perSm;
}

} // namespace
} // namespace restir

using namespace restir;

extern "C" int restir_trace(const RestirParams* params, const RestirScene* scene, const float* rays,
	int32_t* hit_triangle, float* hit_distance, uint32_t n, int kind, void* stream)
{
	(void)params;
	if (scene == nullptr || rays == nullptr || hit_triangle == nullptr || hit_distance == nullptr
		|| kind < RESTIR_TRACE_CLOSEST || kind > RESTIR_TRACE_ANY_WAVE)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	if (n == 0u)
	{
		return RESTIR_OK;
	}
	BvhView bvh = makeBvhView(scene);
	cudaStream_t s = asStream(stream);
	if (kind == RESTIR_TRACE_CLOSEST_QUEUE)
	{
		// The claim counter lives in stream-ordered memory, so that calls on
		// different streams do not share it.
		uint32_t* claimed = nullptr;
		if (cudaMallocAsync(reinterpret_cast<void**>(&claimed), sizeof(uint32_t), s) != cudaSuccess)
		{
			cudaGetLastError();
			return RESTIR_ERROR_OUT_OF_MEMORY;
		}
		cudaMemsetAsync(claimed, 0, sizeof(uint32_t), s);
		RayQueue q;
		q.rays = const_cast<float4*>(reinterpret_cast<const float4*>(rays));
		q.hitTriangle = hit_triangle;
		q.hitDistance = hit_distance;
		q.count = nullptr;
		q.claimed = claimed;
		q.capacity = n;
		static const int blocks = residentQueueBlocks();
		traceQueueKernel<<<blocks, kTraceBlock, 0, s>>>(bvh, q);
		const int status = launchStatus();
		cudaFreeAsync(claimed, s);
		return status;
	}
	traceKernel<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, s>>>(
		bvh, reinterpret_cast<const float4*>(rays), hit_triangle, hit_distance, n, kind);
	return launchStatus();
}
