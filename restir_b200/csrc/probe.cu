// restir_gather_probe: the bandwidth of independent random 32-byte row
// gathers (two 16-byte read-only loads, the size of a BVH node) from a
// buffer, the fetch pattern of the traversal kernels. With a buffer that fits
// the 126 MB L2, it measures the rate at which L2 serves node rows: the
// denominator of the traversal passes' fetched-bytes roofline (their BVH
// rows come from L2, not HBM). A measurement hook, no counterpart in the
// reference.
#include "common.cuh"

namespace restir
{
namespace
{

constexpr int kProbeThreads = 256;

__global__ void __launch_bounds__(kProbeThreads) gatherProbeKernel(const float4* __restrict__ rows, uint32_t rowCount,
	uint32_t gathers, uint32_t seed, float* __restrict__ out)
{
	const uint32_t thread = blockIdx.x * blockDim.x + threadIdx.x;
	uint32_t state = pcg(thread ^ seed);
	float sum = 0.0f;
	for (uint32_t k = 0; k < gathers; ++k)
	{
		state = pcg(state);
		const uint32_t row = state % rowCount;
		const float4 a = __ldg(rows + 2u * row);
		const float4 b = __ldg(rows + 2u * row + 1u);
		sum += (a.x + a.w) + (b.y + b.z);
	}
	out[thread] = sum;
}

} // namespace
} // namespace restir

using namespace restir;

/* Each of blocks x 256 threads gathers `gathers` rows of 32 bytes at seeded
 * random indices of `rows` (row_count rows, 16-byte aligned) and writes one
 * float to out (blocks x 256 floats). Fetched bytes = blocks x 256 x gathers
 * x 32. */
extern "C" int restir_gather_probe(const float* rows, uint32_t row_count, uint32_t blocks, uint32_t gathers,
	uint32_t seed, float* out, void* stream)
{
	if (rows == nullptr || out == nullptr || row_count == 0u || blocks == 0u
		|| (reinterpret_cast<uintptr_t>(rows) & 15u) != 0u)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	gatherProbeKernel<<<blocks, kProbeThreads, 0, asStream(stream)>>>(reinterpret_cast<const float4*>(rows), row_count,
		gathers, seed, out);
	return launchStatus();
}
