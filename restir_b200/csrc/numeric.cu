// restir_numeric_eval: evaluates one function of include/restir_numeric.h
// on the device over an array, so that tests can check that the kernels'
// sin, cos, exp, half and unorm8 conversions are bit-identical to the host's.
#include "grid.cuh"

namespace restir
{
namespace
{

__global__ void numericKernel(int fn, const float* __restrict__ in, float* __restrict__ out, uint32_t n)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	const float x = in[i];
	float y = 0.0f;
	switch (fn)
	{
	case 0: y = rn_sin(x); break;
	case 1: y = rn_cos(x); break;
	case 2: y = rn_exp(x); break;
	case 3: y = __half2float(__float2half_rn(x)); break;
	case 4: y = rn_half_to_float(rn_float_to_half(x)); break;
	case 5: y = float(rn_unorm8(x)); break;
	case 6: y = float(rn_floor_log2(x)); break;
	case 7: y = rn_pow64(x); break;
	case 8: y = __uint_as_float(pcg(__float_as_uint(x))); break;
	case 9: y = __uint_as_float(gridChecksumHash(__float_as_uint(x))); break;
	case 10: y = rn_half_to_float(uint16_t(__float_as_uint(x) & 0xffffu)); break;
	case 11: y = rn_log2(x); break;
	case 12: y = rn_exp2(x); break;
	case 13: y = rn_pow(x, 2.2f); break;
	case 14: y = rn_pow(x, 1.0f / 2.2f); break;
	default: y = x; break;
	}
	out[i] = y;
}

} // namespace
} // namespace restir

extern "C" int restir_numeric_eval(int fn, const float* in, float* out, uint32_t n, void* stream)
{
	if (in == nullptr || out == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	if (n == 0)
	{
		return RESTIR_OK;
	}
	restir::numericKernel<<<(n + 255) / 256, 256, 0, restir::asStream(stream)>>>(fn, in, out, n);
	return restir::launchStatus();
}
