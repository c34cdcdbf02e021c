// The progressive reference and its error pass, in FP64.
//
// restir_reference_accumulate (fs_reference.sc:18-25): mean = mean * (1 - w)
// + colour * w with w = 1 / (frames + 1), per channel in double precision
// (the reference keeps an RGBA32F target; thousands of frames of a float
// running mean lose the low bits). NaN colours keep the mean.
//
// restir_error (cs_error.sc:35-93, renderer.cpp:1152-1166): relative MSE and
// mean luminances over the pixels the reference covers. The reference runs
// one 16x16 group over the whole image; here every SM takes a slice: each
// block reduces its pixels in double precision with warp shuffles, writes
// one partial to the caller's scratch, and a single block sums the partials
// in block order, so the result does not depend on scheduling.
#include "common.cuh"

#include <mutex>

namespace restir
{
namespace
{

constexpr int kErrorBlocks = 148 * 4;
constexpr int kErrorThreads = 256;

// Scratch of restir_error_noalloc: one FP64 partial record (4 doubles) per
// block, one block per kNoAllocPixelsPerBlock pixels, at most
// kNoAllocMaxBlocks blocks (64 KB, resident on every device that loads the
// library until the process exits).
constexpr uint32_t kNoAllocPixelsPerBlock = 4096;
constexpr uint32_t kNoAllocMaxBlocks = 2048;
static __device__ __align__(256) double g_errorNoAllocScratch[kNoAllocMaxBlocks * 4];

__global__ void __launch_bounds__(256) accumulateKernel(const uint16_t* __restrict__ hdr, double* __restrict__ mean,
	uint8_t* __restrict__ alpha, uint32_t n, double weight)
{
	const uint32_t stride = gridDim.x * blockDim.x;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
	{
		V4 c = loadH4(hdr, int(i));
		bool nan = c.x != c.x || c.y != c.y || c.z != c.z;
		double r = mean[i], g = mean[n + i], b = mean[2 * size_t(n) + i];
		mean[i] = r * (1.0 - weight) + (nan ? r : double(c.x)) * weight;
		mean[n + i] = g * (1.0 - weight) + (nan ? g : double(c.y)) * weight;
		mean[2 * size_t(n) + i] = b * (1.0 - weight) + (nan ? b : double(c.z)) * weight;
		alpha[i] = c.w >= 0.5f ? 1 : 0;
	}
}

__device__ __forceinline__ double warpSum(double v)
{
	for (int offset = 16; offset > 0; offset >>= 1)
	{
		v += __shfl_down_sync(0xffffffffu, v, offset);
	}
	return v;
}

__global__ void __launch_bounds__(kErrorThreads) errorPartialKernel(const uint16_t* __restrict__ display,
	const double* __restrict__ mean, const uint8_t* __restrict__ alpha, uint32_t n, double* __restrict__ partials)
{
	__shared__ double warpTotals[kErrorThreads / 32][4];
	double relative = 0.0, image = 0.0, reference = 0.0, count = 0.0;
	const uint32_t stride = gridDim.x * blockDim.x;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
	{
		if (alpha[i] == 0)
		{
			continue;
		}
		V4 c = loadH4(display, int(i));
		double imageLuminance = 0.2126 * double(c.x) + 0.7152 * double(c.y) + 0.0722 * double(c.z);
		double referenceLuminance = 0.2126 * mean[i] + 0.7152 * mean[n + i] + 0.0722 * mean[2 * size_t(n) + i];
		double difference = imageLuminance - referenceLuminance;
		relative += difference * difference / (referenceLuminance * referenceLuminance + 0.01);
		image += imageLuminance;
		reference += referenceLuminance;
		count += 1.0;
	}
	relative = warpSum(relative);
	image = warpSum(image);
	reference = warpSum(reference);
	count = warpSum(count);
	const int warp = int(threadIdx.x >> 5);
	if ((threadIdx.x & 31u) == 0u)
	{
		warpTotals[warp][0] = relative;
		warpTotals[warp][1] = image;
		warpTotals[warp][2] = reference;
		warpTotals[warp][3] = count;
	}
	__syncthreads();
	if (threadIdx.x < 4u)
	{
		double total = 0.0;
		for (int k = 0; k < kErrorThreads / 32; ++k)
		{
			total += warpTotals[k][threadIdx.x];
		}
		partials[blockIdx.x * 4 + threadIdx.x] = total;
	}
}

__global__ void __launch_bounds__(32) errorFinalKernel(const double* __restrict__ partials, int blocks, double* __restrict__ out)
{
	if (threadIdx.x >= 4u)
	{
		return;
	}
	double total = 0.0;
	for (int b = 0; b < blocks; ++b)
	{
		total += partials[b * 4 + threadIdx.x];
	}
	__shared__ double sums[4];
	sums[threadIdx.x] = total;
	__syncwarp(0xfu);
	const double count = sums[3];
	const double denominator = count > 1.0 ? count : 1.0;
	out[threadIdx.x] = threadIdx.x == 3u ? count : total / denominator;
}

} // namespace

// Shared with the no-allocation variant of the error pass.
int launchError(const RestirParams* params, const uint16_t* display, const double* mean, const uint8_t* alpha, double* out,
	double* partials, cudaStream_t stream)
{
	const uint32_t n = params->width * params->height;
	errorPartialKernel<<<kErrorBlocks, kErrorThreads, 0, stream>>>(display, mean, alpha, n, partials);
	errorFinalKernel<<<1, 32, 0, stream>>>(partials, kErrorBlocks, out);
	return launchStatus();
}

uint64_t errorScratchBytes()
{
	return uint64_t(kErrorBlocks) * 4u * sizeof(double);
}

namespace
{

// Device address of g_errorNoAllocScratch on each device, looked up once per
// device with that device current (the symbol's name is only a host-side
// handle, not an address a kernel can use).
constexpr int kMaxDevices = 64;
std::mutex g_noAllocMutex;
double* g_noAllocScratch[kMaxDevices] = {};

int noAllocScratch(double** scratch)
{
	int device = 0;
	if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
	{
		return RESTIR_ERROR_LAUNCH;
	}
	std::lock_guard<std::mutex> lock(g_noAllocMutex);
	if (g_noAllocScratch[device] == nullptr)
	{
		void* address = nullptr;
		if (cudaGetSymbolAddress(&address, g_errorNoAllocScratch) != cudaSuccess || address == nullptr)
		{
			return RESTIR_ERROR_LAUNCH;
		}
		g_noAllocScratch[device] = static_cast<double*>(address);
	}
	*scratch = g_noAllocScratch[device];
	return RESTIR_OK;
}

} // namespace

} // namespace restir

using namespace restir;

extern "C" int restir_reference_accumulate(const RestirParams* params, const uint16_t* hdr, double* mean, uint8_t* alpha,
	uint32_t frames, void* stream)
{
	if (params == nullptr || hdr == nullptr || mean == nullptr || alpha == nullptr || params->width == 0 || params->height == 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const uint64_t pixels = uint64_t(params->width) * params->height;
	if (pixels > uint64_t(UINT32_MAX))
	{
		return RESTIR_ERROR_TOO_LARGE;
	}
	const uint32_t n = uint32_t(pixels);
	uint32_t blocks = (n + 255u) / 256u;
	blocks = blocks < 148u * 16u ? blocks : 148u * 16u;
	accumulateKernel<<<blocks, 256, 0, asStream(stream)>>>(hdr, mean, alpha, n, 1.0 / double(frames + 1u));
	return launchStatus();
}

extern "C" uint64_t restir_error_scratch_bytes(uint32_t width, uint32_t height)
{
	(void)width;
	(void)height;
	return errorScratchBytes();
}

extern "C" int restir_error(const RestirParams* params, const uint16_t* display, const double* mean, const uint8_t* alpha,
	double* out, void* scratch, void* stream)
{
	if (params == nullptr || display == nullptr || mean == nullptr || alpha == nullptr || out == nullptr || scratch == nullptr
		|| params->width == 0 || params->height == 0 || (reinterpret_cast<uintptr_t>(scratch) & 7u) != 0u)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	if (uint64_t(params->width) * params->height > uint64_t(UINT32_MAX))
	{
		return RESTIR_ERROR_TOO_LARGE;
	}
	return launchError(params, display, mean, alpha, out, static_cast<double*>(scratch), asStream(stream));
}

// The error pass without caller scratch, for callers that cannot allocate
// device memory (see include/restir_gpu.h). Same two kernels as
// restir_error, launched with one block per 4096 pixels so that the partial
// records fit the library's static array; every block writes its record, so
// the array needs no clearing between calls.
extern "C" int restir_error_noalloc(const RestirParams* params, const uint16_t* display, const double* mean,
	const uint8_t* alpha, double* out, void* stream)
{
	if (params == nullptr || display == nullptr || mean == nullptr || alpha == nullptr || out == nullptr
		|| params->width == 0 || params->height == 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const uint64_t pixels = uint64_t(params->width) * params->height;
	if (pixels > uint64_t(kNoAllocPixelsPerBlock) * kNoAllocMaxBlocks)
	{
		return RESTIR_ERROR_TOO_LARGE;
	}
	double* scratch = nullptr;
	int status = noAllocScratch(&scratch);
	if (status != RESTIR_OK)
	{
		return status;
	}
	const int blocks = int((pixels + kNoAllocPixelsPerBlock - 1) / kNoAllocPixelsPerBlock);
	cudaStream_t s = asStream(stream);
	errorPartialKernel<<<blocks, kErrorThreads, 0, s>>>(display, mean, alpha, uint32_t(pixels), scratch);
	errorFinalKernel<<<1, 32, 0, s>>>(scratch, blocks, out);
	return launchStatus();
}
