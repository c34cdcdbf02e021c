// The display passes after the composite (include/restir_display.h): auto
// exposure (cs_exposure.sc:30-82), TAA (fs_taa.sc:38-172) and tone mapping
// (fs_tonemap.sc:105-162, tonemap.sh:17-122).
//
// All three are HBM-bound image work. The exposure reduction reads 4,096
// texels with one block. TAA and tone mapping run fused, one thread per pixel
// in 16x8 tiles: a pixel's tone mapping needs only that pixel's TAA output,
// so the fused kernel writes the TAA target (the next frame's history) and
// tone-maps the same value, rounded to half as the target stores it, without
// reading it back. The 3x3 neighbourhood and the history's 5 bilinear
// Catmull-Rom taps (16 texels) are served by L1 from the tile's own rows.
#include "common.cuh"

#include "../../include/restir_display.h"

namespace restir
{
namespace
{

// Blocks per SM the display kernel is compiled for: a register cap of 64 (8 blocks
// of 128 threads) runs the fused TAA + AgX launch at 1080p in 0.21 ms against
// 0.27 ms uncapped (109 registers).
#ifndef RESTIR_DISPLAY_MIN_BLOCKS
#define RESTIR_DISPLAY_MIN_BLOCKS 8
#endif

constexpr int kModeTaa = 1;      // TAA into taaOut
constexpr int kModeTonemap = 2;  // tone mapping into display

__device__ __forceinline__ V2 operator/(V2 a, V2 b) { return { a.x / b.x, a.y / b.y }; }
__device__ __forceinline__ V2 operator+(float s, V2 a) { return { s + a.x, s + a.y }; }
__device__ __forceinline__ V2 operator-(float s, V2 a) { return { s - a.x, s - a.y }; }
__device__ __forceinline__ V2 operator*(float s, V2 a) { return { s * a.x, s * a.y }; }
__device__ __forceinline__ V2 floor2(V2 a) { return { floorf(a.x), floorf(a.y) }; }

// fs_taa.sc:43-70
__device__ __forceinline__ V3 toYCoCg(V3 c)
{
	return v3(dot(c, v3(0.25f, 0.5f, 0.25f)), dot(c, v3(0.5f, 0.0f, -0.5f)), dot(c, v3(-0.25f, 0.5f, -0.25f)));
}

__device__ __forceinline__ V3 fromYCoCg(V3 c)
{
	return v3(c.x + c.y - c.z, c.x + c.z, c.x - c.y - c.z);
}

__device__ __forceinline__ V3 compress(V3 c)
{
	return c / (1.0f + luminance(c));
}

__device__ __forceinline__ V3 decompress(V3 c)
{
	return c / fmaxf(1.0f - luminance(c), 0.0001f);
}

// A texel coordinate from a float index, clamped to the edge (NaN: 0).
__device__ __forceinline__ int clampTexel(float f, int size)
{
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

__device__ __forceinline__ V3 loadH3(const uint16_t* p, int i)
{
	return loadH4(p, i).xyz();
}

// Bilinear RGBA16F fetch with clamp to edge.
__device__ __forceinline__ V3 bilinear(const uint16_t* t, int w, int h, V2 uv)
{
	const float px = uv.x * float(w) - 0.5f;
	const float py = uv.y * float(h) - 0.5f;
	const float bx = floorf(px), by = floorf(py);
	const float fx = px - bx, fy = py - by;
	const int x0 = clampTexel(bx, w), x1 = clampTexel(bx + 1.0f, w);
	const int y0 = clampTexel(by, h), y1 = clampTexel(by + 1.0f, h);
	const V3 c00 = loadH3(t, y0 * w + x0), c10 = loadH3(t, y0 * w + x1);
	const V3 c01 = loadH3(t, y1 * w + x0), c11 = loadH3(t, y1 * w + x1);
	return mix(mix(c00, c10, fx), mix(c01, c11, fx), fy);
}

// fs_taa.sc:74-99
__device__ __forceinline__ V3 sampleHistory(const uint16_t* history, int w, int h, V2 uv, V2 texelSize)
{
	const V2 position = uv / texelSize;
	const V2 center = floor2(position - 0.5f) + 0.5f;
	const V2 f = position - center;
	const V2 w0 = f * (-0.5f + f * (1.0f - 0.5f * f));
	const V2 w1 = 1.0f + f * f * (-2.5f + 1.5f * f);
	const V2 w2 = f * (0.5f + f * (2.0f - 1.5f * f));
	const V2 w3 = f * f * (-0.5f + 0.5f * f);
	const V2 w12 = w1 + w2;
	const V2 offset12 = w2 / w12;
	const V2 uv0 = (center - 1.0f) * texelSize;
	const V2 uv3 = (center + 2.0f) * texelSize;
	const V2 uv12 = (center + offset12) * texelSize;
	const V3 color = bilinear(history, w, h, v2(uv12.x, uv0.y)) * (w12.x * w0.y)
		+ bilinear(history, w, h, v2(uv0.x, uv12.y)) * (w0.x * w12.y)
		+ bilinear(history, w, h, v2(uv12.x, uv12.y)) * (w12.x * w12.y)
		+ bilinear(history, w, h, v2(uv3.x, uv12.y)) * (w3.x * w12.y)
		+ bilinear(history, w, h, v2(uv12.x, uv3.y)) * (w12.x * w3.y);
	const float weight = w12.x * w0.y + w0.x * w12.y + w12.x * w12.y + w3.x * w12.y + w12.x * w3.y;
	return vmax(color / weight, v3s(0.0f));
}

// fs_taa.sc:103-109
__device__ __forceinline__ V3 clipToBox(V3 color, V3 center, V3 extent)
{
	const V3 offset = color - center;
	const V3 units = vabs(offset / vmax(extent, v3s(0.00001f)));
	const float largest = fmaxf(units.x, fmaxf(units.y, units.z));
	return largest > 1.0f ? center + offset / largest : color;
}

__device__ __forceinline__ bool anyNan(V3 v)
{
	return v.x != v.x || v.y != v.y || v.z != v.z;
}

// A tile of 16x8 pixels with a one-texel border: each texel's compressed
// YCoCg colour and depth, computed once for the 9 pixels that read it.
constexpr int kTileW = 16, kTileH = 8;
constexpr int kHaloW = kTileW + 2, kHaloH = kTileH + 2;

// Fills the tile of the block at (x0, y0). A neighbour's texture coordinate
// uv + (dx, dy) / size point-samples texel clamp(x + dx, 0, W - 1) exactly
// for sizes up to 16384: the float sum is within 0.01 of the texel centre.
__device__ __forceinline__ void loadNeighbourhood(float4* tile, const uint16_t* __restrict__ hdr,
	const float* __restrict__ depth, int W, int H, int x0, int y0)
{
	for (int k = int(threadIdx.x); k < kHaloW * kHaloH; k += int(blockDim.x))
	{
		const int gx = min(max(x0 + k % kHaloW - 1, 0), W - 1);
		const int gy = min(max(y0 + k / kHaloW - 1, 0), H - 1);
		const int t = gy * W + gx;
		const V3 c = toYCoCg(compress(loadH3(hdr, t)));
		tile[k] = make_float4(c.x, c.y, c.z, loadF1(depth, t));
	}
}

// fs_taa.sc:111-172 for pixel (x, y), at (lx, ly) in the block's tile.
__device__ __forceinline__ V4 taaPixel(const RestirDisplayParams& P, const uint16_t* __restrict__ hdr,
	const float4* tile, const uint16_t* __restrict__ history, int x, int y, int lx, int ly)
{
	const int W = int(P.width), H = int(P.height);
	const V2 texel = v2(1.0f / float(W), 1.0f / float(H));
	const V2 uv = v2((float(x) + 0.5f) * texel.x, (float(y) + 0.5f) * texel.y);
	const V4 current = loadH4(hdr, texelIndex(uv, W, H));

	V3 sum = v3s(0.0f);
	V3 sumSquares = v3s(0.0f);
	float nearestDepth = 1.0f;
	int nearestX = 0, nearestY = 0;
#pragma unroll
	for (int dy = -1; dy <= 1; ++dy)
	{
#pragma unroll
		for (int dx = -1; dx <= 1; ++dx)
		{
			const float4 v = tile[(ly + 1 + dy) * kHaloW + lx + 1 + dx];
			const V3 color = v3(v.x, v.y, v.z);
			sum = sum + color;
			sumSquares = sumSquares + color * color;
			if (v.w < nearestDepth)
			{
				nearestDepth = v.w;
				nearestX = dx;
				nearestY = dy;
			}
		}
	}
	// The nearest tap's texture coordinate, as the shader forms it (uv itself
	// when no tap is nearer than 1: 0 * texel adds nothing).
	const V2 nearestUv = uv + v2(float(nearestX), float(nearestY)) * texel;
	if (P.taa_history_valid < 0.5f)
	{
		return current;
	}

	V3 clipPosition = v3(nearestUv.x * 2.0f - 1.0f, nearestUv.y * 2.0f - 1.0f, nearestDepth);
	clipPosition.y = P.origin_bottom_left > 0.5f ? clipPosition.y : -clipPosition.y;
	const V4 world = mul(P.inv_view_proj, v4(clipPosition, 1.0f));
	const V3 worldPosition = v3(world.x / world.w, world.y / world.w, world.z / world.w);
	const V4 previousClip = mul(P.previous_view_proj, v4(worldPosition, 1.0f));
	V2 previousUv = v2(previousClip.x / previousClip.w, previousClip.y / previousClip.w);
	previousUv = v2(previousUv.x, P.origin_bottom_left > 0.5f ? previousUv.y : -previousUv.y) * 0.5f + 0.5f;
	previousUv = previousUv + (uv - nearestUv);
	if (previousClip.w <= 0.0001f || previousUv.x < 0.0f || previousUv.x > 1.0f || previousUv.y < 0.0f
		|| previousUv.y > 1.0f)
	{
		return current;
	}

	const V3 mean = sum / 9.0f;
	const V3 variance = vmax(sumSquares / 9.0f - mean * mean, v3s(0.0f));
	const V3 deviation = v3(sqrtf(variance.x), sqrtf(variance.y), sqrtf(variance.z));
	V3 past = toYCoCg(compress(sampleHistory(history, W, H, previousUv, texel)));
	past = clipToBox(past, mean, deviation * 1.25f);
	const V3 blended = mix(fromYCoCg(past), compress(current.xyz()), 0.1f);
	V3 result = decompress(blended);
	if (anyNan(result))
	{
		result = anyNan(current.xyz()) ? v3s(0.0f) : current.xyz();
	}
	return v4(result, current.w);
}

// --- tone mapping (tonemap.sh:17-122) -----------------------------------------

__device__ __forceinline__ V3 mulRows(float m0, float m1, float m2, float m3, float m4, float m5, float m6, float m7,
	float m8, V3 v)
{
	return v3(m0 * v.x + m1 * v.y + m2 * v.z, m3 * v.x + m4 * v.y + m5 * v.z, m6 * v.x + m7 * v.y + m8 * v.z);
}

__device__ __forceinline__ V3 clamp01(V3 v)
{
	return v3(clampf(v.x, 0.0f, 1.0f), clampf(v.y, 0.0f, 1.0f), clampf(v.z, 0.0f, 1.0f));
}

__device__ __forceinline__ V3 tonemapAces(V3 c)
{
	V3 color = mulRows(0.59719f, 0.35458f, 0.04823f, 0.07600f, 0.90834f, 0.01566f, 0.02840f, 0.13383f, 0.83777f, c);
	const V3 a = color * (color + 0.0245786f) - 0.000090537f;
	const V3 b = color * (color * 0.983729f + 0.4329510f) + 0.238081f;
	color = mulRows(1.60475f, -0.53108f, -0.07367f, -0.10208f, 1.10813f, -0.00605f, -0.00327f, -0.07276f, 1.07602f, a / b);
	return clamp01(color);
}

__device__ __forceinline__ V3 agxContrast(V3 x)
{
	const V3 x2 = x * x;
	const V3 x4 = x2 * x2;
	return (x4 * 15.5f) * x2 - (x4 * 40.14f) * x + x4 * 31.96f - (x2 * 6.868f) * x + x2 * 0.4298f + x * 0.1191f - 0.00232f;
}

__device__ __forceinline__ float agxLog(float v, float minEv, float maxEv)
{
	return clampf(rn_log2(fmaxf(v, 1e-10f)), minEv, maxEv);
}

__device__ __forceinline__ V3 tonemapAgx(V3 c)
{
	const float minEv = -12.47393f;
	const float maxEv = 4.026069f;
	V3 color = mulRows(0.842479062253094f, 0.0784335999999992f, 0.0792237451477643f, 0.0423282422610123f, 0.878468636469772f,
		0.0791661274605434f, 0.0423756549057051f, 0.0784336f, 0.879142973793104f, vmax(c, v3s(0.0f)));
	color = v3(agxLog(color.x, minEv, maxEv), agxLog(color.y, minEv, maxEv), agxLog(color.z, minEv, maxEv));
	color = (color - minEv) / (maxEv - minEv);
	color = agxContrast(color);
	color = mulRows(1.19687900512017f, -0.0980208811401368f, -0.0990297440797205f, -0.0528968517574562f, 1.15190312990417f,
		-0.0989611768448433f, -0.0529716355144438f, -0.0980434501171241f, 1.15107367264116f, color);
	color = clamp01(color);
	return v3(rn_pow(color.x, 2.2f), rn_pow(color.y, 2.2f), rn_pow(color.z, 2.2f));
}

__device__ __forceinline__ V3 tonemapNeutral(V3 c)
{
	const float startCompression = 0.8f - 0.04f;
	const float desaturation = 0.15f;
	const float x = fminf(c.x, fminf(c.y, c.z));
	const float offset = x < 0.08f ? x - (6.25f * x) * x : 0.04f;
	V3 color = c - offset;
	const float peak = fmaxf(color.x, fmaxf(color.y, color.z));
	if (peak < startCompression)
	{
		return clamp01(color);
	}
	const float d = 1.0f - startCompression;
	const float newPeak = 1.0f - d * d / (peak + d - startCompression);
	color = color * (newPeak / peak);
	const float g = 1.0f - 1.0f / (desaturation * (peak - newPeak) + 1.0f);
	return clamp01(mix(color, v3s(newPeak), g));
}

__device__ __forceinline__ V3 tonemap(V3 c, int op)
{
	if (op == RESTIR_TONEMAP_ACES)
	{
		return tonemapAces(c);
	}
	if (op == RESTIR_TONEMAP_AGX)
	{
		return tonemapAgx(c);
	}
	if (op == RESTIR_TONEMAP_NEUTRAL)
	{
		return tonemapNeutral(c);
	}
	if (op == RESTIR_TONEMAP_REINHARD)
	{
		return c / (c + 1.0f);
	}
	return clamp01(c);
}

// fs_tonemap.sc:106-118
__device__ __forceinline__ V3 turbo(float t)
{
	const float x = clampf(t, 0.0f, 1.0f);
	const float x2 = x * x, x3 = x2 * x;
	const float a = x2 * x2, b = x3 * x2;
	const float r = 1.0f * 0.13572138f + x * 4.61539260f + x2 * -42.66032258f + x3 * 132.13108234f
		+ (a * -152.94239396f + b * 59.28637943f);
	const float g = 1.0f * 0.09140261f + x * 2.19418839f + x2 * 4.84296658f + x3 * -14.18503333f
		+ (a * 4.27729857f + b * 2.82956604f);
	const float bl = 1.0f * 0.10667330f + x * 12.64194608f + x2 * -60.58204836f + x3 * 110.36276771f
		+ (a * -89.90310912f + b * 27.34824973f);
	return v3(r, g, bl);
}

__device__ __forceinline__ V4 background()
{
	return v4(0.125f, 0.141f, 0.169f, 1.0f);
}

// fs_tonemap.sc:122-162 for pixel i.
__device__ __forceinline__ V4 tonemapPixel(const RestirDisplayParams& P, V4 hdr, const uint32_t* __restrict__ exposure,
	const double* __restrict__ mean, const uint8_t* __restrict__ alpha, size_t i, size_t n)
{
	if (P.reference_view > 1.5f)
	{
		const V3 reference = v3(float(mean[i]), float(mean[n + i]), float(mean[2 * n + i]));
		const float referenceAlpha = alpha[i] ? 1.0f : 0.0f;
		const float imageLuminance = luminance(hdr.xyz());
		const float referenceLuminance = luminance(reference);
		const float error = (imageLuminance - referenceLuminance) / fmaxf(referenceLuminance, 0.01f);
		return referenceAlpha < 0.5f ? background() : v4(turbo(0.5f + clampf(error, -0.5f, 0.5f)), 1.0f);
	}
	if (P.reference_view > 0.5f)
	{
		hdr = v4(float(mean[i]), float(mean[n + i]), float(mean[2 * n + i]), alpha[i] ? 1.0f : 0.0f);
	}
	if (P.pass_through > 0.5f)
	{
		return v4(hdr.xyz(), 1.0f);
	}
	if (hdr.w < 0.5f)
	{
		return background();
	}
	float scale = rn_exp2(P.exposure_ev);
	if (P.auto_exposure > 0.5f)
	{
		scale = scale * (0.18f / rn_exp2(__uint_as_float(*exposure)));
	}
	const V3 color = tonemap(hdr.xyz() * scale, int(P.tonemapper));
	const float gamma = 1.0f / 2.2f;
	return v4(rn_pow(fabsf(color.x), gamma), rn_pow(fabsf(color.y), gamma), rn_pow(fabsf(color.z), gamma), 1.0f);
}

// A value as the RGBA16F target holds it.
__device__ __forceinline__ V4 roundHalf4(V4 v)
{
	return v4(__half2float(__float2half_rn(v.x)), __half2float(__float2half_rn(v.y)), __half2float(__float2half_rn(v.z)),
		__half2float(__float2half_rn(v.w)));
}

template<int kMode>
__global__ void __launch_bounds__(128, RESTIR_DISPLAY_MIN_BLOCKS) displayKernel(const RestirDisplayParams P, const uint16_t* __restrict__ hdr,
	const float* __restrict__ depth, const uint16_t* __restrict__ history, uint16_t* __restrict__ taaOut,
	const uint32_t* __restrict__ exposure, const double* __restrict__ mean, const uint8_t* __restrict__ alpha,
	uint8_t* __restrict__ display)
{
	__shared__ float4 tile[kHaloW * kHaloH];
	const int W = int(P.width), H = int(P.height);
	const int lx = int(threadIdx.x) % kTileW, ly = int(threadIdx.x) / kTileW;
	const int x = int(blockIdx.x) * kTileW + lx;
	const int y = int(blockIdx.y) * kTileH + ly;
	if (kMode & kModeTaa)
	{
		loadNeighbourhood(tile, hdr, depth, W, H, int(blockIdx.x) * kTileW, int(blockIdx.y) * kTileH);
		__syncthreads();
	}
	if (x >= W || y >= H)
	{
		return;
	}
	const int i = y * W + x;
	V4 color;
	if (kMode & kModeTaa)
	{
		color = taaPixel(P, hdr, tile, history, x, y, lx, ly);
		storeH4(taaOut, i, color);
		color = roundHalf4(color);
	}
	else
	{
		color = loadH4(hdr, i);
	}
	if (kMode & kModeTonemap)
	{
		storeU8(display, i, tonemapPixel(P, color, exposure, mean, alpha, size_t(i), size_t(W) * size_t(H)));
	}
}

// cs_exposure.sc:30-82: one block of 16x16 threads.
__global__ void __launch_bounds__(256) exposureKernel(const RestirDisplayParams P, const uint16_t* __restrict__ hdr,
	uint32_t* exposure)
{
	__shared__ float logSum[256];
	__shared__ float count[256];
	const int W = int(P.width), H = int(P.height);
	const int index = int(threadIdx.x);
	const float cellX = float(index % 16) * 4.0f, cellY = float(index / 16) * 4.0f;
	float sum = 0.0f, n = 0.0f;
	for (int y = 0; y < 4; ++y)
	{
		for (int x = 0; x < 4; ++x)
		{
			const V2 uv = v2((cellX + float(x) + 0.5f) / 64.0f, (cellY + float(y) + 0.5f) / 64.0f);
			const V4 color = loadH4(hdr, texelIndex(uv, W, H));
			if (color.w > 0.5f)
			{
				const float lum = luminance(color.xyz());
				sum += clampf(rn_log2(fmaxf(lum, 1e-6f)), -12.0f, 12.0f);
				n += 1.0f;
			}
		}
	}
	logSum[index] = sum;
	count[index] = n;
	__syncthreads();
	for (int stride = 128; stride > 0; stride >>= 1)
	{
		if (index < stride)
		{
			logSum[index] += logSum[index + stride];
			count[index] += count[index + stride];
		}
		__syncthreads();
	}
	if (index == 0 && count[0] >= 1.0f)
	{
		const float average = logSum[0] / count[0];
		const float previous = __uint_as_float(exposure[0]);
		const bool reset = P.exposure_reset > 0.5f || !(fabsf(previous) <= 12.0f);
		exposure[0] = __float_as_uint(reset ? average : mixf(previous, average, P.exposure_adapt));
	}
}

bool validSize(const RestirDisplayParams* p)
{
	return p != nullptr && p->width > 0 && p->height > 0 && p->width <= 16384 && p->height <= 16384;
}

bool tonemapInputs(const RestirDisplayParams* p, const uint32_t* exposure, const double* mean, const uint8_t* alpha)
{
	if (p->auto_exposure > 0.5f && p->pass_through <= 0.5f && exposure == nullptr)
	{
		return false;
	}
	return p->reference_view <= 0.5f || (mean != nullptr && alpha != nullptr);
}

template<int kMode>
int launchDisplay(const RestirDisplayParams* p, const uint16_t* hdr, const float* depth, const uint16_t* history,
	uint16_t* taaOut, const uint32_t* exposure, const double* mean, const uint8_t* alpha, uint8_t* display, cudaStream_t s)
{
	dim3 grid((p->width + kTileW - 1) / kTileW, (p->height + kTileH - 1) / kTileH);
	displayKernel<kMode><<<grid, kTileW * kTileH, 0, s>>>(*p, hdr, depth, history, taaOut, exposure, mean, alpha, display);
	return launchStatus();
}

} // namespace
} // namespace restir

using namespace restir;

extern "C" int restir_exposure(const RestirDisplayParams* params, const uint16_t* hdr, uint32_t* exposure, void* stream)
{
	if (!validSize(params) || hdr == nullptr || exposure == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	exposureKernel<<<1, 256, 0, asStream(stream)>>>(*params, hdr, exposure);
	return launchStatus();
}

extern "C" int restir_taa(const RestirDisplayParams* params, const uint16_t* hdr, const float* depth,
	const uint16_t* history, uint16_t* out, void* stream)
{
	if (!validSize(params) || hdr == nullptr || depth == nullptr || history == nullptr || out == nullptr || out == hdr
		|| out == history)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return launchDisplay<kModeTaa>(params, hdr, depth, history, out, nullptr, nullptr, nullptr, nullptr, asStream(stream));
}

extern "C" int restir_tonemap(const RestirDisplayParams* params, const uint16_t* hdr, const uint32_t* exposure,
	const double* reference_mean, const uint8_t* reference_alpha, uint8_t* display, void* stream)
{
	if (!validSize(params) || hdr == nullptr || display == nullptr
		|| !tonemapInputs(params, exposure, reference_mean, reference_alpha))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return launchDisplay<kModeTonemap>(params, hdr, nullptr, nullptr, nullptr, exposure, reference_mean, reference_alpha,
		display, asStream(stream));
}

extern "C" int restir_display(const RestirDisplayParams* params, const uint16_t* hdr, const float* depth,
	const uint16_t* history, uint16_t* taa_out, uint32_t* exposure, const double* reference_mean,
	const uint8_t* reference_alpha, uint8_t* display, void* stream)
{
	if (!validSize(params) || hdr == nullptr || display == nullptr
		|| !tonemapInputs(params, exposure, reference_mean, reference_alpha))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const bool taa = params->taa > 0.5f;
	if (taa && (depth == nullptr || history == nullptr || taa_out == nullptr || taa_out == hdr || taa_out == history))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	cudaStream_t s = asStream(stream);
	if (params->auto_exposure > 0.5f && params->pass_through <= 0.5f)
	{
		exposureKernel<<<1, 256, 0, s>>>(*params, hdr, exposure);
		const int status = launchStatus();
		if (status != RESTIR_OK)
		{
			return status;
		}
	}
	return taa ? launchDisplay<kModeTaa | kModeTonemap>(params, hdr, depth, history, taa_out, exposure, reference_mean,
					 reference_alpha, display, s)
			   : launchDisplay<kModeTonemap>(params, hdr, nullptr, nullptr, nullptr, exposure, reference_mean,
					 reference_alpha, display, s);
}
