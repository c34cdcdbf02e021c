/*
 * ORACLE (test infrastructure, never linked into the product).
 *
 * CPU restatement of the display passes that follow the composite, in the
 * shaders' own order of operations:
 *   oracle_exposure  shaders/cs_exposure.sc:30-82
 *   oracle_taa       shaders/fs_taa.sc:38-172
 *   oracle_tonemap   shaders/fs_tonemap.sc:105-162 with shaders/tonemap.sh:17-122
 * and the conventions include/restir_display.h fixes (pixel texture
 * coordinates, point and bilinear sampling, restir_numeric.h's log2, exp2 and
 * pow). bgfx's shaderlib helpers the shaders call (toClipSpaceDepth,
 * toClipSpaceY, clipToWorld, toGamma) are not in the reference; they are
 * restated from bgfx's published shaderlib with NDC depth in [0, 1]:
 * toClipSpaceDepth(d) = d, toClipSpaceY(y) = origin_bottom_left ? y : -y,
 * clipToWorld(M, c) = (M (c, 1)).xyz / w, toGamma(c) = pow(abs(c), 1 / 2.2).
 *
 * Parity status: the reference has no tests or golden images for these
 * passes and its shaders need bgfx, which is absent, so this restatement is
 * "parity unpinned" against the reference itself; the CUDA kernels are
 * checked bit for bit against it.
 */
#include "oracle_common.h"

#include "../include/restir_display.h"

namespace oracle
{
namespace
{

const vec3 kLuminance(0.2126f, 0.7152f, 0.0722f);

/* fs_taa.sc:38-70 */
float luminance(vec3 _color)
{
	return dot(_color, kLuminance);
}

vec3 toYCoCg(vec3 _color)
{
	return vec3(
		  dot(_color, vec3(0.25f, 0.5f, 0.25f))
		, dot(_color, vec3(0.5f, 0.0f, -0.5f))
		, dot(_color, vec3(-0.25f, 0.5f, -0.25f)));
}

vec3 fromYCoCg(vec3 _color)
{
	return vec3(_color.x + _color.y - _color.z, _color.x + _color.z, _color.x - _color.y - _color.z);
}

vec3 compress(vec3 _color)
{
	return _color / (1.0f + luminance(_color));
}

vec3 decompress(vec3 _color)
{
	return _color / max(1.0f - luminance(_color), 0.0001f);
}

/* A texel coordinate from a float index, clamped to the edge (NaN: 0). */
int clampTexel(float _f, int _size)
{
	if (!(_f >= 0.0f))
	{
		return 0;
	}
	if (_f > float(_size - 1))
	{
		return _size - 1;
	}
	return int(_f);
}

/* Bilinear RGBA16F fetch with clamp to edge (restir_display.h). */
vec3 bilinear(const TexH4& _t, vec2 _uv)
{
	const float px = _uv.x * float(_t.w) - 0.5f;
	const float py = _uv.y * float(_t.h) - 0.5f;
	const float bx = floor(px), by = floor(py);
	const float fx = px - bx, fy = py - by;
	const int x0 = clampTexel(bx, _t.w), x1 = clampTexel(bx + 1.0f, _t.w);
	const int y0 = clampTexel(by, _t.h), y1 = clampTexel(by + 1.0f, _t.h);
	const vec3 c00 = _t.at(y0 * _t.w + x0).xyz(), c10 = _t.at(y0 * _t.w + x1).xyz();
	const vec3 c01 = _t.at(y1 * _t.w + x0).xyz(), c11 = _t.at(y1 * _t.w + x1).xyz();
	return mix(mix(c00, c10, fx), mix(c01, c11, fx), fy);
}

/* fs_taa.sc:74-99: Catmull-Rom with five bilinear taps. */
vec3 sampleHistory(const TexH4& _history, vec2 _uv, vec2 _texelSize)
{
	const vec2 position = _uv / _texelSize;
	const vec2 center = floor(position - 0.5f) + 0.5f;
	const vec2 f = position - center;
	const vec2 w0 = f * (-0.5f + f * (1.0f - 0.5f * f));
	const vec2 w1 = 1.0f + f * f * (-2.5f + 1.5f * f);
	const vec2 w2 = f * (0.5f + f * (2.0f - 1.5f * f));
	const vec2 w3 = f * f * (-0.5f + 0.5f * f);
	const vec2 w12 = w1 + w2;
	const vec2 offset12 = w2 / w12;

	const vec2 uv0 = (center - 1.0f) * _texelSize;
	const vec2 uv3 = (center + 2.0f) * _texelSize;
	const vec2 uv12 = (center + offset12) * _texelSize;

	const vec3 color =
		  bilinear(_history, vec2(uv12.x, uv0.y)) * (w12.x * w0.y)
		+ bilinear(_history, vec2(uv0.x, uv12.y)) * (w0.x * w12.y)
		+ bilinear(_history, vec2(uv12.x, uv12.y)) * (w12.x * w12.y)
		+ bilinear(_history, vec2(uv3.x, uv12.y)) * (w3.x * w12.y)
		+ bilinear(_history, vec2(uv12.x, uv3.y)) * (w12.x * w3.y);
	const float weight = w12.x * w0.y + w0.x * w12.y + w12.x * w12.y + w3.x * w12.y + w12.x * w3.y;
	return max(color / weight, vec3_splat(0.0f));
}

/* fs_taa.sc:103-109 */
vec3 clipToBox(vec3 _color, vec3 _center, vec3 _extent)
{
	const vec3 offset = _color - _center;
	const vec3 units = abs(offset / max(_extent, vec3_splat(0.00001f)));
	const float largest = max(units.x, max(units.y, units.z));
	return largest > 1.0f ? _center + offset / largest : _color;
}

bool anyNan(vec3 _v)
{
	return _v.x != _v.x || _v.y != _v.y || _v.z != _v.z;
}

/* fs_taa.sc:111-172 for one pixel. */
vec4 taaPixel(const RestirDisplayParams& P, const TexH4& hdr, const TexF1& depth, const TexH4& history, int x, int y)
{
	const vec2 texel(1.0f / float(P.width), 1.0f / float(P.height));
	const vec2 uv((float(x) + 0.5f) * texel.x, (float(y) + 0.5f) * texel.y);
	const vec4 current = hdr.sample(uv);

	vec3 sum = vec3_splat(0.0f);
	vec3 sumSquares = vec3_splat(0.0f);
	float nearestDepth = 1.0f;
	vec2 nearestUv = uv;
	for (int dy = -1; dy <= 1; ++dy)
	{
		for (int dx = -1; dx <= 1; ++dx)
		{
			const vec2 tapUv = uv + vec2(float(dx), float(dy)) * texel;
			const vec3 color = toYCoCg(compress(hdr.sample(tapUv).xyz()));
			sum += color;
			sumSquares += color * color;
			const float d = depth.sample(tapUv);
			if (d < nearestDepth)
			{
				nearestDepth = d;
				nearestUv = tapUv;
			}
		}
	}

	if (P.taa_history_valid < 0.5f)
	{
		return current;
	}

	vec3 clipPosition = vec3(nearestUv.x * 2.0f - 1.0f, nearestUv.y * 2.0f - 1.0f, nearestDepth);
	clipPosition.y = P.origin_bottom_left > 0.5f ? clipPosition.y : -clipPosition.y;
	const vec4 world = mul(make_mat4(P.inv_view_proj), vec4(clipPosition, 1.0f));
	const vec3 worldPosition = world.xyz() / world.w;
	const vec4 previousClip = mul(make_mat4(P.previous_view_proj), vec4(worldPosition, 1.0f));
	vec2 previousUv = previousClip.xy() / previousClip.w;
	previousUv = vec2(previousUv.x, P.origin_bottom_left > 0.5f ? previousUv.y : -previousUv.y) * 0.5f + 0.5f;
	previousUv += uv - nearestUv;
	if (previousClip.w <= 0.0001f
		|| previousUv.x < 0.0f || previousUv.x > 1.0f || previousUv.y < 0.0f || previousUv.y > 1.0f)
	{
		return current;
	}

	const vec3 mean = sum / 9.0f;
	const vec3 variance = max(sumSquares / 9.0f - mean * mean, vec3_splat(0.0f));
	const vec3 deviation(sqrt(variance.x), sqrt(variance.y), sqrt(variance.z));
	vec3 past = toYCoCg(compress(sampleHistory(history, previousUv, texel)));
	past = clipToBox(past, mean, deviation * 1.25f);

	const vec3 blended = mix(fromYCoCg(past), compress(current.xyz()), 0.1f);
	vec3 result = decompress(blended);
	if (anyNan(result))
	{
		result = anyNan(current.xyz()) ? vec3_splat(0.0f) : current.xyz();
	}
	return vec4(result, current.w);
}

/* tonemap.sh:17-122 */
vec3 mulRows(const float _m[9], vec3 _v)
{
	return vec3(
		  _m[0] * _v.x + _m[1] * _v.y + _m[2] * _v.z
		, _m[3] * _v.x + _m[4] * _v.y + _m[5] * _v.z
		, _m[6] * _v.x + _m[7] * _v.y + _m[8] * _v.z);
}

vec3 clamp01(vec3 _v)
{
	return vec3(clamp(_v.x, 0.0f, 1.0f), clamp(_v.y, 0.0f, 1.0f), clamp(_v.z, 0.0f, 1.0f));
}

vec3 tonemapAces(vec3 _color)
{
	static const float input[9] = { 0.59719f, 0.35458f, 0.04823f, 0.07600f, 0.90834f, 0.01566f, 0.02840f, 0.13383f, 0.83777f };
	static const float output[9] = { 1.60475f, -0.53108f, -0.07367f, -0.10208f, 1.10813f, -0.00605f, -0.00327f, -0.07276f, 1.07602f };
	vec3 color = mulRows(input, _color);
	const vec3 a = color * (color + 0.0245786f) - 0.000090537f;
	const vec3 b = color * (0.983729f * color + 0.4329510f) + 0.238081f;
	color = mulRows(output, a / b);
	return clamp01(color);
}

vec3 agxContrast(vec3 _x)
{
	const vec3 x2 = _x * _x;
	const vec3 x4 = x2 * x2;
	return 15.5f * x4 * x2
		- 40.14f * x4 * _x
		+ 31.96f * x4
		- 6.868f * x2 * _x
		+ 0.4298f * x2
		+ 0.1191f * _x
		- 0.00232f;
}

vec3 tonemapAgx(vec3 _color)
{
	static const float inset[9] = {
		0.842479062253094f, 0.0784335999999992f, 0.0792237451477643f,
		0.0423282422610123f, 0.878468636469772f, 0.0791661274605434f,
		0.0423756549057051f, 0.0784336f, 0.879142973793104f };
	static const float outset[9] = {
		1.19687900512017f, -0.0980208811401368f, -0.0990297440797205f,
		-0.0528968517574562f, 1.15190312990417f, -0.0989611768448433f,
		-0.0529716355144438f, -0.0980434501171241f, 1.15107367264116f };
	const float minEv = -12.47393f;
	const float maxEv = 4.026069f;
	vec3 color = mulRows(inset, max(_color, vec3_splat(0.0f)));
	color = vec3(clamp(rn_log2(max(color.x, 1e-10f)), minEv, maxEv), clamp(rn_log2(max(color.y, 1e-10f)), minEv, maxEv),
		clamp(rn_log2(max(color.z, 1e-10f)), minEv, maxEv));
	color = (color - minEv) / (maxEv - minEv);
	color = agxContrast(color);
	color = mulRows(outset, color);
	color = clamp01(color);
	return vec3(rn_pow(color.x, 2.2f), rn_pow(color.y, 2.2f), rn_pow(color.z, 2.2f));
}

vec3 tonemapNeutral(vec3 _color)
{
	const float startCompression = 0.8f - 0.04f;
	const float desaturation = 0.15f;
	const float x = min(_color.x, min(_color.y, _color.z));
	const float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
	vec3 color = _color - offset;
	const float peak = max(color.x, max(color.y, color.z));
	if (peak < startCompression)
	{
		return clamp01(color);
	}
	const float d = 1.0f - startCompression;
	const float newPeak = 1.0f - d * d / (peak + d - startCompression);
	color *= newPeak / peak;
	const float g = 1.0f - 1.0f / (desaturation * (peak - newPeak) + 1.0f);
	return clamp01(mix(color, vec3_splat(newPeak), g));
}

vec3 tonemap(vec3 _color, int _operator)
{
	if (_operator == RESTIR_TONEMAP_ACES)
	{
		return tonemapAces(_color);
	}
	if (_operator == RESTIR_TONEMAP_AGX)
	{
		return tonemapAgx(_color);
	}
	if (_operator == RESTIR_TONEMAP_NEUTRAL)
	{
		return tonemapNeutral(_color);
	}
	if (_operator == RESTIR_TONEMAP_REINHARD)
	{
		return _color / (_color + vec3_splat(1.0f));
	}
	return clamp01(_color);
}

/* fs_tonemap.sc:106-118 */
vec3 turbo(float _x)
{
	const vec4 red4(0.13572138f, 4.61539260f, -42.66032258f, 132.13108234f);
	const vec4 green4(0.09140261f, 2.19418839f, 4.84296658f, -14.18503333f);
	const vec4 blue4(0.10667330f, 12.64194608f, -60.58204836f, 110.36276771f);
	const vec2 red2(-152.94239396f, 59.28637943f);
	const vec2 green2(4.27729857f, 2.82956604f);
	const vec2 blue2(-89.90310912f, 27.34824973f);
	const float x = clamp(_x, 0.0f, 1.0f);
	const vec4 v4(1.0f, x, x * x, x * x * x);
	const vec2 v2(v4.z * v4.z, v4.w * v4.z);
	const auto dot4 = [](const vec4& a, const vec4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; };
	const auto dot2 = [](const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; };
	return vec3(dot4(v4, red4) + dot2(v2, red2), dot4(v4, green4) + dot2(v2, green2), dot4(v4, blue4) + dot2(v2, blue2));
}

const vec4 kBackground(0.125f, 0.141f, 0.169f, 1.0f);

/* fs_tonemap.sc:122-162 for one pixel: the display colour. */
vec4 tonemapPixel(const RestirDisplayParams& P, vec4 hdr, const uint32_t* exposure, const double* mean,
	const uint8_t* alpha, size_t i, size_t n)
{
	if (P.reference_view > 1.5f)
	{
		const vec4 reference(float(mean[i]), float(mean[n + i]), float(mean[2 * n + i]), alpha[i] ? 1.0f : 0.0f);
		const float imageLuminance = dot(hdr.xyz(), kLuminance);
		const float referenceLuminance = dot(reference.xyz(), kLuminance);
		const float error = (imageLuminance - referenceLuminance) / max(referenceLuminance, 0.01f);
		return reference.w < 0.5f ? kBackground : vec4(turbo(0.5f + clamp(error, -0.5f, 0.5f)), 1.0f);
	}
	if (P.reference_view > 0.5f)
	{
		hdr = vec4(float(mean[i]), float(mean[n + i]), float(mean[2 * n + i]), alpha[i] ? 1.0f : 0.0f);
	}
	if (P.pass_through > 0.5f)
	{
		return vec4(hdr.xyz(), 1.0f);
	}
	if (hdr.w < 0.5f)
	{
		return kBackground;
	}
	float scale = rn_exp2(P.exposure_ev);
	if (P.auto_exposure > 0.5f)
	{
		scale *= 0.18f / rn_exp2(rn_bits_float(exposure[0]));
	}
	const vec3 color = tonemap(hdr.xyz() * scale, int(P.tonemapper));
	return vec4(rn_pow(abs(color.x), 1.0f / 2.2f), rn_pow(abs(color.y), 1.0f / 2.2f), rn_pow(abs(color.z), 1.0f / 2.2f), 1.0f);
}

} // namespace
} // namespace oracle

using namespace oracle;

extern "C" int oracle_exposure(const RestirDisplayParams* P, const uint16_t* hdr_p, uint32_t* exposure)
{
	TexH4 hdr{ hdr_p, int(P->width), int(P->height) };
	float logSum[256], count[256];
	for (int index = 0; index < 256; ++index)
	{
		const vec2 cell(float(index % 16) * 4.0f, float(index / 16) * 4.0f);
		float sum = 0.0f, n = 0.0f;
		for (int y = 0; y < 4; ++y)
		{
			for (int x = 0; x < 4; ++x)
			{
				const vec2 uv = (cell + vec2(float(x), float(y)) + 0.5f) / 64.0f;
				const vec4 color = hdr.sample(uv);
				if (color.w > 0.5f)
				{
					const float lum = dot(color.xyz(), kLuminance);
					sum += clamp(rn_log2(max(lum, 1e-6f)), -12.0f, 12.0f);
					n += 1.0f;
				}
			}
		}
		logSum[index] = sum;
		count[index] = n;
	}
	for (int stride = 128; stride > 0; stride >>= 1)
	{
		for (int index = 0; index < stride; ++index)
		{
			logSum[index] += logSum[index + stride];
			count[index] += count[index + stride];
		}
	}
	if (count[0] < 1.0f)
	{
		return 0;
	}
	const float average = logSum[0] / count[0];
	const float previous = rn_bits_float(exposure[0]);
	const bool reset = P->exposure_reset > 0.5f || !(abs(previous) <= 12.0f);
	const float adapted = reset ? average : mix(previous, average, P->exposure_adapt);
	exposure[0] = rn_float_bits(adapted);
	return 0;
}

extern "C" int oracle_taa(const RestirDisplayParams* P, const uint16_t* hdr_p, const float* depth_p,
	const uint16_t* history_p, uint16_t* out)
{
	const int W = int(P->width), H = int(P->height);
	TexH4 hdr{ hdr_p, W, H };
	TexF1 depth{ depth_p, W, H };
	TexH4 history{ history_p, W, H };
	for (int y = 0; y < H; ++y)
	{
		for (int x = 0; x < W; ++x)
		{
			storeH4(out, y * W + x, taaPixel(*P, hdr, depth, history, x, y));
		}
	}
	return 0;
}

extern "C" int oracle_tonemap(const RestirDisplayParams* P, const uint16_t* hdr_p, const uint32_t* exposure,
	const double* mean, const uint8_t* alpha, uint8_t* display)
{
	const int W = int(P->width), H = int(P->height);
	TexH4 hdr{ hdr_p, W, H };
	const size_t n = size_t(W) * size_t(H);
	for (int y = 0; y < H; ++y)
	{
		for (int x = 0; x < W; ++x)
		{
			const size_t i = size_t(y) * W + x;
			storeU8(display, int(i), tonemapPixel(*P, hdr.at(int(i)), exposure, mean, alpha, i, n));
		}
	}
	return 0;
}
