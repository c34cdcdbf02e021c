// Image-space passes: the SVGF denoiser (svgf.sh:26-36, fs_svgf_variance.sc:29-76,
// fs_svgf_atrous.sc:29-95) at GI resolution, and the composite
// (fs_composite.sc:48-143) at full resolution. One thread per pixel in 16x8
// tiles; the stencil taps hit L1 and L2 (the a-trous footprint at step 16 is
// 64 texels wide, so tiles share few texels, and the GI-resolution targets
// stay resident in the 126 MB L2 across the iterations).
#include "bvh.cuh"
#include "gi.cuh"
#include "screen.cuh"

namespace restir
{
namespace
{

__device__ __forceinline__ float geometryWeight(float sceneScale, V3 p, V3 n, V3 np, V3 nn)
{
	if (dot(nn, nn) < 0.5f)
	{
		return 0.0f;
	}
	float planeDistance = fabsf(dot(n, np - p)) / (0.02f * sceneScale);
	float normalWeight = rn_pow64(fmaxf(dot(n, normalize(nn)), 0.0f));
	return rn_exp(-planeDistance) * normalWeight;
}

__device__ __forceinline__ bool isInside(V2 uv)
{
	return uv.x >= 0.0f && uv.x <= 1.0f && uv.y >= 0.0f && uv.y <= 1.0f;
}

__device__ __forceinline__ V3 xyz4(const float4* p, int i)
{
	float4 q = __ldg(p + i);
	return v3(q.x, q.y, q.z);
}

__global__ void __launch_bounds__(128) varianceKernel(const RestirParams P, const uint16_t* __restrict__ color,
	const uint16_t* __restrict__ moments, const float4* __restrict__ receiver, const float4* __restrict__ normal, uint16_t* out)
{
	const int w = int(P.gi_width), h = int(P.gi_height);
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	if (px >= w || py >= h)
	{
		return;
	}
	const int i = py * w + px;
	const V2 texel = v2(1.0f / float(w), 1.0f / float(h));
	const V2 uv = pixelUv(px, py, texel);
	const int c = texelIndex(uv, w, h);
	V3 n = xyz4(normal, c);
	if (dot(n, n) < 0.5f)
	{
		storeH4(out, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	n = normalize(n);
	const V3 col = loadH4(color, c).xyz();
	const V4 m = loadH4(moments, c);
	const float historyLength = m.z;
	if (historyLength >= 4.0f)
	{
		storeH4(out, i, v4(col, fmaxf(m.y - m.x * m.x, 0.0f)));
		return;
	}
	const V3 position = xyz4(receiver, c);
	float sumX = 0.0f, sumY = 0.0f;
	float weightSum = 0.0f;
	for (int y = -3; y <= 3; ++y)
	{
		for (int x = -3; x <= 3; ++x)
		{
			V2 tap = v2(uv.x + float(x) * texel.x, uv.y + float(y) * texel.y);
			if (!isInside(tap))
			{
				continue;
			}
			int j = texelIndex(tap, w, h);
			float weight = geometryWeight(P.scene_scale, position, n, xyz4(receiver, j), xyz4(normal, j));
			V4 mj = loadH4(moments, j);
			sumX += mj.x * weight;
			sumY += mj.y * weight;
			weightSum += weight;
		}
	}
	const float denominator = fmaxf(weightSum, 0.0001f);
	const float mx = sumX / denominator;
	const float my = sumY / denominator;
	const float variance = fmaxf(my - mx * mx, 0.0f) * (4.0f / fmaxf(historyLength, 1.0f));
	storeH4(out, i, v4(col, variance));
}

__device__ __forceinline__ float splineWeight(int offset)
{
	int d = offset < 0 ? -offset : offset;
	return d == 0 ? 0.375f : (d == 1 ? 0.25f : 0.0625f);
}

__global__ void __launch_bounds__(128) atrousKernel(const RestirParams P, int step, const uint16_t* __restrict__ input,
	const float4* __restrict__ receiver, const float4* __restrict__ normal, uint16_t* out)
{
	const int w = int(P.gi_width), h = int(P.gi_height);
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	if (px >= w || py >= h)
	{
		return;
	}
	const int i = py * w + px;
	const V2 texel = v2(1.0f / float(w), 1.0f / float(h));
	const V2 uv = pixelUv(px, py, texel);
	const int c = texelIndex(uv, w, h);
	V3 n = xyz4(normal, c);
	if (dot(n, n) < 0.5f)
	{
		storeH4(out, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	n = normalize(n);
	const V3 position = xyz4(receiver, c);
	const V4 center = loadH4(input, c);
	const float centerLuminance = luminance(center.xyz());
	float variance = 0.0f;
	for (int by = -1; by <= 1; ++by)
	{
		for (int bx = -1; bx <= 1; ++bx)
		{
			float weight = (bx == 0 ? 0.5f : 0.25f) * (by == 0 ? 0.5f : 0.25f);
			V2 tap = v2(uv.x + float(bx) * texel.x, uv.y + float(by) * texel.y);
			variance += loadH4(input, texelIndex(tap, w, h)).w * weight;
		}
	}
	const float luminanceScale = 1.0f / (4.0f * sqrtf(fmaxf(variance, 0.0f)) + 0.0001f);
	const float stepSize = float(step);
	const V2 spacing = v2(stepSize * texel.x, stepSize * texel.y);
	// The taps' texel columns and rows (the coordinates are separable: a tap's
	// u depends on x only, its v on y only), -1 outside the image.
	int columns[5];
	int rows[5];
	for (int k = 0; k < 5; ++k)
	{
		const float u = uv.x + float(k - 2) * spacing.x;
		const float v = uv.y + float(k - 2) * spacing.y;
		columns[k] = u >= 0.0f && u <= 1.0f ? texelCoord(u, w) : -1;
		rows[k] = v >= 0.0f && v <= 1.0f ? texelCoord(v, h) * w : -1;
	}
	V3 colorSum = v3s(0.0f);
	float varianceSum = 0.0f;
	float weightSum = 0.0f;
	for (int y = -2; y <= 2; ++y)
	{
		for (int x = -2; x <= 2; ++x)
		{
			if (rows[y + 2] < 0 || columns[x + 2] < 0)
			{
				continue;
			}
			int j = rows[y + 2] + columns[x + 2];
			V4 tap = loadH4(input, j);
			float weight = splineWeight(x) * splineWeight(y);
			if (x != 0 || y != 0)
			{
				weight *= geometryWeight(P.scene_scale, position, n, xyz4(receiver, j), xyz4(normal, j));
				weight *= rn_exp(-fabsf(luminance(tap.xyz()) - centerLuminance) * luminanceScale);
			}
			colorSum = colorSum + tap.xyz() * weight;
			varianceSum += tap.w * weight * weight;
			weightSum += weight;
		}
	}
	storeH4(out, i, v4(colorSum / weightSum, varianceSum / (weightSum * weightSum)));
}

// The split-sum specular albedo, brdf.sh:68-76 (Karis' analytic fit).
__device__ __forceinline__ V3 compositeSpecularAlbedo(V3 f0, float roughness, float normalView)
{
	const float rx = -1.0f * roughness + 1.0f, ry = -0.0275f * roughness + 0.0425f;
	const float rz = -0.572f * roughness + 1.04f, rw = 0.022f * roughness + -0.04f;
	const float a004 = fminf(rx * rx, rn_exp2(-9.28f * normalView)) * rx + ry;
	const float scale = -1.04f * a004 + rz, bias = 1.04f * a004 + rw;
	return f0 * scale + bias;
}

// fs_composite.sc:48-143 with the final view's options; the indirect
// specular when a specular target is given.
__global__ void __launch_bounds__(128) compositeKernel(const RestirParams P, RestirGBuffer gb, const float* __restrict__ atlas,
	const uint16_t* __restrict__ gi, const uint16_t* __restrict__ diDiffuse, const uint16_t* __restrict__ diSpecular,
	const uint16_t* __restrict__ specularTarget, uint16_t* hdr)
{
	const int W = int(P.width), H = int(P.height);
	const int w = int(P.gi_width), h = int(P.gi_height);
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	if (px >= W || py >= H)
	{
		return;
	}
	const int i = py * W + px;
	const V2 texel = v2(1.0f / float(W), 1.0f / float(H));
	const V2 uv = pixelUv(px, py, texel);
	const V3 camera = v3(P.camera_position[0], P.camera_position[1], P.camera_position[2]);
	const int c = texelIndex(uv, W, H);
	const float depth = loadF1(gb.depth, c);
	if (depth >= 0.99999f)
	{
		V3 farPosition = reconstructWorldPosition(P, uv, 1.0f);
		V3 direction = normalize(farPosition - camera);
		storeH4(hdr, i, skyEnabled(P) ? v4(skyRadiance(P, direction), 1.0f) : v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	const V4 albedoRoughness = loadU8(gb.albedo, c);
	const V4 normalMetallic = loadU8(gb.normal, c);
	const V3 albedo = albedoRoughness.xyz();
	const float roughness = fmaxf(albedoRoughness.w, 0.05f);
	const float metallic = normalMetallic.w;
	const V3 surfaceNormal = normalize(v3(normalMetallic.x * 2.0f - 1.0f, normalMetallic.y * 2.0f - 1.0f, normalMetallic.z * 2.0f - 1.0f));
	const V4 sh = loadU8(gb.shading_normal, c);
	const V3 normal = normalize(v3(sh.x * 2.0f - 1.0f, sh.y * 2.0f - 1.0f, sh.z * 2.0f - 1.0f));
	const V4 emissiveOcclusion = loadH4(gb.emissive, c);
	const V3 position = reconstructWorldPosition(P, uv, depth);
	const V3 viewDirection = normalize(camera - position);
	const V3 lightPosition = v3(P.light_position[0], P.light_position[1], P.light_position[2]);
	const V3 lightColor = v3(P.light_color[0], P.light_color[1], P.light_color[2]);
	const float s = P.scene_scale;
	const V3 toLight = lightPosition - position;
	const float distanceSquared = fmaxf(dot(toLight, toLight), 0.01f * s * s);
	const V3 lightDirection = toLight * inversesqrt(distanceSquared);

	// evaluateBrdf (brdf.sh:41-62)
	const float normalLight = fmaxf(dot(normal, lightDirection), 0.0f);
	const float normalView = fmaxf(dot(normal, viewDirection), 0.0f);
	const V3 halfway = normalize(viewDirection + lightDirection);
	const V3 f0 = mix(v3s(0.04f), albedo, metallic);
	const float cosine = clampf(dot(halfway, viewDirection), 0.0f, 1.0f);
	const V3 fresnel = f0 + (v3s(1.0f) - f0) * rn_pow5(1.0f - cosine);
	const float rough = fmaxf(roughness, 0.05f);
	const float alpha = rough * rough;
	const float alphaSquared = alpha * alpha;
	const float nh = fmaxf(dot(normal, halfway), 0.0f);
	const float dd = nh * nh * (alphaSquared - 1.0f) + 1.0f;
	const float distribution = alphaSquared / fmaxf(kPi * dd * dd, 0.0001f);
	const float k = (rough + 1.0f) * (rough + 1.0f) / 8.0f;
	const float gl = normalLight / fmaxf(normalLight * (1.0f - k) + k, 0.0001f);
	const float gv = normalView / fmaxf(normalView * (1.0f - k) + k, 0.0001f);
	const float geometry = gl * gv;
	const V3 specular = fresnel * (distribution * geometry) / fmaxf(4.0f * normalLight * normalView, 0.001f) * normalLight;
	const V3 diffuse = (v3s(1.0f) - fresnel) * (1.0f - metallic) * albedo / kPi * normalLight;

	float visibility = 0.0f;
	if (dot(normal, lightDirection) > 0.0f)
	{
		visibility = lightVisibilitySoft(P, atlas, position, surfaceNormal);
	}
	const V3 direct = (diffuse + specular) * (lightColor / distanceSquared) * visibility + loadH4(diDiffuse, c).xyz()
		+ loadH4(diSpecular, c).xyz();

	// upsampleIndirect (fs_composite.sc:48-80), diffuse part.
	const V2 texelCoord = v2(uv.x * float(w) - 0.5f, uv.y * float(h) - 0.5f);
	const V2 baseCoord = v2(floorf(texelCoord.x), floorf(texelCoord.y));
	const V2 blend = texelCoord - baseCoord;
	const V2 giTexel = v2(1.0f / float(w), 1.0f / float(h));
	V3 sum = v3s(0.0f);
	V3 specularSum = v3s(0.0f);
	float weightSum = 0.0f;
	for (int tapIndex = 0; tapIndex < 4; ++tapIndex)
	{
		const V2 offset = v2(float(tapIndex & 1), float(tapIndex >> 1));
		const V2 tapUv = v2((baseCoord.x + offset.x + 0.5f) * giTexel.x, (baseCoord.y + offset.y + 0.5f) * giTexel.y);
		const int t = texelIndex(tapUv, W, H);
		const float tapDepth = loadF1(gb.depth, t);
		if (tapDepth >= 0.99999f)
		{
			continue;
		}
		const V3 tapPosition = reconstructWorldPosition(P, tapUv, tapDepth);
		const V3 tapNormal = decodeNormal(gb.normal, t);
		const V2 bilinear = v2(mixf(1.0f - blend.x, blend.x, offset.x), mixf(1.0f - blend.y, blend.y, offset.y));
		const float weight = (bilinear.x * bilinear.y + 0.01f) * stepf(fabsf(dot(tapPosition - position, surfaceNormal)), 0.03f * s)
			* stepf(0.9f, dot(tapNormal, surfaceNormal));
		sum = sum + loadH4(gi, texelIndex(tapUv, w, h)).xyz() * weight;
		if (specularTarget != nullptr)
		{
			specularSum = specularSum + loadH4(specularTarget, texelIndex(tapUv, w, h)).xyz() * weight;
		}
		weightSum += weight;
	}
	const V3 irradiance = weightSum > 0.0f ? sum / weightSum : loadH4(gi, texelIndex(uv, w, h)).xyz();
	V3 indirect = irradiance
		* (P.composite_options[2] > 0.5f ? albedo * (1.0f - metallic) * emissiveOcclusion.w : v3s(1.0f));
	if (specularTarget != nullptr)
	{
		// fs_composite.sc:131-136
		const V3 specularRadiance = weightSum > 0.0f ? specularSum / weightSum
			: loadH4(specularTarget, texelIndex(uv, w, h)).xyz();
		indirect = indirect + specularRadiance * compositeSpecularAlbedo(f0, roughness, fmaxf(dot(normal, viewDirection), 0.001f))
			* emissiveOcclusion.w * P.composite_specular;
	}
	const V3 result = direct * P.composite_options[0] + indirect * P.composite_options[1]
		+ emissiveOcclusion.xyz() * P.composite_options[3];
	storeH4(hdr, i, v4(result, 1.0f));
}

} // namespace
} // namespace restir

using namespace restir;

extern "C" int restir_svgf_variance(const RestirParams* params, const uint16_t* color, const uint16_t* moments,
	const float* receiver, const float* normal, uint16_t* output, void* stream)
{
	if (params == nullptr || color == nullptr || moments == nullptr || receiver == nullptr || normal == nullptr || output == nullptr
		|| params->gi_width == 0 || params->gi_height == 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	dim3 grid((params->gi_width + 15) / 16, (params->gi_height + 7) / 8);
	varianceKernel<<<grid, 128, 0, asStream(stream)>>>(*params, color, moments, reinterpret_cast<const float4*>(receiver),
		reinterpret_cast<const float4*>(normal), output);
	return launchStatus();
}

extern "C" int restir_svgf_atrous(const RestirParams* params, int step, const uint16_t* input, const float* receiver,
	const float* normal, uint16_t* output, void* stream)
{
	if (params == nullptr || input == nullptr || receiver == nullptr || normal == nullptr || output == nullptr || step < 1
		|| params->gi_width == 0 || params->gi_height == 0 || input == output)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	dim3 grid((params->gi_width + 15) / 16, (params->gi_height + 7) / 8);
	atrousKernel<<<grid, 128, 0, asStream(stream)>>>(*params, step, input, reinterpret_cast<const float4*>(receiver),
		reinterpret_cast<const float4*>(normal), output);
	return launchStatus();
}

extern "C" int restir_composite(const RestirParams* params, const RestirGBuffer* gbuffer, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, uint16_t* hdr, void* stream)
{
	if (params == nullptr || gbuffer == nullptr || gbuffer->albedo == nullptr || gbuffer->normal == nullptr
		|| gbuffer->emissive == nullptr || gbuffer->shading_normal == nullptr || gbuffer->depth == nullptr
		|| shadow_atlas == nullptr || gi == nullptr || hdr == nullptr || params->width == 0 || params->height == 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	dim3 grid((params->width + 15) / 16, (params->height + 7) / 8);
	compositeKernel<<<grid, 128, 0, asStream(stream)>>>(*params, *gbuffer, shadow_atlas, gi, di_diffuse, di_specular, nullptr,
		hdr);
	return launchStatus();
}

extern "C" int restir_composite_specular(const RestirParams* params, const RestirGBuffer* gbuffer, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, const uint16_t* specular, uint16_t* hdr,
	void* stream)
{
	if (params == nullptr || gbuffer == nullptr || gbuffer->albedo == nullptr || gbuffer->normal == nullptr
		|| gbuffer->emissive == nullptr || gbuffer->shading_normal == nullptr || gbuffer->depth == nullptr
		|| shadow_atlas == nullptr || gi == nullptr || hdr == nullptr || params->width == 0 || params->height == 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	dim3 grid((params->width + 15) / 16, (params->height + 7) / 8);
	compositeKernel<<<grid, 128, 0, asStream(stream)>>>(*params, *gbuffer, shadow_atlas, gi, di_diffuse, di_specular, specular,
		hdr);
	return launchStatus();
}
