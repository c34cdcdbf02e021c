// ReSTIR DI passes: restir_di_temporal (cs_di_temporal.sc:32-180) and
// restir_di_spatial (cs_di_spatial.sc:30-169), with the light-list
// sampling and BRDF of di.sh:53-242 and brdf.sh:14-62. Full resolution, one
// thread per pixel in 16x8 tiles; shadow rays are stackless any-hit
// traversals. The light list's CDF is searched in the read-only cache.
#include "bvh.cuh"
#include "screen.cuh"

// Minimum resident blocks per SM (register budget) of the two DI kernels:
// 8 blocks of 128 threads (64 registers) measured fastest on the 1080p
// frame; the shadow rays are latency-bound, so more warps in flight win
// over the few registers spilled to L1.
#ifndef RESTIR_DI_TEMPORAL_MIN_BLOCKS
#	define RESTIR_DI_TEMPORAL_MIN_BLOCKS 8
#endif
#ifndef RESTIR_DI_SPATIAL_MIN_BLOCKS
#	define RESTIR_DI_SPATIAL_MIN_BLOCKS 8
#endif

namespace restir
{
namespace
{

struct Surface
{
	V3 position;
	V3 normal;
	V3 surfaceNormal;
	V3 albedo;
	float roughness;
	float metallic;
	V3 eye;
	bool valid;
};

// brdf.sh:14-62
__device__ __forceinline__ float distributionGGX(V3 n, V3 h, float roughness)
{
	float alpha = roughness * roughness;
	float alphaSquared = alpha * alpha;
	float nh = fmaxf(dot(n, h), 0.0f);
	float denominator = nh * nh * (alphaSquared - 1.0f) + 1.0f;
	return alphaSquared / fmaxf(kPi * denominator * denominator, 0.0001f);
}

__device__ __forceinline__ float geometrySchlickGGX(float nd, float roughness)
{
	float k = (roughness + 1.0f) * (roughness + 1.0f) / 8.0f;
	return nd / fmaxf(nd * (1.0f - k) + k, 0.0001f);
}

__device__ __forceinline__ void evaluateBrdf(V3 n, V3 v, V3 l, V3 albedo, float roughnessIn, float metallic, V3& diffuse,
	V3& specular)
{
	float normalLight = fmaxf(dot(n, l), 0.0f);
	float normalView = fmaxf(dot(n, v), 0.0f);
	V3 halfway = normalize(v + l);
	V3 f0 = mix(v3s(0.04f), albedo, metallic);
	float cosine = clampf(dot(halfway, v), 0.0f, 1.0f);
	V3 fresnel = f0 + (v3s(1.0f) - f0) * rn_pow5(1.0f - cosine);
	float roughness = fmaxf(roughnessIn, 0.05f);
	float distribution = distributionGGX(n, halfway, roughness);
	float geometry = geometrySchlickGGX(normalLight, roughness) * geometrySchlickGGX(normalView, roughness);
	specular = fresnel * (distribution * geometry) / fmaxf(4.0f * normalLight * normalView, 0.001f) * normalLight;
	diffuse = (v3s(1.0f) - fresnel) * (1.0f - metallic) * albedo / kPi * normalLight;
}

struct DiPass
{
	const RestirParams& P;
	BvhView bvh;
	const float4* lights;
	const uint8_t* albedoTex;
	const uint8_t* normalTex;
	const uint8_t* shadingTex;
	const float* depthTex;
	int W, H;

	__device__ __forceinline__ float s() const { return P.scene_scale; }
	__device__ __forceinline__ float kDiRayBias() const { return 0.01f * s(); }
	__device__ __forceinline__ float kDiReceiverRadius() const { return 0.1f * s(); }
	__device__ __forceinline__ float kDiReceiverPlane() const { return 0.03f * s(); }
	__device__ __forceinline__ float kDiMinDistanceSquared() const { return 0.0001f * s() * s(); }
	__device__ __forceinline__ int lightCount() const { return P.di_light_count; }
	__device__ __forceinline__ V4 lightData(int light, int row) const
	{
		if (!checkedIndex(uint32_t(light), uint32_t(lightCount())))
		{
			return { 0.0f, 0.0f, 0.0f, 0.0f };
		}
		float4 q = __ldg(lights + light * 4 + row);
		return { q.x, q.y, q.z, q.w };
	}
	__device__ __forceinline__ bool isPointLight(int light) const { return lightData(light, 0).w > 0.5f; }

	__device__ __forceinline__ Surface loadSurface(V2 uv) const
	{
		Surface surface;
		int i = texelIndex(uv, W, H);
		float depth = loadF1(depthTex, i);
		V4 albedoRoughness = loadU8(albedoTex, i);
		V4 normalMetallic = loadU8(normalTex, i);
		V4 shading = loadU8(shadingTex, i);
		surface.valid = depth < kSkyDepth;
		surface.position = reconstructWorldPosition(P, uv, fminf(depth, kSkyDepth));
		surface.surfaceNormal = normalize(v3(normalMetallic.x * 2.0f - 1.0f, normalMetallic.y * 2.0f - 1.0f,
			normalMetallic.z * 2.0f - 1.0f));
		surface.normal = normalize(v3(shading.x * 2.0f - 1.0f, shading.y * 2.0f - 1.0f, shading.z * 2.0f - 1.0f));
		surface.albedo = albedoRoughness.xyz();
		surface.roughness = albedoRoughness.w;
		surface.metallic = normalMetallic.w;
		surface.eye = v3(P.camera_position[0], P.camera_position[1], P.camera_position[2]);
		return surface;
	}

	__device__ __forceinline__ int selectLight(float random, float& pmf) const
	{
		int low = 0;
		int high = lightCount() - 1;
		for (int step = 0; step < 24 && low < high; ++step)
		{
			int middle = (low + high) >> 1;
			if (__ldg(&lights[middle * 4 + 2].w) < random)
			{
				low = middle + 1;
			}
			else
			{
				high = middle;
			}
		}
		pmf = __ldg(&lights[low * 4 + 3].w);
		return low;
	}

	__device__ __forceinline__ float triangleArea(int light) const
	{
		V3 v0 = lightData(light, 0).xyz();
		return 0.5f * length(cross(lightData(light, 1).xyz() - v0, lightData(light, 2).xyz() - v0));
	}

	__device__ __forceinline__ V3 sampleLightPoint(int light, float r0, float r1, float& density) const
	{
		V3 v0 = lightData(light, 0).xyz();
		if (isPointLight(light))
		{
			density = 1.0f;
			return v0;
		}
		float root = sqrtf(r0);
		float u = 1.0f - root;
		float v = r1 * root;
		density = 1.0f / fmaxf(triangleArea(light), 1e-12f);
		return v0 + (lightData(light, 1).xyz() - v0) * u + (lightData(light, 2).xyz() - v0) * v;
	}

	__device__ __forceinline__ void evaluateLightSample(const Surface& surface, int light, V3 point, V3& diffuse, V3& specular) const
	{
		diffuse = v3s(0.0f);
		specular = v3s(0.0f);
		if (light < 0 || light >= lightCount())
		{
			return;
		}
		V3 toLight = point - surface.position;
		float distanceSquared = fmaxf(dot(toLight, toLight), kDiMinDistanceSquared());
		V3 direction = toLight * inversesqrt(distanceSquared);
		if (dot(surface.surfaceNormal, direction) <= 0.0f)
		{
			return;
		}
		V3 radiance = lightData(light, 3).xyz() / distanceSquared;
		if (!isPointLight(light))
		{
			V3 v0 = lightData(light, 0).xyz();
			V3 lightNormal = normalize(cross(lightData(light, 1).xyz() - v0, lightData(light, 2).xyz() - v0));
			radiance = radiance * fabsf(dot(lightNormal, direction));
		}
		V3 d, sp;
		evaluateBrdf(surface.normal, normalize(surface.eye - surface.position), direction, surface.albedo, surface.roughness,
			surface.metallic, d, sp);
		diffuse = d * radiance;
		specular = sp * radiance;
	}

	__device__ __forceinline__ float lightTarget(const Surface& surface, int light, V3 point) const
	{
		V3 d, sp;
		evaluateLightSample(surface, light, point, d, sp);
		return luminance(d + sp);
	}

	__device__ __forceinline__ bool lightVisible(const Surface& surface, V3 point) const
	{
		V3 origin = surface.position + surface.surfaceNormal * kDiRayBias();
		V3 toPoint = point - origin;
		float pointDistance = length(toPoint);
		float occluderDistance = 0.0f;
		return traceVisibility(bvh, origin, toPoint / fmaxf(pointDistance, 0.0001f), pointDistance * 0.999f - kDiRayBias(),
			occluderDistance, P.wave_visibility > 0.5f) < 0;
	}

	__device__ __forceinline__ bool sameSurface(V3 p, V3 n, V3 otherP, V3 otherN, float radius) const
	{
		V3 offset = otherP - p;
		return dot(otherN, otherN) > 0.5f && dot(offset, offset) <= radius * radius
			&& fabsf(dot(offset, n)) <= kDiReceiverPlane() && dot(normalize(otherN), n) >= 0.9f;
	}
};

__device__ __forceinline__ DiPass makeDiPass(const RestirParams& P, const BvhView& bvh, const float* lights, const RestirGBuffer& gb)
{
	DiPass d{ P };
	d.bvh = bvh;
	d.lights = reinterpret_cast<const float4*>(lights);
	d.albedoTex = gb.albedo;
	d.normalTex = gb.normal;
	d.shadingTex = gb.shading_normal;
	d.depthTex = gb.depth;
	d.W = int(P.width);
	d.H = int(P.height);
	return d;
}

__global__ void __launch_bounds__(128, RESTIR_DI_TEMPORAL_MIN_BLOCKS) diTemporalKernel(const RestirParams P, BvhView bvh, const float* lights, RestirGBuffer gb,
	RestirDiReservoirs previous, RestirDiReservoirs out)
{
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	DiPass d = makeDiPass(P, bvh, lights, gb);
	if (px >= d.W || py >= d.H)
	{
		return;
	}
	const int i = py * d.W + px;
	const V2 texel = v2(1.0f / float(d.W), 1.0f / float(d.H));
	const V2 uv = pixelUv(px, py, texel);
	const Surface surface = d.loadSurface(uv);
	if (!surface.valid || d.lightCount() == 0)
	{
		storeF4(out.sample, i, v4(0.0f, 0.0f, 0.0f, -1.0f));
		storeF4(out.receiver, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		storeH4(out.normal, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	uint32_t rng = pcg(uint32_t(px) + pcg(uint32_t(py) + pcg(uint32_t(P.frame_index) ^ 0x3c6ef372u)));
	const int candidates = P.di_candidates;
	float weightSum = 0.0f;
	V3 chosenPoint = v3s(0.0f);
	int chosenLight = -1;
	float chosenTarget = 0.0f;
	for (int candidate = 0; candidate < candidates; ++candidate)
	{
		float pmf;
		int light = d.selectLight(nextRandom(rng), pmf);
		float density;
		float r0 = nextRandom(rng);
		float r1 = nextRandom(rng);
		V3 lightPoint = d.sampleLightPoint(light, r0, r1, density);
		float target = d.lightTarget(surface, light, lightPoint);
		float sourcePdf = pmf * density;
		float weight = sourcePdf > 0.0f ? target / sourcePdf : 0.0f;
		weightSum += weight;
		if (nextRandom(rng) * weightSum < weight)
		{
			chosenPoint = lightPoint;
			chosenLight = light;
			chosenTarget = target;
		}
	}
	const float canonicalCount = float(candidates);
	const float canonicalWeight = chosenTarget > 0.0f ? weightSum / (canonicalCount * chosenTarget) : 0.0f;
	const V3 canonicalPoint = chosenPoint;
	const int canonicalLight = chosenLight;
	const float canonicalTarget = chosenTarget;

	float temporalCount = 0.0f;
	float temporalWeight = 0.0f;
	V3 temporalPoint = v3s(0.0f);
	int temporalLight = -1;
	Surface prev = surface;
	const V4 clip = mul(P.prev_view_proj, v4(surface.position, 1.0f));
	if (P.di_history_valid > 0.5f && clip.w > 0.0001f)
	{
		float cy = P.origin_bottom_left > 0.5f ? clip.y : -clip.y;
		V2 puv = v2(clip.x / clip.w * 0.5f + 0.5f, cy / clip.w * 0.5f + 0.5f);
		if (puv.x > 0.0f && puv.x < 1.0f && puv.y > 0.0f && puv.y < 1.0f)
		{
			int j = texelIndex(puv, d.W, d.H);
			V4 sampleData = loadF4(previous.sample, j);
			V4 receiver = loadF4(previous.receiver, j);
			V4 normal = loadH4(previous.normal, j);
			int light = int(sampleData.w + 0.5f);
			if (sampleData.w >= 0.0f && light < d.lightCount()
				&& d.sameSurface(surface.position, surface.normal, receiver.xyz(), normal.xyz(), d.kDiReceiverRadius()))
			{
				temporalCount = fminf(normal.w, 20.0f);
				temporalWeight = receiver.w;
				temporalPoint = sampleData.xyz();
				temporalLight = light;
				prev.position = receiver.xyz();
				prev.normal = normalize(normal.xyz());
				prev.eye = v3(P.prev_camera_position[0], P.prev_camera_position[1], P.prev_camera_position[2]);
			}
		}
	}

	weightSum = 0.0f;
	chosenLight = -1;
	chosenTarget = 0.0f;
	if (canonicalTarget > 0.0f)
	{
		float previousTarget = 0.0f;
		if (temporalCount > 0.0f)
		{
			if (d.lightVisible(prev, canonicalPoint))
			{
				previousTarget = d.lightTarget(prev, canonicalLight, canonicalPoint);
			}
		}
		float denominator = canonicalCount * canonicalTarget + temporalCount * previousTarget;
		float weight = canonicalCount * canonicalTarget / denominator * canonicalTarget * canonicalWeight;
		weightSum += weight;
		chosenPoint = canonicalPoint;
		chosenLight = canonicalLight;
		chosenTarget = canonicalTarget;
	}
	if (temporalCount > 0.0f && temporalWeight > 0.0f)
	{
		float target = d.lightTarget(surface, temporalLight, temporalPoint);
		float previousTarget = d.lightTarget(prev, temporalLight, temporalPoint);
		float denominator = temporalCount * previousTarget + canonicalCount * target;
		float weight = denominator > 0.0f ? temporalCount * previousTarget / denominator * target * temporalWeight : 0.0f;
		weightSum += weight;
		if (weight > 0.0f && nextRandom(rng) * weightSum < weight)
		{
			chosenPoint = temporalPoint;
			chosenLight = temporalLight;
			chosenTarget = target;
		}
	}
	float combinedWeight = chosenTarget > 0.0f ? weightSum / chosenTarget : 0.0f;
	if (combinedWeight > 0.0f)
	{
		if (!d.lightVisible(surface, chosenPoint))
		{
			combinedWeight = 0.0f;
		}
	}
	storeF4(out.sample, i, v4(chosenPoint, float(chosenLight)));
	storeF4(out.receiver, i, v4(surface.position, combinedWeight));
	storeH4(out.normal, i, v4(surface.normal, canonicalCount + temporalCount));
}

__global__ void __launch_bounds__(128, RESTIR_DI_SPATIAL_MIN_BLOCKS) diSpatialKernel(const RestirParams P, BvhView bvh, const float* lights, RestirGBuffer gb,
	RestirDiReservoirs current, uint16_t* diffuseOut, uint16_t* specularOut)
{
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	DiPass d = makeDiPass(P, bvh, lights, gb);
	if (px >= d.W || py >= d.H)
	{
		return;
	}
	const int i = py * d.W + px;
	const V2 texel = v2(1.0f / float(d.W), 1.0f / float(d.H));
	const V2 uv = pixelUv(px, py, texel);
	const Surface surface = d.loadSurface(uv);
	const int own = texelIndex(uv, d.W, d.H);
	const V4 ownSample = loadF4(current.sample, own);
	const V4 ownReceiver = loadF4(current.receiver, own);
	const V4 ownNormal = loadH4(current.normal, own);
	if (!surface.valid || d.lightCount() == 0)
	{
		storeH4(diffuseOut, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		storeH4(specularOut, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	uint32_t rng = pcg(uint32_t(px) + pcg(uint32_t(py) + pcg(uint32_t(P.frame_index) ^ 0x9e3779b9u)));
	const int taps = P.di_spatial_taps;
	const float canonicalCount = fmaxf(fminf(ownNormal.w, 20.0f), 1.0f);
	const int canonicalLight = ownSample.w >= 0.0f ? int(ownSample.w + 0.5f) : -1;
	const V3 canonicalPoint = ownSample.xyz();
	const float canonicalTarget = canonicalLight >= 0 && ownReceiver.w > 0.0f ? d.lightTarget(surface, canonicalLight, canonicalPoint)
		: 0.0f;
	const float pairCanonical = canonicalCount / float(taps > 1 ? taps : 1);
	float totalCount = canonicalCount;
	float canonicalShare = taps > 0 ? 0.0f : canonicalCount;
	float weightSum = 0.0f;
	V3 chosenPoint = canonicalPoint;
	int chosenLight = -1;
	float chosenTarget = 0.0f;
	bool neighbourSelected = false;
	for (int tap = 0; tap < taps; ++tap)
	{
		float radius = 16.0f * sqrtf(nextRandom(rng));
		float angle = 2.0f * kPi * nextRandom(rng);
		float randomSelect = nextRandom(rng);
		float sn, cs;
		rn_sincos(angle, &sn, &cs);
		V2 nuv = v2(uv.x + cs * radius * texel.x, uv.y + sn * radius * texel.y);
		Surface neighbour = d.loadSurface(nuv);
		int j = texelIndex(nuv, d.W, d.H);
		V4 sampleData = loadF4(current.sample, j);
		V4 receiver = loadF4(current.receiver, j);
		V4 normal = loadH4(current.normal, j);
		int light = sampleData.w >= 0.0f ? int(sampleData.w + 0.5f) : -1;
		if (nuv.x <= 0.0f || nuv.x >= 1.0f || nuv.y <= 0.0f || nuv.y >= 1.0f || !neighbour.valid
			|| !d.sameSurface(surface.position, surface.normal, neighbour.position, neighbour.normal, 4.0f * d.kDiReceiverRadius()))
		{
			canonicalShare += pairCanonical;
			continue;
		}
		float neighbourCount = fminf(normal.w, 20.0f);
		float pairWeight = neighbourCount + pairCanonical;
		totalCount += neighbourCount;
		if (canonicalTarget > 0.0f)
		{
			float neighbourTarget = 0.0f;
			if (d.lightVisible(neighbour, canonicalPoint))
			{
				neighbourTarget = d.lightTarget(neighbour, canonicalLight, canonicalPoint);
			}
			float canonicalDensity = pairCanonical * canonicalTarget;
			float denominator = neighbourCount * neighbourTarget + canonicalDensity;
			canonicalShare += pairWeight * canonicalDensity / denominator;
		}
		if (light >= 0 && light < d.lightCount() && receiver.w > 0.0f)
		{
			float target = d.lightTarget(surface, light, sampleData.xyz());
			float neighbourTarget = d.lightTarget(neighbour, light, sampleData.xyz());
			float neighbourDensity = neighbourCount * neighbourTarget;
			float denominator = neighbourDensity + pairCanonical * target;
			float weight = denominator > 0.0f ? pairWeight * neighbourDensity / denominator * target * receiver.w : 0.0f;
			weightSum += weight;
			if (weight > 0.0f && randomSelect * weightSum < weight)
			{
				chosenPoint = sampleData.xyz();
				chosenLight = light;
				chosenTarget = target;
				neighbourSelected = true;
			}
		}
	}
	if (canonicalTarget > 0.0f)
	{
		float weight = canonicalShare * canonicalTarget * ownReceiver.w;
		weightSum += weight;
		if (nextRandom(rng) * weightSum < weight)
		{
			chosenPoint = canonicalPoint;
			chosenLight = canonicalLight;
			chosenTarget = canonicalTarget;
			neighbourSelected = false;
		}
	}
	float combinedWeight = chosenTarget > 0.0f ? weightSum / (totalCount * chosenTarget) : 0.0f;
	if (combinedWeight > 0.0f && neighbourSelected)
	{
		if (!d.lightVisible(surface, chosenPoint))
		{
			combinedWeight = 0.0f;
		}
	}
	V3 diffuse, specular;
	d.evaluateLightSample(surface, chosenLight, chosenPoint, diffuse, specular);
	storeH4(diffuseOut, i, v4(diffuse * combinedWeight, 1.0f));
	storeH4(specularOut, i, v4(specular * combinedWeight, 1.0f));
}

bool validGBuffer(const RestirGBuffer* gb)
{
	return gb != nullptr && gb->albedo != nullptr && gb->normal != nullptr && gb->shading_normal != nullptr && gb->depth != nullptr;
}

} // namespace
} // namespace restir

using namespace restir;

extern "C" int restir_di_temporal(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirDiReservoirs* previous, const RestirDiReservoirs* output, void* stream)
{
	if (params == nullptr || scene == nullptr || !validGBuffer(gbuffer) || previous == nullptr || output == nullptr
		|| output->sample == nullptr || output->receiver == nullptr || output->normal == nullptr
		|| (params->di_light_count > 0 && scene->lights == nullptr) || uint32_t(params->di_light_count) > scene->light_count
		|| (params->di_history_valid > 0.5f && (previous->sample == nullptr || previous->receiver == nullptr || previous->normal == nullptr)))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	dim3 grid((params->width + 15) / 16, (params->height + 7) / 8);
	diTemporalKernel<<<grid, 128, 0, asStream(stream)>>>(*params, makeBvhView(scene), scene->lights, *gbuffer, *previous, *output);
	return launchStatus();
}

extern "C" int restir_di_spatial(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirDiReservoirs* current, uint16_t* diffuse, uint16_t* specular, void* stream)
{
	if (params == nullptr || scene == nullptr || !validGBuffer(gbuffer) || current == nullptr || current->sample == nullptr
		|| current->receiver == nullptr || current->normal == nullptr || diffuse == nullptr || specular == nullptr
		|| (params->di_light_count > 0 && scene->lights == nullptr) || uint32_t(params->di_light_count) > scene->light_count)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	dim3 grid((params->width + 15) / 16, (params->height + 7) / 8);
	diSpatialKernel<<<grid, 128, 0, asStream(stream)>>>(*params, makeBvhView(scene), scene->lights, *gbuffer, *current, diffuse,
		specular);
	return launchStatus();
}
