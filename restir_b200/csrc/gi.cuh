// ReSTIR GI device code: the shared functions of shaders/restir.sh
// (lines 117-931) with the shadow-atlas lookup of shadow.sh (31-133) and the
// sky of sky.sh (15-31), in the same order of operations as the shader, so
// that every reservoir matches the CPU restatement bit for bit.
#pragma once

#include "bvh.cuh"
#include "grid.cuh"
#include "screen.cuh"

namespace restir
{

struct GiReservoir
{
	V3 contribution;
	V3 position;
	V3 normal;
	float id;
	float target;
	float weightSum;
	float count;
};

__device__ __forceinline__ GiReservoir emptyReservoir()
{
	GiReservoir r;
	r.contribution = v3s(0.0f);
	r.position = v3s(0.0f);
	r.normal = v3(0.0f, 0.0f, 1.0f);
	r.id = 0.0f;
	r.target = 0.0f;
	r.weightSum = 0.0f;
	r.count = 0.0f;
	return r;
}

__device__ __forceinline__ bool updateReservoir(GiReservoir& r, V3 contribution, V3 position, V3 normal, float id,
	float target, float weight, float random)
{
	r.weightSum += weight;
	if (random * r.weightSum < weight)
	{
		r.contribution = contribution;
		r.position = position;
		r.normal = normal;
		r.id = id;
		r.target = target;
		return true;
	}
	return false;
}

struct NeighbourReservoir
{
	V3 samplePosition;
	float sampleId;
	V3 receiverPosition;
	V3 receiverNormal;
	float count;
	float weight;
	int cacheSlot;  // the radiance cache's value for this sample, or -1
};

struct PairwiseMis
{
	GiReservoir combined;
	V3 canonicalPosition;
	V3 canonicalNormal;
	float canonicalId;
	float pairCanonical;
	float canonicalGeometry;
	float canonicalShare;
	float totalCount;
	bool hasCanonical;
	bool neighbourSelected;
};

__device__ __forceinline__ bool isSkySample(float id)
{
	return id > kSkySampleId * 0.5f;
}

// shadow.sh:31-108
__device__ __forceinline__ int shadowFace(V3 d)
{
	V3 a = vabs(d);
	if (a.x >= a.y && a.x >= a.z)
	{
		return d.x >= 0.0f ? 0 : 1;
	}
	if (a.y >= a.z)
	{
		return d.y >= 0.0f ? 2 : 3;
	}
	return d.z >= 0.0f ? 4 : 5;
}

__device__ __forceinline__ V2 shadowAtlasUv(const RestirParams& P, V3 position, int face)
{
	V4 clip = mul(P.shadow_view_proj[face], v4(position, 1.0f));
	V2 ndc = v2(clip.x / clip.w, clip.y / clip.w);
	bool originBottomLeft = P.origin_bottom_left > 0.5f;
	V2 local = v2(ndc.x * 0.5f + 0.5f, originBottomLeft ? ndc.y * 0.5f + 0.5f : 0.5f - ndc.y * 0.5f);
	float row = face >= 3 ? 1.0f : 0.0f;
	float column = float(face) - 3.0f * row;
	if (originBottomLeft)
	{
		row = 1.0f - row;
	}
	return v2((column + local.x) * (1.0f / 3.0f), (row + local.y) * 0.5f);
}

__device__ __forceinline__ bool shadowLookup(const RestirParams& P, V3 p, V3 n, float filterRadius, V2& uv, float& reference)
{
	uv = v2(0.0f, 0.0f);
	reference = 0.0f;
	if (P.shadows_enabled < 0.5f)
	{
		return false;
	}
	V3 light = v3(P.light_position[0], P.light_position[1], P.light_position[2]);
	float lightDistance = length(light - p);
	float texelSize = 2.0f * lightDistance * P.shadow_tan_half_fov * P.shadow_inv_face_size;
	V3 position = p + n * (texelSize * 1.5f);
	V3 fromLight = position - light;
	uv = shadowAtlasUv(P, position, shadowFace(fromLight));
	float cosine = clampf(dot(n, -normalize(fromLight)), 0.0f, 1.0f);
	float slope = fminf(sqrtf(1.0f - cosine * cosine) / fmaxf(cosine, 0.0001f), 8.0f);
	float bias = texelSize * (1.0f + filterRadius * slope);
	reference = (length(fromLight) - bias) / P.shadow_far;
	return true;
}

__device__ __forceinline__ float lightVisibilityHard(const RestirParams& P, const float* atlas, V3 p, V3 n)
{
	V2 uv;
	float reference;
	if (!shadowLookup(P, p, n, 0.5f, uv, reference))
	{
		return 1.0f;
	}
	int f = int(P.shadow_face_size);
	return reference <= loadF1(atlas, texelIndex(uv, 3 * f, 2 * f)) ? 1.0f : 0.0f;
}

__device__ __forceinline__ float lightVisibilitySoft(const RestirParams& P, const float* atlas, V3 p, V3 n)
{
	V2 uv;
	float reference;
	if (!shadowLookup(P, p, n, 2.0f, uv, reference))
	{
		return 1.0f;
	}
	int f = int(P.shadow_face_size);
	V2 atlasTexel = v2(P.shadow_inv_face_size / 3.0f, P.shadow_inv_face_size * 0.5f);
	float lit = 0.0f;
	for (int y = 0; y < 4; ++y)
	{
		for (int x = 0; x < 4; ++x)
		{
			V2 offset = v2((float(x) - 1.5f) * atlasTexel.x, (float(y) - 1.5f) * atlasTexel.y);
			lit += reference <= loadF1(atlas, texelIndex(uv + offset, 3 * f, 2 * f)) ? 1.0f : 0.0f;
		}
	}
	return lit / 16.0f;
}

// sky.sh:15-31
__device__ __forceinline__ bool skyEnabled(const RestirParams& P)
{
	return P.sky_zenith[3] > 0.5f;
}

__device__ __forceinline__ V3 skyRadiance(const RestirParams& P, V3 d)
{
	if (!skyEnabled(P))
	{
		return v3s(0.0f);
	}
	V3 zenith = v3(P.sky_zenith[0], P.sky_zenith[1], P.sky_zenith[2]);
	V3 horizon = v3(P.sky_horizon[0], P.sky_horizon[1], P.sky_horizon[2]);
	V3 ground = v3(P.sky_ground[0], P.sky_ground[1], P.sky_ground[2]);
	float height = clampf(d.y, -1.0f, 1.0f);
	return height >= 0.0f ? mix(horizon, zenith, sqrtf(height)) : mix(horizon, ground, sqrtf(-height));
}

// The resources a GI pass binds (renderer.cpp:772-802) and restir.sh's
// functions over them.
struct GiPass
{
	const RestirParams& P;
	BvhView bvh;
	GridView grid;
	const uint8_t* albedoTex;
	const uint8_t* normalTex;
	const float* depthTex;
	const float4* historyNormal;
	const float4* historyReceiver;
	const uint16_t* historyColor;
	const uint16_t* surfaceLight;
	const float* shadowAtlas;
	int* stack;      // short-stack storage of this thread (temporal pass), or null
	int stackStride;
	int W, H, w, h;
	V2 giSize, giTexel;
	// Radiance-cache values (half4: irradiance, valid) indexed by a slot, in
	// place of previousIndirect when P.radiance_cache is set; reused
	// neighbours' samples sit at cacheNeighbourBase + their pixel index.
	const uint16_t* cache;
	int cacheNeighbourBase;

	__device__ __forceinline__ float s() const { return P.scene_scale; }
	__device__ __forceinline__ float kRayBias() const { return 0.02f * s(); }
	__device__ __forceinline__ float kSurfaceBias() const { return 0.01f * s(); }
	__device__ __forceinline__ float kMaxRayDistance() const { return 3.6f * s(); }
	__device__ __forceinline__ float kMaxBvhRayDistance() const { return 4.0f * s(); }
	__device__ __forceinline__ float kSampleTolerance() const { return 0.1f * s(); }
	__device__ __forceinline__ float kReceiverRadius() const { return 0.4f * s(); }
	__device__ __forceinline__ float kReceiverPlane() const { return 0.03f * s(); }
	__device__ __forceinline__ float kMinDistanceSquared() const { return 0.0001f * s() * s(); }
	__device__ __forceinline__ float kBounceRadius() const { return 0.1f * s(); }
	__device__ __forceinline__ V3 lightPosition() const { return v3(P.light_position[0], P.light_position[1], P.light_position[2]); }
	__device__ __forceinline__ V3 lightColor() const { return v3(P.light_color[0], P.light_color[1], P.light_color[2]); }

	__device__ __forceinline__ int full(V2 uv) const { return texelIndex(uv, W, H); }
	__device__ __forceinline__ int gi(V2 uv) const { return texelIndex(uv, w, h); }

	__device__ __forceinline__ V3 diffuseAlbedo(V2 uv) const
	{
		int i = full(uv);
		V3 albedo = loadU8(albedoTex, i).xyz();
		float metallic = loadU8(normalTex, i).w;
		return albedo * (1.0f - metallic);
	}

	__device__ __forceinline__ V3 decode(V2 uv) const { return decodeNormal(normalTex, full(uv)); }
	__device__ __forceinline__ float depthAt(V2 uv) const { return loadF1(depthTex, full(uv)); }

	__device__ __forceinline__ V2 giPixelUv(uint32_t index) const
	{
		uint32_t width = uint32_t(giSize.x);
		return v2((float(index % width) + 0.5f) * giTexel.x, (float(index / width) + 0.5f) * giTexel.y);
	}

	__device__ __forceinline__ bool projectToScreen(V3 p, V2& uv, float& viewDepth) const
	{
		V4 clip = mul(P.view_proj, v4(p, 1.0f));
		viewDepth = clip.w;
		uv = v2(0.0f, 0.0f);
		if (clip.w <= 0.0001f)
		{
			return false;
		}
		uv = clipToUv(P, clip);
		return isOnScreen(uv);
	}

	__device__ __forceinline__ static V3 cosineHemisphere(V3 n, float r0, float r1)
	{
		float radius = sqrtf(r0);
		float angle = 2.0f * kPi * r1;
		float sn, cs;
		rn_sincos(angle, &sn, &cs);
		V3 local = v3(radius * cs, radius * sn, sqrtf(fmaxf(1.0f - r0, 0.0f)));
		V3 tangent = normalize(fabsf(n.y) < 0.99f ? cross(n, v3(0.0f, 1.0f, 0.0f)) : cross(n, v3(1.0f, 0.0f, 0.0f)));
		V3 bitangent = cross(n, tangent);
		return normalize(tangent * local.x + bitangent * local.y + n * local.z);
	}

	__device__ __forceinline__ V3 directFromLight(V3 albedo, V3 p, V3 n) const
	{
		V3 toLight = lightPosition() - p;
		float distanceSquared = fmaxf(dot(toLight, toLight), 0.01f * s() * s());
		float normalLight = fmaxf(dot(n, toLight * inversesqrt(distanceSquared)), 0.0f);
		V3 direct = v3s(0.0f);
		if (normalLight > 0.0f)
		{
			direct = albedo * (lightColor() / distanceSquared) * (normalLight / kPi) * lightVisibilityHard(P, shadowAtlas, p, n);
		}
		return direct;
	}

	__device__ __forceinline__ float encodeSampleId(int t, V3 d) const
	{
		V3 v0 = bvh.vertex(t, 0);
		V3 planeNormal = cross(bvh.vertex(t, 1) - v0, bvh.vertex(t, 2) - v0);
		return dot(planeNormal, d) <= 0.0f ? float(t + 1) : -float(t + 1);
	}

	__device__ __forceinline__ bool sameHistorySurface(int i, V3 p, V3 n) const
	{
		float4 rp4 = __ldg(historyReceiver + i);
		float4 rn4 = __ldg(historyNormal + i);
		V3 receiverPosition = v3(rp4.x, rp4.y, rp4.z);
		V3 receiverNormal = v3(rn4.x, rn4.y, rn4.z);
		V3 offset = receiverPosition - p;
		return !(dot(receiverNormal, receiverNormal) < 0.5f
			|| dot(offset, offset) > kBounceRadius() * kBounceRadius()
			|| fabsf(dot(offset, n)) > kReceiverPlane()
			|| dot(normalize(receiverNormal), n) < 0.9f);
	}

	__device__ __forceinline__ V3 previousIndirect(V3 p, V3 n, V3 albedo) const
	{
		if (P.history_valid < 0.5f || P.multiple_bounces < 0.5f)
		{
			return v3s(0.0f);
		}
		V4 clip = mul(P.prev_view_proj, v4(p, 1.0f));
		if (clip.w <= 0.0001f)
		{
			return v3s(0.0f);
		}
		V2 uv = clipToUv(P, clip);
		if (!isOnScreen(uv))
		{
			return v3s(0.0f);
		}
		int i = gi(uv);
		if (!sameHistorySurface(i, p, n))
		{
			return v3s(0.0f);
		}
		return loadH4(historyColor, i).xyz() * albedo;
	}

	__device__ __forceinline__ bool historyIrradiance(V2 uv, V3 p, V3 n, V3& irradiance) const
	{
		irradiance = v3s(0.0f);
		if (!isOnScreen(uv))
		{
			return false;
		}
		int i = gi(uv);
		if (!sameHistorySurface(i, p, n))
		{
			return false;
		}
		irradiance = loadH4(historyColor, i).xyz();
		return true;
	}

	__device__ __forceinline__ float depthBehindSurface(V3 rayPosition, V2& uv, V3& surfacePosition, bool& onScreen) const
	{
		float rayDepth;
		surfacePosition = v3s(0.0f);
		onScreen = projectToScreen(rayPosition, uv, rayDepth);
		if (!onScreen)
		{
			return -1.0f;
		}
		int i = full(uv);
		float depth = loadF1(depthTex, i);
		if (depth >= kSkyDepth)
		{
			return -1.0f;
		}
		surfacePosition = reconstructWorldPosition(P, uv, depth);
		float behind = rayDepth - mulW(P.view_proj, surfacePosition);
		if (behind > 0.0f)
		{
			V3 surfaceNormal = decodeNormal(normalTex, i);
			if (dot(rayPosition - surfacePosition, surfaceNormal) > -kSurfaceBias())
			{
				return -1.0f;
			}
		}
		return behind;
	}

	__device__ inline bool traceScreenSpaceRay(V3 origin, V3 direction, float maxDistance, V3& hitPosition) const
	{
		uint32_t steps = 0;
		bool hit = marchDepthBuffer(origin, direction, maxDistance, hitPosition, steps);
		countWork(RESTIR_COUNT_SCREEN, steps, 0u);
		return hit;
	}

	// traceScreenSpaceRay (restir.sh:364-436); steps counts the depth fetches.
	__device__ inline bool marchDepthBuffer(V3 origin, V3 direction, float maxDistance, V3& hitPosition, uint32_t& steps) const
	{
		hitPosition = v3s(0.0f);
		float previousDistance = 0.0f;
		bool previousInFront = true;
		int traceSteps = P.trace_steps;
		float stepScale = 32.0f / float(traceSteps);
		for (int stepIndex = 1; stepIndex <= traceSteps; ++stepIndex)
		{
			if (previousDistance >= maxDistance)
			{
				break;
			}
			float stepPosition = float(stepIndex) * stepScale;
			float rayDistance = fminf((0.02f + stepPosition * stepPosition * 0.0035f) * s(), maxDistance);
			V2 uv;
			V3 surfacePosition;
			bool onScreen;
			++steps;
			float behind = depthBehindSurface(origin + direction * rayDistance, uv, surfacePosition, onScreen);
			if (!onScreen)
			{
				return false;
			}
			bool inFront = behind <= 0.0f;
			if (!inFront && previousInFront)
			{
				float nearDistance = previousDistance;
				float farDistance = rayDistance;
				for (int refineIndex = 0; refineIndex < 5; ++refineIndex)
				{
					float middle = 0.5f * (nearDistance + farDistance);
					V2 middleUv;
					V3 middleSurface;
					bool middleOnScreen;
					++steps;
					float middleBehind = depthBehindSurface(origin + direction * middle, middleUv, middleSurface, middleOnScreen);
					if (middleOnScreen && middleBehind > 0.0f)
					{
						farDistance = middle;
						behind = middleBehind;
						surfacePosition = middleSurface;
					}
					else
					{
						nearDistance = middle;
					}
				}
				float thickness = 0.03f * s() + 0.03f * farDistance;
				if (behind < thickness)
				{
					hitPosition = surfacePosition;
					return true;
				}
			}
			previousInFront = inFront;
			previousDistance = rayDistance;
		}
		return false;
	}

	// The surface a (non-sky) sample lies on, as evaluateSample shades it
	// (restir.sh:466-495): the visible surface from the G-buffer when the
	// sample projects onto it, else its triangle from the BVH. False when
	// neither holds.
	__device__ inline bool sampleSurface(V3 samplePosition, float sampleId, bool& visibleSurface, V2& sampleUv,
		int& triangleIndex, V3& sampleNormal) const
	{
		visibleSurface = false;
		float sampleViewDepth;
		if (projectToScreen(samplePosition, sampleUv, sampleViewDepth))
		{
			float sampleDepth = depthAt(sampleUv);
			visibleSurface = sampleDepth < kSkyDepth
				&& distance(reconstructWorldPosition(P, sampleUv, sampleDepth), samplePosition) <= kSampleTolerance();
		}
		triangleIndex = int(fabsf(sampleId) + 0.5f) - 1;
		if (!visibleSurface && (triangleIndex < 0 || !bvh.available()))
		{
			return false;
		}
		if (visibleSurface)
		{
			sampleNormal = decode(sampleUv);
		}
		else
		{
			V3 v0 = bvh.vertex(triangleIndex, 0);
			sampleNormal = normalize(cross(bvh.vertex(triangleIndex, 1) - v0, bvh.vertex(triangleIndex, 2) - v0))
				* (sampleId < 0.0f ? -1.0f : 1.0f);
		}
		return true;
	}

	// Indirect light leaving the sample point: the radiance cache's value when
	// one is given, else previousIndirect.
	__device__ __forceinline__ V3 sampleIndirect(V3 p, V3 n, V3 albedo, int cacheSlot) const
	{
		if (cache != nullptr && cacheSlot >= 0)
		{
			V4 cached = loadH4(cache, cacheSlot);
			return cached.w > 0.5f ? cached.xyz() * albedo : v3s(0.0f);
		}
		return previousIndirect(p, n, albedo);
	}

	__device__ inline bool evaluateSample(V3 receiverPosition, V3 receiverNormal, V3 receiverAlbedo, V3 samplePosition,
		float sampleId, V3& contribution, V3& sampleNormal, int cacheSlot = -1) const
	{
		contribution = v3s(0.0f);
		sampleNormal = v3(0.0f, 0.0f, 1.0f);
		if (isSkySample(sampleId))
		{
			sampleNormal = -samplePosition;
			contribution = receiverAlbedo * skyRadiance(P, samplePosition)
				* (fmaxf(dot(receiverNormal, samplePosition), 0.0f) / kPi);
			return skyEnabled(P);
		}
		bool visibleSurface;
		V2 sampleUv;
		int triangleIndex;
		if (!sampleSurface(samplePosition, sampleId, visibleSurface, sampleUv, triangleIndex, sampleNormal))
		{
			return false;
		}
		V3 toReceiver = receiverPosition - samplePosition;
		float distanceSquared = dot(toReceiver, toReceiver);
		if (distanceSquared < kMinDistanceSquared() * 0.01f)
		{
			return true;
		}
		V3 directionToReceiver = toReceiver * inversesqrt(distanceSquared);
		float sampleCosine = dot(sampleNormal, directionToReceiver);
		float receiverCosine = -dot(receiverNormal, directionToReceiver);
		if (sampleCosine <= 0.0f || receiverCosine <= 0.0f)
		{
			return true;
		}
		// The sample point's albedo and its own light (the surface light of a
		// visible point, a triangle's emission otherwise), then one call site
		// each for the light terms, which keeps the kernels that inline this small.
		V3 albedo;
		V3 ownLight;
		if (visibleSurface)
		{
			albedo = diffuseAlbedo(sampleUv);
			ownLight = loadH4(surfaceLight, full(sampleUv)).xyz() * P.surface_light_scale;
		}
		else
		{
			albedo = bvh.albedo(triangleIndex);
			ownLight = bvh.emission(triangleIndex) * P.emission_scale;
		}
		const V3 radiance = directFromLight(albedo, samplePosition, sampleNormal)
			+ sampleIndirect(samplePosition, sampleNormal, albedo, cacheSlot) + ownLight;
		contribution = receiverAlbedo * radiance * (receiverCosine / kPi);
		return true;
	}

	__device__ __forceinline__ float geometryTerm(V3 receiverPosition, V3 receiverNormal, V3 samplePosition, V3 sampleNormal,
		float sampleId) const
	{
		if (isSkySample(sampleId))
		{
			return fmaxf(dot(receiverNormal, samplePosition), 0.0f);
		}
		V3 offset = samplePosition - receiverPosition;
		float distanceSquared = dot(offset, offset);
		if (distanceSquared < kMinDistanceSquared() * 0.01f)
		{
			return 0.0f;
		}
		V3 direction = offset * inversesqrt(distanceSquared);
		float receiverCosine = dot(receiverNormal, direction);
		float sampleCosine = -dot(sampleNormal, direction);
		return receiverCosine > 0.0f && sampleCosine > 0.0f ? receiverCosine * sampleCosine / distanceSquared : 0.0f;
	}

	__device__ inline bool isVisible(V3 receiverPosition, V3 receiverNormal, V3 samplePosition, float sampleId) const
	{
		V3 origin = receiverPosition + receiverNormal * kRayBias();
		bool sky = isSkySample(sampleId);
		V3 toSample = sky ? samplePosition * kMaxBvhRayDistance() : samplePosition - origin;
		float sampleDistance = length(toSample);
		V3 direction = toSample / fmaxf(sampleDistance, 0.0001f);
		// One traversal call site for both ray kinds (a sky sample without a BVH
		// is not visible), which keeps the kernels that inline this small.
		const bool bvhRay = sky ? bvh.available() : P.ray_mode == RESTIR_RAY_MODE_BVH && bvh.available();
		if (bvhRay)
		{
			float occluderDistance = 0.0f;
			return traceVisibility(bvh, origin, direction, sky ? kMaxBvhRayDistance() : sampleDistance - kRayBias(),
				occluderDistance, P.wave_visibility > 0.5f) < 0;
		}
		if (sky)
		{
			return false;
		}
		V3 occluderPosition;
		return !traceScreenSpaceRay(origin, direction, sampleDistance * 0.95f - 0.05f * s(), occluderPosition);
	}

	__device__ __forceinline__ float reconnectionJacobian(V3 here, V3 there, V3 samplePosition, V3 sampleNormal, float sampleId) const
	{
		if (isSkySample(sampleId))
		{
			return 1.0f;
		}
		V3 toHere = here - samplePosition;
		V3 toThere = there - samplePosition;
		float hereSquared = dot(toHere, toHere);
		float thereSquared = dot(toThere, toThere);
		if (hereSquared < kMinDistanceSquared() * 0.01f || thereSquared < kMinDistanceSquared() * 0.01f)
		{
			return 0.0f;
		}
		float cosineHere = dot(sampleNormal, toHere) * inversesqrt(hereSquared);
		float cosineThere = dot(sampleNormal, toThere) * inversesqrt(thereSquared);
		if (cosineThere <= 0.001f)
		{
			return 0.0f;
		}
		float jacobian = fmaxf((cosineHere / cosineThere) * (thereSquared / hereSquared), 0.0f);
		return P.jacobian_clamp > 0.0f ? fminf(jacobian, P.jacobian_clamp) : jacobian;
	}

	__device__ __forceinline__ bool acceptNeighbour(V4 sample, V4 receiver, V4 receiverNormal, V3 p, V3 n, float radius,
		NeighbourReservoir& nb) const
	{
		nb.samplePosition = sample.xyz();
		nb.sampleId = receiverNormal.w;
		nb.receiverPosition = receiver.xyz();
		nb.receiverNormal = v3(0.0f, 0.0f, 1.0f);
		nb.count = fminf(sample.w, 20.0f);
		nb.weight = receiver.w;
		nb.cacheSlot = -1;
		V3 rn = receiverNormal.xyz();
		if (sample.w <= 0.0f || dot(rn, rn) < 0.5f)
		{
			return false;
		}
		nb.receiverNormal = normalize(rn);
		V3 receiverOffset = receiver.xyz() - p;
		return dot(receiverOffset, receiverOffset) <= radius * radius
			&& fabsf(dot(receiverOffset, n)) <= kReceiverPlane()
			&& dot(nb.receiverNormal, n) >= 0.9f;
	}

	__device__ __forceinline__ float reuseRadius(V3 p) const
	{
		return grid.worldSpace ? fmaxf(kReceiverRadius(), 2.0f * grid.cellSize(p)) : kReceiverRadius();
	}

	__device__ __forceinline__ PairwiseMis beginPairwiseMis(V3 p, V3 n, const GiReservoir& canonical, float canonicalCount,
		int taps) const
	{
		PairwiseMis mis;
		mis.combined = emptyReservoir();
		mis.canonicalPosition = canonical.position;
		mis.canonicalNormal = canonical.normal;
		mis.canonicalId = canonical.id;
		mis.pairCanonical = canonicalCount / float(taps > 1 ? taps : 1);
		mis.totalCount = canonicalCount;
		mis.hasCanonical = canonical.target > 0.000001f;
		mis.canonicalGeometry = mis.hasCanonical ? geometryTerm(p, n, canonical.position, canonical.normal, canonical.id) : 0.0f;
		mis.canonicalShare = taps > 0 ? 0.0f : canonicalCount;
		mis.neighbourSelected = false;
		return mis;
	}

	__device__ __forceinline__ static void skipNeighbour(PairwiseMis& mis)
	{
		mis.canonicalShare += mis.pairCanonical;
	}

	// addNeighbour and finishPairwiseMis in parts around their visibility test
	// and sample evaluation, so that a kernel can run all of its reuse's tests
	// and evaluations at one call site each (its code then fits the
	// instruction cache); the arithmetic is the same either way.
	//
	// Neighbour, part 1: the count, and the canonical sample's geometry term
	// at the neighbour; true when that term needs the visibility test from the
	// neighbour's receiver to the canonical sample.
	__device__ __forceinline__ bool neighbourBegin(PairwiseMis& mis, const NeighbourReservoir& nb, float& neighbourGeometry) const
	{
		mis.totalCount += nb.count;
		neighbourGeometry = 0.0f;
		if (!mis.hasCanonical)
		{
			return false;
		}
		neighbourGeometry = geometryTerm(nb.receiverPosition, nb.receiverNormal, mis.canonicalPosition, mis.canonicalNormal,
			mis.canonicalId);
		return neighbourGeometry > 0.0f;
	}

	// Neighbour, part 2: the canonical sample's pairwise share, given the test.
	__device__ __forceinline__ void neighbourShare(PairwiseMis& mis, const NeighbourReservoir& nb, float neighbourGeometry,
		bool occluded) const
	{
		if (mis.hasCanonical)
		{
			if (occluded)
			{
				neighbourGeometry = 0.0f;
			}
			float pairWeight = nb.count + mis.pairCanonical;
			float canonicalDensity = mis.pairCanonical * mis.canonicalGeometry;
			float denominator = nb.count * neighbourGeometry + canonicalDensity;
			mis.canonicalShare += denominator > 0.0f ? pairWeight * canonicalDensity / denominator : pairWeight;
		}
	}

	// Neighbour, part 3: its sample shifted to this pixel, from the sample's
	// evaluation here (evaluated only when nb.weight > 0).
	__device__ __forceinline__ void neighbourShift(PairwiseMis& mis, V3 p, V3 n, const NeighbourReservoir& nb, bool shifted,
		V3 contribution, V3 sampleNormal, float random) const
	{
		if (shifted)
		{
			float pairWeight = nb.count + mis.pairCanonical;
			float target = luminance(contribution);
			float jacobian = reconnectionJacobian(p, nb.receiverPosition, nb.samplePosition, sampleNormal, nb.sampleId);
			float hereGeometry = geometryTerm(p, n, nb.samplePosition, sampleNormal, nb.sampleId);
			float thereGeometry = geometryTerm(nb.receiverPosition, nb.receiverNormal, nb.samplePosition, sampleNormal, nb.sampleId);
			float neighbourDensity = nb.count * thereGeometry;
			float denominator = neighbourDensity + mis.pairCanonical * hereGeometry;
			float misWeight = denominator > 0.0f ? pairWeight * neighbourDensity / denominator : 0.0f;
			float weight = misWeight * target * nb.weight * jacobian;
			if (weight > 0.0f
				&& updateReservoir(mis.combined, contribution, nb.samplePosition, sampleNormal, nb.sampleId, target, weight, random))
			{
				mis.neighbourSelected = true;
			}
		}
	}

	__device__ inline void addNeighbour(PairwiseMis& mis, V3 p, V3 n, V3 albedo, const NeighbourReservoir& nb, float random) const
	{
		float neighbourGeometry;
		bool occluded = false;
		if (neighbourBegin(mis, nb, neighbourGeometry))
		{
			occluded = !isVisible(nb.receiverPosition, nb.receiverNormal, mis.canonicalPosition, mis.canonicalId);
		}
		neighbourShare(mis, nb, neighbourGeometry, occluded);
		V3 contribution = v3s(0.0f);
		V3 sampleNormal = v3(0.0f, 0.0f, 1.0f);
		bool shifted = false;
		if (nb.weight > 0.0f)
		{
			shifted = evaluateSample(p, n, albedo, nb.samplePosition, nb.sampleId, contribution, sampleNormal, nb.cacheSlot);
		}
		neighbourShift(mis, p, n, nb, shifted, contribution, sampleNormal, random);
	}

	// The combination, part 1: the canonical sample's update and the combined
	// weight; true when a chosen neighbour's sample needs the visibility test
	// from this pixel (part 2: a failed test zeroes the weight).
	__device__ __forceinline__ bool finishBegin(PairwiseMis& mis, const GiReservoir& canonical, float canonicalWeight, float random,
		float& combinedWeight) const
	{
		if (mis.hasCanonical)
		{
			float weight = mis.canonicalShare * canonical.target * canonicalWeight;
			if (updateReservoir(mis.combined, canonical.contribution, canonical.position, canonical.normal, canonical.id,
				canonical.target, weight, random))
			{
				mis.neighbourSelected = false;
			}
		}
		combinedWeight = mis.combined.target > 0.000001f
			? mis.combined.weightSum / (mis.totalCount * mis.combined.target)
			: 0.0f;
		return combinedWeight > 0.0f && mis.neighbourSelected;
	}

	__device__ inline float finishPairwiseMis(PairwiseMis& mis, V3 p, V3 n, const GiReservoir& canonical, float canonicalWeight,
		float random) const
	{
		float combinedWeight;
		if (finishBegin(mis, canonical, canonicalWeight, random, combinedWeight))
		{
			if (!isVisible(p, n, mis.combined.position, mis.combined.id))
			{
				combinedWeight = 0.0f;
			}
		}
		return combinedWeight;
	}
};

} // namespace restir
