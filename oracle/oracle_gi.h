/*
 * ORACLE (test infrastructure, never linked into the product).
 *
 * shaders/restir.sh (lines 117-931), shaders/shadow.sh (31-108) and
 * shaders/sky.sh (lines 15-31: skyEnabled,
 * skyRadiance), restated on the CPU for one GI pass. The member functions
 * keep the shader's names, argument order and order of operations.
 */
#ifndef ORACLE_GI_H
#define ORACLE_GI_H

#include "oracle_common.h"

namespace oracle
{

/* shadow.sh: the point light's cube shadow atlas. */
struct Shadow
{
	const RestirParams* P = nullptr;
	TexF1 atlas;
	mat4 viewProj[6];

	void init(const RestirParams* _p, const float* _atlas)
	{
		P = _p;
		atlas.p = _atlas;
		atlas.w = int(3 * _p->shadow_face_size);
		atlas.h = int(2 * _p->shadow_face_size);
		for (int f = 0; f < 6; ++f)
		{
			viewProj[f] = make_mat4(_p->shadow_view_proj[f]);
		}
	}

	vec3 lightPosition() const { return vec3(P->light_position[0], P->light_position[1], P->light_position[2]); }

	static int face(vec3 _direction)
	{
		vec3 absolute = abs(_direction);
		if (absolute.x >= absolute.y && absolute.x >= absolute.z)
		{
			return _direction.x >= 0.0f ? 0 : 1;
		}
		if (absolute.y >= absolute.z)
		{
			return _direction.y >= 0.0f ? 2 : 3;
		}
		return _direction.z >= 0.0f ? 4 : 5;
	}

	vec2 atlasUv(vec3 _position, int _face) const
	{
		vec4 clip = mul(viewProj[_face], vec4(_position, 1.0f));
		vec2 ndc = clip.xy() / clip.w;
		bool originBottomLeft = P->origin_bottom_left > 0.5f;
		vec2 local(ndc.x * 0.5f + 0.5f, originBottomLeft ? ndc.y * 0.5f + 0.5f : 0.5f - ndc.y * 0.5f);
		float row = _face >= 3 ? 1.0f : 0.0f;
		float column = float(_face) - 3.0f * row;
		if (originBottomLeft)
		{
			row = 1.0f - row;
		}
		return (vec2(column, row) + local) * vec2(1.0f / 3.0f, 0.5f);
	}

	bool lookup(vec3 _position, vec3 _normal, float _filterRadius, vec2& _uv, float& _reference) const
	{
		_uv = vec2_splat(0.0f);
		_reference = 0.0f;
		if (P->shadows_enabled < 0.5f)
		{
			return false;
		}
		float lightDistance = length(lightPosition() - _position);
		float texelSize = 2.0f * lightDistance * P->shadow_tan_half_fov * P->shadow_inv_face_size;
		vec3 position = _position + _normal * (texelSize * 1.5f);
		vec3 fromLight = position - lightPosition();
		_uv = atlasUv(position, face(fromLight));
		float cosine = clamp(dot(_normal, -normalize(fromLight)), 0.0f, 1.0f);
		float slope = min(sqrt(1.0f - cosine * cosine) / max(cosine, 0.0001f), 8.0f);
		float bias = texelSize * (1.0f + _filterRadius * slope);
		_reference = (length(fromLight) - bias) / P->shadow_far;
		return true;
	}

	float visibilityHard(vec3 _position, vec3 _normal) const
	{
		vec2 uv;
		float reference;
		if (!lookup(_position, _normal, 0.5f, uv, reference))
		{
			return 1.0f;
		}
		return reference <= atlas.sample(uv) ? 1.0f : 0.0f;
	}

	float visibilitySoft(vec3 _position, vec3 _normal) const
	{
		vec2 uv;
		float reference;
		if (!lookup(_position, _normal, 2.0f, uv, reference))
		{
			return 1.0f;
		}
		vec2 atlasTexel(P->shadow_inv_face_size / 3.0f, P->shadow_inv_face_size * 0.5f);
		float lit = 0.0f;
		for (int y = 0; y < 4; ++y)
		{
			for (int x = 0; x < 4; ++x)
			{
				vec2 offset = vec2(float(x) - 1.5f, float(y) - 1.5f) * atlasTexel;
				lit += reference <= atlas.sample(uv + offset) ? 1.0f : 0.0f;
			}
		}
		return lit / 16.0f;
	}
};

/* sky.sh */
struct Sky
{
	vec4 zenith, horizon, ground;

	void init(const RestirParams* _p)
	{
		zenith = vec4(_p->sky_zenith[0], _p->sky_zenith[1], _p->sky_zenith[2], _p->sky_zenith[3]);
		horizon = vec4(_p->sky_horizon[0], _p->sky_horizon[1], _p->sky_horizon[2], _p->sky_horizon[3]);
		ground = vec4(_p->sky_ground[0], _p->sky_ground[1], _p->sky_ground[2], _p->sky_ground[3]);
	}

	bool enabled() const { return zenith.w > 0.5f; }

	vec3 radiance(vec3 _direction) const
	{
		if (!enabled())
		{
			return vec3_splat(0.0f);
		}
		float height = clamp(_direction.y, -1.0f, 1.0f);
		return height >= 0.0f
			? mix(horizon.xyz(), zenith.xyz(), sqrt(height))
			: mix(horizon.xyz(), ground.xyz(), sqrt(-height));
	}
};

/* Screen conventions shared by the passes (restir.sh:150-199, di.sh:71-76). */
struct Screen
{
	mat4 viewProj, invViewProj, prevViewProj;
	bool originBottomLeft = false;

	void init(const RestirParams* _p)
	{
		viewProj = make_mat4(_p->view_proj);
		invViewProj = make_mat4(_p->inv_view_proj);
		prevViewProj = make_mat4(_p->prev_view_proj);
		originBottomLeft = _p->origin_bottom_left > 0.5f;
	}

	/* bgfx shaderlib's toClipSpaceY / clipToWorld, with NDC depth in [0, 1]. */
	float toClipSpaceY(float _y) const { return originBottomLeft ? _y : -_y; }

	vec3 reconstructWorldPosition(vec2 _uv, float _depth) const
	{
		vec3 clipPosition = vec3(_uv.x * 2.0f - 1.0f, _uv.y * 2.0f - 1.0f, _depth);
		clipPosition.y = toClipSpaceY(clipPosition.y);
		vec4 world = mul(invViewProj, vec4(clipPosition, 1.0f));
		return world.xyz() / world.w;
	}

	vec2 clipToUv(vec4 _clip) const
	{
		float originSign = originBottomLeft ? 1.0f : -1.0f;
		return vec2(_clip.x, _clip.y * originSign) / _clip.w * 0.5f + 0.5f;
	}
};

inline bool isOnScreen(vec2 _uv)
{
	return _uv.x > 0.001f && _uv.x < 0.999f && _uv.y > 0.001f && _uv.y < 0.999f;
}

#define kSkySampleId 30000000.0f
inline bool isSkySample(float _sampleId) { return _sampleId > kSkySampleId * 0.5f; }

struct Reservoir
{
	vec3 contribution;
	vec3 position;
	vec3 normal = vec3(0.0f, 0.0f, 1.0f);
	float id = 0.0f;
	float target = 0.0f;
	float weightSum = 0.0f;
	float count = 0.0f;
};

inline bool updateReservoir(Reservoir& _r, vec3 _contribution, vec3 _position, vec3 _normal, float _id,
	float _target, float _weight, float _random)
{
	_r.weightSum += _weight;
	if (_random * _r.weightSum < _weight)
	{
		_r.contribution = _contribution;
		_r.position = _position;
		_r.normal = _normal;
		_r.id = _id;
		_r.target = _target;
		return true;
	}
	return false;
}

struct NeighbourReservoir
{
	vec3 samplePosition;
	float sampleId = 0.0f;
	vec3 receiverPosition;
	vec3 receiverNormal;
	float count = 0.0f;
	float weight = 0.0f;
	int cacheSlot = -1;  // the radiance cache's value for this sample, or -1
};

struct PairwiseMis
{
	Reservoir combined;
	vec3 canonicalPosition;
	vec3 canonicalNormal;
	float canonicalId = 0.0f;
	float pairCanonical = 0.0f;
	float canonicalGeometry = 0.0f;
	float canonicalShare = 0.0f;
	float totalCount = 0.0f;
	bool hasCanonical = false;
	bool neighbourSelected = false;
};

/* One GI pass: its bound resources and restir.sh's functions. */
struct GiPass
{
	const RestirParams* P = nullptr;
	Screen screen;
	Shadow shadow;
	Sky sky;
	Bvh bvh;
	Grid grid;
	bool sharedStack = false; // BVH_SHARED_STACK: the temporal pass

	TexU8 albedoTex, normalTex;
	TexF1 depthTex;
	TexH4 historyColor, surfaceLight;
	TexF4 historyNormal, historyReceiver;
	vec2 giSize, giTexel;
	// The radiance cache's values (half4 per slot), when the pass takes the
	// indirect light at sample points from it (restir_cache.h): an input here,
	// like a texture. Reused neighbours sit at cacheNeighbourBase + pixel.
	const uint16_t* cache = nullptr;
	int cacheNeighbourBase = 0;

	float s() const { return P->scene_scale; }
	float kRayBias() const { return 0.02f * s(); }
	float kSurfaceBias() const { return 0.01f * s(); }
	float kMaxRayDistance() const { return 3.6f * s(); }
	float kMaxBvhRayDistance() const { return 4.0f * s(); }
	float kSampleTolerance() const { return 0.1f * s(); }
	float kReceiverRadius() const { return 0.4f * s(); }
	float kReceiverPlane() const { return 0.03f * s(); }
	float kMinDistanceSquared() const { return 0.0001f * s() * s(); }
	float kBounceRadius() const { return 0.1f * s(); }
	vec3 lightPosition() const { return shadow.lightPosition(); }
	vec3 lightColor() const { return vec3(P->light_color[0], P->light_color[1], P->light_color[2]); }

	vec3 diffuseAlbedo(vec2 _uv) const
	{
		vec3 albedo = albedoTex.sample(_uv).xyz();
		float metallic = normalTex.sample(_uv).w;
		return albedo * (1.0f - metallic);
	}

	vec3 decodeNormal(vec2 _uv) const
	{
		return normalize(normalTex.sample(_uv).xyz() * 2.0f - 1.0f);
	}

	vec3 reconstructWorldPosition(vec2 _uv, float _depth) const { return screen.reconstructWorldPosition(_uv, _depth); }

	vec2 giPixel(vec2 _uv) const { return floor(_uv * giSize); }
	uint giPixelIndex(vec2 _pixel) const { return uint(_pixel.y) * uint(giSize.x) + uint(_pixel.x); }
	vec2 giPixelUv(uint _index) const
	{
		uint width = uint(giSize.x);
		return (vec2(float(_index % width), float(_index / width)) + 0.5f) * giTexel;
	}

	bool projectToScreen(vec3 _position, vec2& _uv, float& _viewDepth) const
	{
		vec4 clip = mul(screen.viewProj, vec4(_position, 1.0f));
		_viewDepth = clip.w;
		_uv = vec2_splat(0.0f);
		if (clip.w <= 0.0001f)
		{
			return false;
		}
		_uv = screen.clipToUv(clip);
		return isOnScreen(_uv);
	}

	static vec3 cosineHemisphere(vec3 _normal, float _random0, float _random1)
	{
		float radius = sqrt(_random0);
		float angle = 2.0f * kPi * _random1;
		vec3 localDirection = vec3(radius * cos(angle), radius * sin(angle), sqrt(max(1.0f - _random0, 0.0f)));
		vec3 tangent = normalize(abs(_normal.y) < 0.99f
			? cross(_normal, vec3(0.0f, 1.0f, 0.0f))
			: cross(_normal, vec3(1.0f, 0.0f, 0.0f)));
		vec3 bitangent = cross(_normal, tangent);
		return normalize(tangent * localDirection.x + bitangent * localDirection.y + _normal * localDirection.z);
	}

	vec3 evaluateSecondaryDirect(vec2 _uv, vec3 _position, vec3 _normal) const
	{
		vec3 albedo = diffuseAlbedo(_uv);
		vec3 toLight = lightPosition() - _position;
		float distanceSquared = max(dot(toLight, toLight), 0.01f * s() * s());
		float normalLight = max(dot(_normal, toLight * inversesqrt(distanceSquared)), 0.0f);
		vec3 direct = vec3_splat(0.0f);
		if (normalLight > 0.0f)
		{
			direct = albedo * (lightColor() / distanceSquared) * (normalLight / kPi)
				* shadow.visibilityHard(_position, _normal);
		}
		return direct;
	}

	vec3 evaluateWorldDirect(vec3 _albedo, vec3 _position, vec3 _normal) const
	{
		vec3 toLight = lightPosition() - _position;
		float distanceSquared = max(dot(toLight, toLight), 0.01f * s() * s());
		float normalLight = max(dot(_normal, toLight * inversesqrt(distanceSquared)), 0.0f);
		vec3 direct = vec3_splat(0.0f);
		if (normalLight > 0.0f)
		{
			direct = _albedo * (lightColor() / distanceSquared) * (normalLight / kPi)
				* shadow.visibilityHard(_position, _normal);
		}
		return direct;
	}

	float encodeSampleId(int _triangle, vec3 _rayDirection) const
	{
		vec3 v0 = bvh.vertex(_triangle, 0);
		vec3 planeNormal = cross(bvh.vertex(_triangle, 1) - v0, bvh.vertex(_triangle, 2) - v0);
		return dot(planeNormal, _rayDirection) <= 0.0f ? float(_triangle + 1) : -float(_triangle + 1);
	}

	bool sameHistorySurface(vec2 _uv, vec3 _position, vec3 _normal) const
	{
		vec3 receiverPosition = historyReceiver.sample(_uv).xyz();
		vec3 receiverNormal = historyNormal.sample(_uv).xyz();
		vec3 offset = receiverPosition - _position;
		return !(dot(receiverNormal, receiverNormal) < 0.5f
			|| dot(offset, offset) > kBounceRadius() * kBounceRadius()
			|| abs(dot(offset, _normal)) > kReceiverPlane()
			|| dot(normalize(receiverNormal), _normal) < 0.9f);
	}

	vec3 previousIndirect(vec3 _position, vec3 _normal, vec3 _albedo) const
	{
		if (P->history_valid < 0.5f || P->multiple_bounces < 0.5f)
		{
			return vec3_splat(0.0f);
		}
		vec4 clip = mul(screen.prevViewProj, vec4(_position, 1.0f));
		if (clip.w <= 0.0001f)
		{
			return vec3_splat(0.0f);
		}
		vec2 uv = screen.clipToUv(clip);
		if (!isOnScreen(uv))
		{
			return vec3_splat(0.0f);
		}
		if (!sameHistorySurface(uv, _position, _normal))
		{
			return vec3_splat(0.0f);
		}
		return historyColor.sample(uv).xyz() * _albedo;
	}

	bool historyIrradiance(vec2 _uv, vec3 _position, vec3 _normal, vec3& _irradiance) const
	{
		_irradiance = vec3_splat(0.0f);
		if (!isOnScreen(_uv))
		{
			return false;
		}
		if (!sameHistorySurface(_uv, _position, _normal))
		{
			return false;
		}
		_irradiance = historyColor.sample(_uv).xyz();
		return true;
	}

	float depthBehindSurface(vec3 _rayPosition, vec2& _uv, vec3& _surfacePosition, bool& _onScreen) const
	{
		float rayDepth;
		_surfacePosition = vec3_splat(0.0f);
		_onScreen = projectToScreen(_rayPosition, _uv, rayDepth);
		if (!_onScreen)
		{
			return -1.0f;
		}
		float depth = depthTex.sample(_uv);
		if (depth >= kSkyDepth)
		{
			return -1.0f;
		}
		_surfacePosition = reconstructWorldPosition(_uv, depth);
		float behind = rayDepth - mul(screen.viewProj, vec4(_surfacePosition, 1.0f)).w;
		if (behind > 0.0f)
		{
			vec3 surfaceNormal = decodeNormal(_uv);
			if (dot(_rayPosition - _surfacePosition, surfaceNormal) > -kSurfaceBias())
			{
				return -1.0f;
			}
		}
		return behind;
	}

	bool traceScreenSpaceRay(vec3 _origin, vec3 _direction, float _maxDistance, vec3& _hitPosition) const
	{
		_hitPosition = vec3_splat(0.0f);
		float previousDistance = 0.0f;
		bool previousInFront = true;
		int traceSteps = P->trace_steps;
		float stepScale = 32.0f / float(traceSteps);
		for (int stepIndex = 1; stepIndex <= traceSteps; ++stepIndex)
		{
			if (previousDistance >= _maxDistance)
			{
				break;
			}
			float stepPosition = float(stepIndex) * stepScale;
			float rayDistance = min((0.02f + stepPosition * stepPosition * 0.0035f) * s(), _maxDistance);
			vec2 uv;
			vec3 surfacePosition;
			bool onScreen;
			float behind = depthBehindSurface(_origin + _direction * rayDistance, uv, surfacePosition, onScreen);
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
					vec2 middleUv;
					vec3 middleSurface;
					bool middleOnScreen;
					float middleBehind = depthBehindSurface(_origin + _direction * middle, middleUv, middleSurface, middleOnScreen);
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
					_hitPosition = surfacePosition;
					return true;
				}
			}
			previousInFront = inFront;
			previousDistance = rayDistance;
		}
		return false;
	}

	// previousIndirect, or the radiance cache's value for the slot times the
	// albedo (zero for a padding row).
	vec3 sampleIndirect(vec3 _position, vec3 _normal, vec3 _albedo, int _cacheSlot) const
	{
		if (cache != nullptr && _cacheSlot >= 0)
		{
			const uint16_t* c = cache + size_t(_cacheSlot) * 4;
			if (rn_half_to_float(c[3]) > 0.5f)
			{
				return vec3(rn_half_to_float(c[0]), rn_half_to_float(c[1]), rn_half_to_float(c[2])) * _albedo;
			}
			return vec3_splat(0.0f);
		}
		return previousIndirect(_position, _normal, _albedo);
	}

	bool evaluateSample(vec3 _receiverPosition, vec3 _receiverNormal, vec3 _receiverAlbedo, vec3 _samplePosition,
		float _sampleId, vec3& _contribution, vec3& _sampleNormal, int _cacheSlot = -1) const
	{
		_contribution = vec3_splat(0.0f);
		_sampleNormal = vec3(0.0f, 0.0f, 1.0f);
		if (isSkySample(_sampleId))
		{
			_sampleNormal = -_samplePosition;
			_contribution = _receiverAlbedo * sky.radiance(_samplePosition)
				* (max(dot(_receiverNormal, _samplePosition), 0.0f) / kPi);
			return sky.enabled();
		}
		bool visibleSurface = false;
		vec2 sampleUv;
		float sampleViewDepth;
		if (projectToScreen(_samplePosition, sampleUv, sampleViewDepth))
		{
			float sampleDepth = depthTex.sample(sampleUv);
			visibleSurface = sampleDepth < kSkyDepth
				&& distance(reconstructWorldPosition(sampleUv, sampleDepth), _samplePosition) <= kSampleTolerance();
		}
		int triangleIndex = int(abs(_sampleId) + 0.5f) - 1;
		if (!visibleSurface && (triangleIndex < 0 || !bvh.available()))
		{
			return false;
		}
		if (visibleSurface)
		{
			_sampleNormal = decodeNormal(sampleUv);
		}
		else
		{
			vec3 v0 = bvh.vertex(triangleIndex, 0);
			_sampleNormal = normalize(cross(bvh.vertex(triangleIndex, 1) - v0, bvh.vertex(triangleIndex, 2) - v0))
				* (_sampleId < 0.0f ? -1.0f : 1.0f);
		}
		vec3 toReceiver = _receiverPosition - _samplePosition;
		float distanceSquared = dot(toReceiver, toReceiver);
		if (distanceSquared < kMinDistanceSquared() * 0.01f)
		{
			return true;
		}
		vec3 directionToReceiver = toReceiver * inversesqrt(distanceSquared);
		float sampleCosine = dot(_sampleNormal, directionToReceiver);
		float receiverCosine = -dot(_receiverNormal, directionToReceiver);
		if (sampleCosine <= 0.0f || receiverCosine <= 0.0f)
		{
			return true;
		}
		vec3 radiance;
		if (visibleSurface)
		{
			radiance = evaluateSecondaryDirect(sampleUv, _samplePosition, _sampleNormal)
				+ sampleIndirect(_samplePosition, _sampleNormal, diffuseAlbedo(sampleUv), _cacheSlot)
				+ surfaceLight.sample(sampleUv).xyz() * P->surface_light_scale;
		}
		else
		{
			radiance = evaluateWorldDirect(bvhTriangleAlbedo(bvh, triangleIndex), _samplePosition, _sampleNormal)
				+ sampleIndirect(_samplePosition, _sampleNormal, bvhTriangleAlbedo(bvh, triangleIndex), _cacheSlot)
				+ bvhTriangleEmission(bvh, triangleIndex) * P->emission_scale;
		}
		_contribution = _receiverAlbedo * radiance * (receiverCosine / kPi);
		return true;
	}

	float geometryTerm(vec3 _receiverPosition, vec3 _receiverNormal, vec3 _samplePosition, vec3 _sampleNormal, float _sampleId) const
	{
		if (isSkySample(_sampleId))
		{
			return max(dot(_receiverNormal, _samplePosition), 0.0f);
		}
		vec3 offset = _samplePosition - _receiverPosition;
		float distanceSquared = dot(offset, offset);
		if (distanceSquared < kMinDistanceSquared() * 0.01f)
		{
			return 0.0f;
		}
		vec3 direction = offset * inversesqrt(distanceSquared);
		float receiverCosine = dot(_receiverNormal, direction);
		float sampleCosine = -dot(_sampleNormal, direction);
		return receiverCosine > 0.0f && sampleCosine > 0.0f
			? receiverCosine * sampleCosine / distanceSquared
			: 0.0f;
	}

	bool isVisible(vec3 _receiverPosition, vec3 _receiverNormal, vec3 _samplePosition, float _sampleId) const
	{
		vec3 origin = _receiverPosition + _receiverNormal * kRayBias();
		bool skySample = isSkySample(_sampleId);
		vec3 toSample = skySample ? _samplePosition * kMaxBvhRayDistance() : _samplePosition - origin;
		float sampleDistance = length(toSample);
		vec3 direction = toSample / max(sampleDistance, 0.0001f);
		bool visible = true;
		if (skySample)
		{
			float occluderDistance = 0.0f;
			visible = false;
			if (bvh.available())
			{
				visible = traceBvh(bvh, origin, direction, kMaxBvhRayDistance(), true, occluderDistance, sharedStack) < 0;
			}
		}
		else if (P->ray_mode == RESTIR_RAY_MODE_BVH && bvh.available())
		{
			float occluderDistance = 0.0f;
			visible = traceBvh(bvh, origin, direction, sampleDistance - kRayBias(), true, occluderDistance, sharedStack) < 0;
		}
		else
		{
			vec3 occluderPosition;
			visible = !traceScreenSpaceRay(origin, direction, sampleDistance * 0.95f - 0.05f * s(), occluderPosition);
		}
		return visible;
	}

	float reconnectionJacobian(vec3 _here, vec3 _there, vec3 _samplePosition, vec3 _sampleNormal, float _sampleId) const
	{
		if (isSkySample(_sampleId))
		{
			return 1.0f;
		}
		vec3 toHere = _here - _samplePosition;
		vec3 toThere = _there - _samplePosition;
		float hereSquared = dot(toHere, toHere);
		float thereSquared = dot(toThere, toThere);
		if (hereSquared < kMinDistanceSquared() * 0.01f || thereSquared < kMinDistanceSquared() * 0.01f)
		{
			return 0.0f;
		}
		float cosineHere = dot(_sampleNormal, toHere) * inversesqrt(hereSquared);
		float cosineThere = dot(_sampleNormal, toThere) * inversesqrt(thereSquared);
		if (cosineThere <= 0.001f)
		{
			return 0.0f;
		}
		float jacobian = max((cosineHere / cosineThere) * (thereSquared / hereSquared), 0.0f);
		return P->jacobian_clamp > 0.0f ? min(jacobian, P->jacobian_clamp) : jacobian;
	}

	bool acceptNeighbour(vec4 _sample, vec4 _receiver, vec4 _receiverNormal, vec3 _position, vec3 _normal,
		float _radius, NeighbourReservoir& _neighbour) const
	{
		_neighbour.samplePosition = _sample.xyz();
		_neighbour.sampleId = _receiverNormal.w;
		_neighbour.receiverPosition = _receiver.xyz();
		_neighbour.receiverNormal = vec3(0.0f, 0.0f, 1.0f);
		_neighbour.count = min(_sample.w, 20.0f);
		_neighbour.weight = _receiver.w;
		if (_sample.w <= 0.0f || dot(_receiverNormal.xyz(), _receiverNormal.xyz()) < 0.5f)
		{
			return false;
		}
		_neighbour.receiverNormal = normalize(_receiverNormal.xyz());
		vec3 receiverOffset = _receiver.xyz() - _position;
		return dot(receiverOffset, receiverOffset) <= _radius * _radius
			&& abs(dot(receiverOffset, _normal)) <= kReceiverPlane()
			&& dot(_neighbour.receiverNormal, _normal) >= 0.9f;
	}

	float reuseRadius(vec3 _position) const
	{
		return grid.worldSpace
			? max(kReceiverRadius(), 2.0f * grid.cellSize(_position))
			: kReceiverRadius();
	}

	PairwiseMis beginPairwiseMis(vec3 _position, vec3 _normal, const Reservoir& _canonical, float _canonicalCount, int _taps) const
	{
		PairwiseMis mis;
		mis.canonicalPosition = _canonical.position;
		mis.canonicalNormal = _canonical.normal;
		mis.canonicalId = _canonical.id;
		mis.pairCanonical = _canonicalCount / float(max(_taps, 1));
		mis.totalCount = _canonicalCount;
		mis.hasCanonical = _canonical.target > 0.000001f;
		mis.canonicalGeometry = mis.hasCanonical
			? geometryTerm(_position, _normal, _canonical.position, _canonical.normal, _canonical.id)
			: 0.0f;
		mis.canonicalShare = _taps > 0 ? 0.0f : _canonicalCount;
		mis.neighbourSelected = false;
		return mis;
	}

	static void skipNeighbour(PairwiseMis& _mis)
	{
		_mis.canonicalShare += _mis.pairCanonical;
	}

	void addNeighbour(PairwiseMis& _mis, vec3 _position, vec3 _normal, vec3 _albedo, const NeighbourReservoir& _neighbour, float _random) const
	{
		float neighbourCount = _neighbour.count;
		float pairWeight = neighbourCount + _mis.pairCanonical;
		_mis.totalCount += neighbourCount;
		if (_mis.hasCanonical)
		{
			float neighbourGeometry = geometryTerm(_neighbour.receiverPosition, _neighbour.receiverNormal,
				_mis.canonicalPosition, _mis.canonicalNormal, _mis.canonicalId);
			if (neighbourGeometry > 0.0f)
			{
				if (!isVisible(_neighbour.receiverPosition, _neighbour.receiverNormal, _mis.canonicalPosition, _mis.canonicalId))
				{
					neighbourGeometry = 0.0f;
				}
			}
			float canonicalDensity = _mis.pairCanonical * _mis.canonicalGeometry;
			float denominator = neighbourCount * neighbourGeometry + canonicalDensity;
			_mis.canonicalShare += denominator > 0.0f
				? pairWeight * canonicalDensity / denominator
				: pairWeight;
		}
		vec3 contribution = vec3_splat(0.0f);
		vec3 sampleNormal = vec3(0.0f, 0.0f, 1.0f);
		bool shifted = false;
		if (_neighbour.weight > 0.0f)
		{
			shifted = evaluateSample(_position, _normal, _albedo, _neighbour.samplePosition, _neighbour.sampleId,
				contribution, sampleNormal, _neighbour.cacheSlot);
		}
		if (shifted)
		{
			float target = luminance(contribution);
			float jacobian = reconnectionJacobian(_position, _neighbour.receiverPosition, _neighbour.samplePosition,
				sampleNormal, _neighbour.sampleId);
			float hereGeometry = geometryTerm(_position, _normal, _neighbour.samplePosition, sampleNormal, _neighbour.sampleId);
			float thereGeometry = geometryTerm(_neighbour.receiverPosition, _neighbour.receiverNormal,
				_neighbour.samplePosition, sampleNormal, _neighbour.sampleId);
			float neighbourDensity = neighbourCount * thereGeometry;
			float denominator = neighbourDensity + _mis.pairCanonical * hereGeometry;
			float misWeight = denominator > 0.0f ? pairWeight * neighbourDensity / denominator : 0.0f;
			float weight = misWeight * target * _neighbour.weight * jacobian;
			if (weight > 0.0f
				&& updateReservoir(_mis.combined, contribution, _neighbour.samplePosition, sampleNormal,
					_neighbour.sampleId, target, weight, _random))
			{
				_mis.neighbourSelected = true;
			}
		}
	}

	float finishPairwiseMis(PairwiseMis& _mis, vec3 _position, vec3 _normal, const Reservoir& _canonical,
		float _canonicalWeight, float _random) const
	{
		if (_mis.hasCanonical)
		{
			float weight = _mis.canonicalShare * _canonical.target * _canonicalWeight;
			if (updateReservoir(_mis.combined, _canonical.contribution, _canonical.position, _canonical.normal,
				_canonical.id, _canonical.target, weight, _random))
			{
				_mis.neighbourSelected = false;
			}
		}
		float combinedWeight = _mis.combined.target > 0.000001f
			? _mis.combined.weightSum / (_mis.totalCount * _mis.combined.target)
			: 0.0f;
		if (combinedWeight > 0.0f && _mis.neighbourSelected)
		{
			if (!isVisible(_position, _normal, _mis.combined.position, _mis.combined.id))
			{
				combinedWeight = 0.0f;
			}
		}
		return combinedWeight;
	}
};

} // namespace oracle

#endif // ORACLE_GI_H
