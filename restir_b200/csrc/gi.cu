// ReSTIR GI passes: restir_gi_temporal (cs_restir_temporal.sc:57-297) and
// restir_gi_spatial (cs_restir_spatial.sc:49-246).
//
// The temporal pass runs one warp per 4x8 pixel group of the reference
// (compute.sh:31-35): the boiling filter's tile mean is a warp-shuffle tree
// in the order of the shader's shared-memory reduction (compute.sh:375-386),
// and closest-hit candidate rays keep their short traversal stack in shared
// memory, interleaved across the block's lanes.
#include "gi.cuh"
#include "wavefront.cuh"

#include "../../include/restir_cache.h"

namespace restir
{
namespace
{

constexpr int kGiWarps = 4;
constexpr int kGiThreads = 32 * kGiWarps;

// Minimum resident blocks per SM (register budget) of the two GI kernels.
// Measured on the 1080p frame (launch-bound sweep): the spatial pass gains
// from 8 blocks (64 registers, a little spilling to L1); the temporal pass is
// bound by divergence and instruction fetch more than occupancy: its
// wavefront form took 3.00 ms at its natural 150 registers (3 blocks) and
// 2.91 ms at 6 blocks (80 registers); once its code was made smaller the
// shading kernel takes 1.11 / 1.06 / 1.02 ms at 6 / 7 / 8 blocks (8: 64
// registers, a few hundred bytes spilled to L1).
#ifndef RESTIR_GI_TEMPORAL_MIN_BLOCKS
#	define RESTIR_GI_TEMPORAL_MIN_BLOCKS 8
#endif
#ifndef RESTIR_GI_SPATIAL_MIN_BLOCKS
#	define RESTIR_GI_SPATIAL_MIN_BLOCKS 8
#endif

struct GiBindings
{
	const uint8_t* albedo;
	const uint8_t* normal;
	const float* depth;
	const float4* historySample;
	const float4* historyReceiver;
	const float4* historyNormal;
	const uint16_t* historyColor;
	const uint16_t* historyMoments;
	const uint16_t* surfaceLight;
	const float* shadowAtlas;
	const uint32_t* grid;
	const float4* reservoirSample;   // spatial: this frame's reservoirs
	const float4* reservoirReceiver;
	const float4* reservoirNormal;
	float4* outSample;               // temporal outputs
	float4* outReceiver;
	float4* outNormal;
	uint16_t* outColor;              // spatial outputs
	uint16_t* outMoments;
	const uint16_t* cache;           // radiance-cache values (half4), or null
	int cacheNeighbourBase;          // slot of reused neighbour 0
};

__device__ __forceinline__ GiPass makePass(const RestirParams& P, const BvhView& bvh, const GiBindings& b, const float* gridCamera,
	int* stack, int stride)
{
	GiPass g{ P };
	g.bvh = bvh;
	g.grid = makeGridView(&P, b.grid, gridCamera);
	g.albedoTex = b.albedo;
	g.normalTex = b.normal;
	g.depthTex = b.depth;
	g.historyNormal = b.historyNormal;
	g.historyReceiver = b.historyReceiver;
	g.historyColor = b.historyColor;
	g.surfaceLight = b.surfaceLight;
	g.shadowAtlas = b.shadowAtlas;
	g.stack = stack;
	g.stackStride = stride;
	g.W = int(P.width);
	g.H = int(P.height);
	g.w = int(P.gi_width);
	g.h = int(P.gi_height);
	g.giSize = v2(float(g.w), float(g.h));
	g.giTexel = v2(1.0f / float(g.w), 1.0f / float(g.h));
	g.cache = b.cache;
	g.cacheNeighbourBase = b.cacheNeighbourBase;
	return g;
}

__device__ __forceinline__ V4 f4(float4 q)
{
	return { q.x, q.y, q.z, q.w };
}

// The largest reservoir weight the GI passes with the radiance cache store
// (about 30x the median weight on the 1080p city view; 0.05% of the stored
// weights are above it there).
constexpr float kCachedReservoirWeightCap = 64.0f;

// The end of the temporal pass: the boiling filter against the group's mean
// estimate (summed as compute.sh's shared-memory tree), then the reservoir's
// store. Every lane of the warp calls it.
__device__ __forceinline__ void boilAndStore(const RestirParams& P, const GiPass& g, const GiBindings& b, int lane, bool inside,
	bool working, int px, int py, V3 position, V3 normal, V3 albedo, const GiReservoir& canonical, float canonicalWeight,
	V2 previousUv, const PairwiseMis& mis, float combinedWeight)
{
	const bool historyValid = P.history_valid > 0.5f;
	const float estimate = working ? mis.combined.target * combinedWeight : 0.0f;
	float sumEstimate = estimate;
	float sumWorking = working ? 1.0f : 0.0f;
	for (int stride = 16; stride > 0; stride >>= 1)
	{
		float e = __shfl_down_sync(0xffffffffu, sumEstimate, stride);
		float c = __shfl_down_sync(0xffffffffu, sumWorking, stride);
		if (lane < stride)
		{
			sumEstimate += e;
			sumWorking += c;
		}
	}
	sumEstimate = __shfl_sync(0xffffffffu, sumEstimate, 0);
	sumWorking = __shfl_sync(0xffffffffu, sumWorking, 0);
	const float tileMean = sumEstimate / fmaxf(sumWorking, 1.0f);
	if (working && P.boiling_filter > 0.0f && combinedWeight > 0.0f)
	{
		float reference = canonical.target * canonicalWeight;
		V3 historyColor;
		if (historyValid && g.historyIrradiance(previousUv, position, normal, historyColor))
		{
			reference = fmaxf(reference, luminance(historyColor * albedo));
		}
		else
		{
			reference = fmaxf(reference, tileMean);
		}
		float limit = P.boiling_filter * reference;
		if (estimate > limit)
		{
			combinedWeight *= limit / estimate;
		}
	}
	if (g.cache != nullptr)
	{
		// With the radiance cache every sample point carries indirect light, and
		// a reservoir's weight can ratchet up through temporal reuse from
		// receiver to receiver until the pixel's estimate sits at the outlier
		// clamp (a growing bright patch in some runs after 100-300 frames). The
		// stored weight is capped in this form only; the plain path keeps the
		// reference's arithmetic.
		combinedWeight = fminf(combinedWeight, kCachedReservoirWeightCap);
	}
	if (inside)
	{
		const int i = py * g.w + px;
		b.outSample[i] = working ? make_float4(mis.combined.position.x, mis.combined.position.y, mis.combined.position.z,
			mis.totalCount) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		b.outReceiver[i] = working ? make_float4(position.x, position.y, position.z, combinedWeight)
			: make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		b.outNormal[i] = working ? make_float4(normal.x, normal.y, normal.z, mis.combined.id) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	}
}

// cs_restir_temporal.sc:192-296 after the fresh candidates: temporal reuse
// with pairwise MIS, the boiling filter over the warp's 4x8 group, the
// reservoir stores. Every lane of the warp must call it (the group sum).
__device__ __forceinline__ void temporalReuseAndStore(const RestirParams& P, const GiPass& g, const GiBindings& b, int lane,
	bool inside, bool working, int px, int py, V3 position, V3 normal, V3 albedo, const GiReservoir& canonical, uint32_t rng)
{
	const float canonicalWeight = canonical.target > 0.000001f ? canonical.weightSum / (canonical.count * canonical.target) : 0.0f;
	const bool historyValid = P.history_valid > 0.5f;
	V2 previousUv = v2(0.0f, 0.0f);
	const V4 clipPrevious = mul(P.prev_view_proj, v4(position, 1.0f));
	if (clipPrevious.w > 0.0001f)
	{
		previousUv = clipToUv(P, clipPrevious);
	}
	const float radius = g.reuseRadius(position);
	PairwiseMis mis = g.beginPairwiseMis(position, normal, canonical, canonical.count, P.temporal_taps);
	float combinedWeight = 0.0f;
	if (working)
	{
		for (int tapIndex = 0; tapIndex < P.temporal_taps; ++tapIndex)
		{
			float random0 = nextRandom(rng);
			float random1 = nextRandom(rng);
			float random2 = nextRandom(rng);
			float randomSelect = nextRandom(rng);
			V2 historyUv = v2(-1.0f, -1.0f);
			if (historyValid)
			{
				if (g.grid.worldSpace)
				{
					uint32_t entry = gridPickEntry(g.grid, position, normal, random0, random1, random2);
					if (entry != kGridInvalid)
					{
						historyUv = g.giPixelUv(entry);
					}
				}
				else if (tapIndex == 0 && clipPrevious.w > 0.0001f)
				{
					historyUv = previousUv;
				}
			}
			NeighbourReservoir neighbour;
			bool accepted = false;
			if (isOnScreen(historyUv))
			{
				int i = g.gi(historyUv);
				accepted = g.acceptNeighbour(f4(__ldg(b.historySample + i)), f4(__ldg(b.historyReceiver + i)),
					f4(__ldg(b.historyNormal + i)), position, normal, radius, neighbour);
				neighbour.cacheSlot = g.cache != nullptr ? g.cacheNeighbourBase + i : -1;
			}
			if (!accepted)
			{
				GiPass::skipNeighbour(mis);
				continue;
			}
			g.addNeighbour(mis, position, normal, albedo, neighbour, randomSelect);
		}
		combinedWeight = g.finishPairwiseMis(mis, position, normal, canonical, canonicalWeight, nextRandom(rng));
	}
	boilAndStore(P, g, b, lane, inside, working, px, py, position, normal, albedo, canonical, canonicalWeight, previousUv, mis,
		combinedWeight);
}

__global__ void __launch_bounds__(kGiThreads, RESTIR_GI_TEMPORAL_MIN_BLOCKS) giTemporalKernel(const RestirParams P, BvhView bvh,
	GiBindings b)
{
	__shared__ int stackStorage[kBvhShortStack * kGiThreads];
	const int lane = int(threadIdx.x & 31u);
	const int groupsX = (int(P.gi_width) + 3) / 4;
	const int groupsY = (int(P.gi_height) + 7) / 8;
	const int group = int(blockIdx.x) * kGiWarps + int(threadIdx.x >> 5);
	if (group >= groupsX * groupsY)
	{
		return; // whole warp
	}
	GiPass g = makePass(P, bvh, b, P.prev_camera_position, stackStorage + threadIdx.x, kGiThreads);
	const int px = (group % groupsX) * 4 + (lane & 3);
	const int py = (group / groupsX) * 8 + (lane >> 2);
	const bool inside = px < g.w && py < g.h;
	const V2 uv = pixelUv(px, py, g.giTexel);
	const float depth = inside ? g.depthAt(uv) : 1.0f;
	const bool working = inside && depth < kSkyDepth;

	const V3 position = reconstructWorldPosition(P, uv, depth);
	const V3 normal = g.decode(uv);
	const V3 albedo = g.diffuseAlbedo(uv);
	const V3 rayOrigin = position + normal * g.kRayBias();
	const V2 giPixelCoord = v2(floorf(uv.x * g.giSize.x), floorf(uv.y * g.giSize.y));
	uint32_t rng = pcg(uint32_t(giPixelCoord.x) + pcg(uint32_t(giPixelCoord.y) + pcg(uint32_t(P.frame_index))));

	GiReservoir canonical = emptyReservoir();
	for (int sampleIndex = 0; sampleIndex < P.initial_candidates; ++sampleIndex)
	{
		float random0 = nextRandom(rng);
		float random1 = nextRandom(rng);
		float randomSelect = nextRandom(rng);
		V3 direction = GiPass::cosineHemisphere(normal, random0, random1);
		canonical.count += 1.0f;
		V3 hitPosition = v3s(0.0f);
		float hitId = 0.0f;
		bool hit = false;
		if (working && P.ray_mode != RESTIR_RAY_MODE_BVH)
		{
			hit = g.traceScreenSpaceRay(rayOrigin, direction, g.kMaxRayDistance(), hitPosition);
		}
		bool needBvh = working && !hit && P.ray_mode != RESTIR_RAY_MODE_SCREEN;
		if (needBvh)
		{
			float queueDistance;
			int queueTriangle = traceBvh(g.bvh, rayOrigin, direction, g.kMaxBvhRayDistance(), false, queueDistance,
				g.stack, g.stackStride);
			if (queueTriangle >= 0)
			{
				hit = true;
				hitPosition = rayOrigin + direction * queueDistance;
				hitId = g.encodeSampleId(queueTriangle, direction);
			}
			else if (skyEnabled(P))
			{
				hit = true;
				hitPosition = direction;
				hitId = kSkySampleId;
			}
		}
		V3 contribution = v3s(0.0f);
		V3 hitNormal = v3s(0.0f);
		bool evaluated = false;
		if (hit)
		{
			evaluated = g.evaluateSample(position, normal, albedo, hitPosition, hitId, contribution, hitNormal);
		}
		if (evaluated)
		{
			float target = luminance(contribution);
			float sourcePdf = dot(normal, direction) / kPi;
			if (!isSkySample(hitId))
			{
				V3 fromReceiver = hitPosition - position;
				V3 fromOrigin = hitPosition - rayOrigin;
				float receiverSquared = fmaxf(dot(fromReceiver, fromReceiver), g.kMinDistanceSquared() * 0.01f);
				float originSquared = fmaxf(dot(fromOrigin, fromOrigin), g.kMinDistanceSquared() * 0.01f);
				float hitCosineOrigin = fmaxf(-dot(hitNormal, fromOrigin), 0.0f) * inversesqrt(originSquared);
				float hitCosineReceiver = -dot(hitNormal, fromReceiver) * inversesqrt(receiverSquared);
				sourcePdf = hitCosineReceiver > 0.0001f
					? sourcePdf * (hitCosineOrigin / originSquared) * (receiverSquared / hitCosineReceiver)
					: 0.0f;
			}
			if (target > 0.0f && sourcePdf > 0.0001f)
			{
				updateReservoir(canonical, contribution, hitPosition, hitNormal, hitId, target, target / sourcePdf, randomSelect);
			}
		}
	}

	temporalReuseAndStore(P, g, b, lane, inside, working, px, py, position, normal, albedo, canonical, rng);
}

__global__ void __launch_bounds__(128, RESTIR_GI_SPATIAL_MIN_BLOCKS) giSpatialKernel(const RestirParams P, BvhView bvh, GiBindings b)
{
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	if (px >= g.w || py >= g.h)
	{
		return;
	}
	const int outIndex = py * g.w + px;
	const V2 uv = pixelUv(px, py, g.giTexel);
	const float depth = g.depthAt(uv);
	if (depth >= kSkyDepth)
	{
		storeH4(b.outColor, outIndex, v4(0.0f, 0.0f, 0.0f, 0.0f));
		storeH4(b.outMoments, outIndex, v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	const V3 position = reconstructWorldPosition(P, uv, depth);
	const V3 normal = g.decode(uv);
	const V3 albedo = g.diffuseAlbedo(uv);
	const V2 pixel = v2(floorf(uv.x * g.giSize.x), floorf(uv.y * g.giSize.y));
	const uint32_t pixelIndex = uint32_t(pixel.y) * uint32_t(g.giSize.x) + uint32_t(pixel.x);
	uint32_t rng = pcg(uint32_t(pixel.x) + pcg(uint32_t(pixel.y) + pcg(uint32_t(P.frame_index) ^ 0x68e31da4u)));

	const int own = g.gi(uv);
	const V4 ownSample = f4(b.reservoirSample[own]);
	const float canonicalWeight = b.reservoirReceiver[own].w;
	const float ownId = b.reservoirNormal[own].w;
	const float canonicalCount = fmaxf(fminf(ownSample.w, 20.0f), 1.0f);
	GiReservoir canonical = emptyReservoir();
	V3 canonicalContribution = v3s(0.0f);
	V3 canonicalNormal = v3(0.0f, 0.0f, 1.0f);
	bool canonicalValid = false;
	if (canonicalWeight > 0.0f)
	{
		canonicalValid = g.evaluateSample(position, normal, albedo, ownSample.xyz(), ownId, canonicalContribution, canonicalNormal,
			g.cache != nullptr ? g.cacheNeighbourBase + own : -1);
	}
	if (canonicalValid)
	{
		canonical.contribution = canonicalContribution;
		canonical.position = ownSample.xyz();
		canonical.normal = canonicalNormal;
		canonical.id = ownId;
		canonical.target = luminance(canonicalContribution);
	}

	const float radius = g.reuseRadius(position);
	PairwiseMis mis = g.beginPairwiseMis(position, normal, canonical, canonicalCount, P.spatial_taps);
	for (int tapIndex = 0; tapIndex < P.spatial_taps; ++tapIndex)
	{
		float random0 = nextRandom(rng);
		float random1 = nextRandom(rng);
		float random2 = nextRandom(rng);
		float randomSelect = nextRandom(rng);
		V2 neighbourUv = v2(-1.0f, -1.0f);
		if (g.grid.worldSpace)
		{
			uint32_t entry = gridPickEntry(g.grid, position, normal, random0, random1, random2);
			if (entry != kGridInvalid && entry != pixelIndex)
			{
				neighbourUv = g.giPixelUv(entry);
			}
		}
		else
		{
			float diskRadius = 12.0f * sqrtf(random0);
			float angle = 2.0f * kPi * random1;
			float sn, cs;
			rn_sincos(angle, &sn, &cs);
			V2 neighbourPixel = v2(floorf(pixel.x + cs * diskRadius), floorf(pixel.y + sn * diskRadius));
			if (neighbourPixel.x != pixel.x || neighbourPixel.y != pixel.y)
			{
				neighbourUv = v2((neighbourPixel.x + 0.5f) * g.giTexel.x, (neighbourPixel.y + 0.5f) * g.giTexel.y);
			}
		}
		NeighbourReservoir neighbour;
		bool accepted = false;
		if (isOnScreen(neighbourUv))
		{
			int i = g.gi(neighbourUv);
			accepted = g.acceptNeighbour(f4(b.reservoirSample[i]), f4(b.reservoirReceiver[i]), f4(b.reservoirNormal[i]),
				position, normal, radius, neighbour);
			neighbour.cacheSlot = g.cache != nullptr ? g.cacheNeighbourBase + i : -1;
		}
		if (!accepted)
		{
			GiPass::skipNeighbour(mis);
			continue;
		}
		g.addNeighbour(mis, position, normal, albedo, neighbour, randomSelect);
	}

	const float combinedWeight = g.finishPairwiseMis(mis, position, normal, canonical, canonicalWeight, nextRandom(rng));
	V3 estimate = mis.combined.contribution * combinedWeight;
	if (P.outlier_clamp > 0.0f)
	{
		estimate = vmin(estimate, v3s(P.outlier_clamp));
	}
	const V3 irradiance = estimate / vmax(albedo, v3s(0.001f));
	const float irradianceLuminance = luminance(irradiance);

	V3 previousColor = v3s(0.0f);
	V3 previousMoments = v3s(0.0f);
	const V4 clipPrevious = mul(P.prev_view_proj, v4(position, 1.0f));
	if (P.history_valid > 0.5f && clipPrevious.w > 0.0001f)
	{
		// reprojectHistory (cs_restir_spatial.sc:49-93)
		const V2 previousUv = clipToUv(P, clipPrevious);
		V3 c = v3s(0.0f);
		V3 m = v3s(0.0f);
		const V2 texelCoord = v2(previousUv.x * g.giSize.x - 0.5f, previousUv.y * g.giSize.y - 0.5f);
		const V2 baseCoord = v2(floorf(texelCoord.x), floorf(texelCoord.y));
		const V2 blend = texelCoord - baseCoord;
		float weightSum = 0.0f;
		for (int tapIndex = 0; tapIndex < 4; ++tapIndex)
		{
			const V2 offset = v2(float(tapIndex & 1), float(tapIndex >> 1));
			const V2 tapUv = v2((baseCoord.x + offset.x + 0.5f) * g.giTexel.x, (baseCoord.y + offset.y + 0.5f) * g.giTexel.y);
			if (!isOnScreen(tapUv))
			{
				continue;
			}
			const int i = g.gi(tapUv);
			if (!g.sameHistorySurface(i, position, normal))
			{
				continue;
			}
			const V2 bilinear = v2(mixf(1.0f - blend.x, blend.x, offset.x), mixf(1.0f - blend.y, blend.y, offset.y));
			const float weight = bilinear.x * bilinear.y;
			c = c + loadH4(b.historyColor, i).xyz() * weight;
			m = m + loadH4(b.historyMoments, i).xyz() * weight;
			weightSum += weight;
		}
		if (weightSum < 0.01f)
		{
			c = v3s(0.0f);
			m = v3s(0.0f);
		}
		else
		{
			c = c / weightSum;
			m = m / weightSum;
		}
		previousColor = c;
		previousMoments = m;
	}
	const float historyLength = fminf(previousMoments.z + 1.0f, 16.0f);
	const float blendWeight = 1.0f / historyLength;
	const V3 color = mix(previousColor, irradiance, blendWeight);
	const float m0 = mixf(previousMoments.x, irradianceLuminance, blendWeight);
	const float m1 = mixf(previousMoments.y, irradianceLuminance * irradianceLuminance, blendWeight);
	storeH4(b.outColor, outIndex, v4(color, historyLength));
	storeH4(b.outMoments, outIndex, v4(m0, m1, historyLength, 0.0f));
}

// --- the temporal pass as a wavefront -----------------------------------------
//
// A: candidate directions and depth-buffer marches; the rays the march cannot
//    answer go to a ray queue (warp-vote compaction).
// B: the persistent closest-hit tracer over the queue (wavefront.cuh).
// C: the rest of cs_restir_temporal.sc, reading A's and B's results where
//    the megakernel traced; the random stream is replayed from the pixel's
//    seed, so every number is the megakernel's.

struct CandidateRecords
{
	float4* screenHit;  // per pixel and candidate: (hit position, 1 if the march hit)
	int* slot;          // per pixel and candidate: queue slot, or -1
	int candidates;
};

// Minimum resident blocks per SM of the GI candidates kernel: 0.347 ms at its
// natural 83 registers (5 blocks), 0.329 / 0.313 ms at 6 / 8 blocks (8: 64
// registers) on the 1080p frame; its depth-buffer marches are latency-bound.
#ifndef RESTIR_GI_CANDIDATES_MIN_BLOCKS
#	define RESTIR_GI_CANDIDATES_MIN_BLOCKS 8
#endif

__global__ void __launch_bounds__(kGiThreads, RESTIR_GI_CANDIDATES_MIN_BLOCKS) giCandidatesKernel(const RestirParams P, BvhView bvh, GiBindings b,
	CandidateRecords records, RayQueue queue)
{
	const int lane = int(threadIdx.x & 31u);
	const int groupsX = (int(P.gi_width) + 3) / 4;
	const int groupsY = (int(P.gi_height) + 7) / 8;
	const int group = int(blockIdx.x) * kGiWarps + int(threadIdx.x >> 5);
	if (group >= groupsX * groupsY)
	{
		return; // whole warp
	}
	GiPass g = makePass(P, bvh, b, P.prev_camera_position, nullptr, 0);
	const int px = (group % groupsX) * 4 + (lane & 3);
	const int py = (group / groupsX) * 8 + (lane >> 2);
	const bool inside = px < g.w && py < g.h;
	const V2 uv = pixelUv(px, py, g.giTexel);
	const float depth = inside ? g.depthAt(uv) : 1.0f;
	const bool working = inside && depth < kSkyDepth;
	const V3 position = reconstructWorldPosition(P, uv, depth);
	const V3 normal = g.decode(uv);
	const V3 rayOrigin = position + normal * g.kRayBias();
	const V2 giPixelCoord = v2(floorf(uv.x * g.giSize.x), floorf(uv.y * g.giSize.y));
	uint32_t rng = pcg(uint32_t(giPixelCoord.x) + pcg(uint32_t(giPixelCoord.y) + pcg(uint32_t(P.frame_index))));
	const int pixel = py * g.w + px;
	for (int sampleIndex = 0; sampleIndex < P.initial_candidates; ++sampleIndex)
	{
		float random0 = nextRandom(rng);
		float random1 = nextRandom(rng);
		nextRandom(rng); // randomSelect, used by pass C
		V3 direction = GiPass::cosineHemisphere(normal, random0, random1);
		V3 hitPosition = v3s(0.0f);
		bool hit = false;
		if (working && P.ray_mode != RESTIR_RAY_MODE_BVH)
		{
			hit = g.traceScreenSpaceRay(rayOrigin, direction, g.kMaxRayDistance(), hitPosition);
		}
		const bool needBvh = working && !hit && P.ray_mode != RESTIR_RAY_MODE_SCREEN && bvh.available();
		const int slot = queuePush(queue, needBvh, rayOrigin, g.kMaxBvhRayDistance(), direction);
		if (inside)
		{
			const int r = pixel * records.candidates + sampleIndex;
			records.screenHit[r] = make_float4(hitPosition.x, hitPosition.y, hitPosition.z, hit ? 1.0f : 0.0f);
			records.slot[r] = needBvh ? slot : -2 - int(working && !hit && P.ray_mode != RESTIR_RAY_MODE_SCREEN);
		}
	}
}

__global__ void __launch_bounds__(128) traceQueueKernel(BvhView bvh, RayQueue queue)
{
	__shared__ int stackStorage[kBvhShortStack * 128];
	traceQueueClosest<128>(bvh, queue, stackStorage);
}

// The queue tracer at other block sizes (restir_trace_queue's tuning knob).
template<int kThreads>
__global__ void __launch_bounds__(kThreads) traceQueueSizedKernel(BvhView bvh, RayQueue queue)
{
	__shared__ int stackStorage[kBvhShortStack * kThreads];
	traceQueueClosest<kThreads>(bvh, queue, stackStorage);
}

__global__ void __launch_bounds__(kGiThreads, RESTIR_GI_TEMPORAL_MIN_BLOCKS) giTemporalShadeKernel(const RestirParams P,
	BvhView bvh, GiBindings b, CandidateRecords records, RayQueue queue)
{
	const int lane = int(threadIdx.x & 31u);
	const int groupsX = (int(P.gi_width) + 3) / 4;
	const int groupsY = (int(P.gi_height) + 7) / 8;
	const int group = int(blockIdx.x) * kGiWarps + int(threadIdx.x >> 5);
	if (group >= groupsX * groupsY)
	{
		return; // whole warp
	}
	GiPass g = makePass(P, bvh, b, P.prev_camera_position, nullptr, 0);
	const int px = (group % groupsX) * 4 + (lane & 3);
	const int py = (group / groupsX) * 8 + (lane >> 2);
	const bool inside = px < g.w && py < g.h;
	const V2 uv = pixelUv(px, py, g.giTexel);
	const float depth = inside ? g.depthAt(uv) : 1.0f;
	const bool working = inside && depth < kSkyDepth;
	const V3 position = reconstructWorldPosition(P, uv, depth);
	const V3 normal = g.decode(uv);
	const V3 albedo = g.diffuseAlbedo(uv);
	const V3 rayOrigin = position + normal * g.kRayBias();
	const V2 giPixelCoord = v2(floorf(uv.x * g.giSize.x), floorf(uv.y * g.giSize.y));
	uint32_t rng = pcg(uint32_t(giPixelCoord.x) + pcg(uint32_t(giPixelCoord.y) + pcg(uint32_t(P.frame_index))));
	const int pixel = py * g.w + px;

	// The candidates, the temporal reuse (temporalReuseAndStore) and the
	// combination as one loop with one call site each for the sample
	// evaluation and the visibility test (the kernel is bound by instruction
	// fetch): steps 0..C-1 shade the candidates, steps C..C+T-1 take the
	// temporal neighbours and step C+T combines, the last two for working
	// pixels only. The random draws and every operation are the
	// straight-line form's, in its order.
	const int candidates = P.initial_candidates;
	const int taps = P.temporal_taps;
	const int last = working ? candidates + taps : candidates - 1;
	const bool historyValid = P.history_valid > 0.5f;
	V2 previousUv = v2(0.0f, 0.0f);
	const V4 clipPrevious = mul(P.prev_view_proj, v4(position, 1.0f));
	if (clipPrevious.w > 0.0001f)
	{
		previousUv = clipToUv(P, clipPrevious);
	}
	const float radius = g.reuseRadius(position);
	GiReservoir canonical = emptyReservoir();
	float canonicalWeight = 0.0f;
	PairwiseMis mis;
	float combinedWeight = 0.0f;
	bool misStarted = false;
#pragma unroll 1
	for (int step = 0; step <= last; ++step)
	{
		if (step >= candidates && !misStarted)
		{
			canonicalWeight = canonical.target > 0.000001f ? canonical.weightSum / (canonical.count * canonical.target) : 0.0f;
			mis = g.beginPairwiseMis(position, normal, canonical, canonical.count, taps);
			misStarted = true;
		}
		// What this step evaluates and tests.
		bool evaluate = false;
		V3 samplePosition = v3s(0.0f);
		float sampleId = 0.0f;
		int cacheSlot = -1;
		V3 direction = v3s(0.0f);
		float randomSelect = 0.0f;
		NeighbourReservoir neighbour;
		float neighbourGeometry = 0.0f;
		bool test = false;
		V3 from = position, fromNormal = normal, to = v3s(0.0f);
		float toId = 0.0f;
		if (step < candidates)
		{
			const int sampleIndex = step;
			float random0 = nextRandom(rng);
			float random1 = nextRandom(rng);
			randomSelect = nextRandom(rng);
			direction = GiPass::cosineHemisphere(normal, random0, random1);
			canonical.count += 1.0f;
			bool hit = false;
			if (inside)
			{
				const int r = pixel * records.candidates + sampleIndex;
				const float4 screen = records.screenHit[r];
				hit = screen.w > 0.5f;
				samplePosition = v3(screen.x, screen.y, screen.z);
				const int slot = records.slot[r];
				// -3: the BVH was wanted but there is none (traceBvh returns -1 at once).
				if (slot >= 0 || slot == -3)
				{
					int triangle = -1;
					float t = 0.0f;
					if (slot >= 0)
					{
						triangle = queue.hitTriangle[slot];
						t = queue.hitDistance[slot];
					}
					if (triangle >= 0)
					{
						hit = true;
						samplePosition = rayOrigin + direction * t;
						sampleId = g.encodeSampleId(triangle, direction);
					}
					else if (skyEnabled(P))
					{
						hit = true;
						samplePosition = direction;
						sampleId = kSkySampleId;
					}
				}
			}
			evaluate = hit;
			cacheSlot = g.cache != nullptr ? pixel * records.candidates + sampleIndex : -1;
		}
		else if (step < candidates + taps)
		{
			const int tapIndex = step - candidates;
			float random0 = nextRandom(rng);
			float random1 = nextRandom(rng);
			float random2 = nextRandom(rng);
			randomSelect = nextRandom(rng);
			V2 historyUv = v2(-1.0f, -1.0f);
			if (historyValid)
			{
				if (g.grid.worldSpace)
				{
					uint32_t entry = gridPickEntry(g.grid, position, normal, random0, random1, random2);
					if (entry != kGridInvalid)
					{
						historyUv = g.giPixelUv(entry);
					}
				}
				else if (tapIndex == 0 && clipPrevious.w > 0.0001f)
				{
					historyUv = previousUv;
				}
			}
			bool accepted = false;
			if (isOnScreen(historyUv))
			{
				int i = g.gi(historyUv);
				accepted = g.acceptNeighbour(f4(__ldg(b.historySample + i)), f4(__ldg(b.historyReceiver + i)),
					f4(__ldg(b.historyNormal + i)), position, normal, radius, neighbour);
				neighbour.cacheSlot = g.cache != nullptr ? g.cacheNeighbourBase + i : -1;
			}
			if (!accepted)
			{
				GiPass::skipNeighbour(mis);
				continue;
			}
			test = g.neighbourBegin(mis, neighbour, neighbourGeometry);
			from = neighbour.receiverPosition;
			fromNormal = neighbour.receiverNormal;
			to = mis.canonicalPosition;
			toId = mis.canonicalId;
		}
		else
		{
			test = g.finishBegin(mis, canonical, canonicalWeight, nextRandom(rng), combinedWeight);
			to = mis.combined.position;
			toId = mis.combined.id;
		}
		const bool occluded = test && !g.isVisible(from, fromNormal, to, toId);
		if (step == candidates + taps)
		{
			if (occluded)
			{
				combinedWeight = 0.0f;
			}
			break;
		}
		if (step >= candidates)
		{
			g.neighbourShare(mis, neighbour, neighbourGeometry, occluded);
			evaluate = neighbour.weight > 0.0f;
			samplePosition = neighbour.samplePosition;
			sampleId = neighbour.sampleId;
			cacheSlot = neighbour.cacheSlot;
		}
		V3 contribution = v3s(0.0f);
		V3 sampleNormal = step < candidates ? v3s(0.0f) : v3(0.0f, 0.0f, 1.0f);
		bool valid = false;
		if (evaluate)
		{
			valid = g.evaluateSample(position, normal, albedo, samplePosition, sampleId, contribution, sampleNormal, cacheSlot);
		}
		if (step >= candidates)
		{
			g.neighbourShift(mis, position, normal, neighbour, valid, contribution, sampleNormal, randomSelect);
		}
		else if (valid)
		{
			// The candidate's source density and its update (cs_restir_temporal.sc).
			const V3 hitPosition = samplePosition;
			const V3 hitNormal = sampleNormal;
			float target = luminance(contribution);
			float sourcePdf = dot(normal, direction) / kPi;
			if (!isSkySample(sampleId))
			{
				V3 fromReceiver = hitPosition - position;
				V3 fromOrigin = hitPosition - rayOrigin;
				float receiverSquared = fmaxf(dot(fromReceiver, fromReceiver), g.kMinDistanceSquared() * 0.01f);
				float originSquared = fmaxf(dot(fromOrigin, fromOrigin), g.kMinDistanceSquared() * 0.01f);
				float hitCosineOrigin = fmaxf(-dot(hitNormal, fromOrigin), 0.0f) * inversesqrt(originSquared);
				float hitCosineReceiver = -dot(hitNormal, fromReceiver) * inversesqrt(receiverSquared);
				sourcePdf = hitCosineReceiver > 0.0001f
					? sourcePdf * (hitCosineOrigin / originSquared) * (receiverSquared / hitCosineReceiver)
					: 0.0f;
			}
			if (target > 0.0f && sourcePdf > 0.0001f)
			{
				updateReservoir(canonical, contribution, hitPosition, hitNormal, sampleId, target, target / sourcePdf, randomSelect);
			}
		}
	}
	if (!misStarted)
	{
		canonicalWeight = canonical.target > 0.000001f ? canonical.weightSum / (canonical.count * canonical.target) : 0.0f;
		mis = g.beginPairwiseMis(position, normal, canonical, canonical.count, taps);
	}
	boilAndStore(P, g, b, lane, inside, working, px, py, position, normal, albedo, canonical, canonicalWeight, previousUv, mis,
		combinedWeight);
}

// --- indirect specular (fs_specular.sc) --------------------------------------------------

// fs_specular.sc:41-47
__device__ __forceinline__ void tangentFrame(V3 n, V3& tangent, V3& bitangent)
{
	tangent = normalize(fabsf(n.y) < 0.99f ? cross(n, v3(0.0f, 1.0f, 0.0f)) : cross(n, v3(1.0f, 0.0f, 0.0f)));
	bitangent = cross(n, tangent);
}

// GGX visible normals (Heitz 2018), fs_specular.sc:51-67.
__device__ __forceinline__ V3 sampleVisibleNormal(V3 view, float alpha, float random0, float random1)
{
	const V3 stretched = normalize(v3(alpha * view.x, alpha * view.y, view.z));
	const float lengthSquared = stretched.x * stretched.x + stretched.y * stretched.y;
	const V3 t1 = lengthSquared > 0.0f ? v3(-stretched.y, stretched.x, 0.0f) * inversesqrt(lengthSquared) : v3(1.0f, 0.0f, 0.0f);
	const V3 t2 = cross(stretched, t1);
	const float radius = sqrtf(random0);
	const float angle = 2.0f * kPi * random1;
	float sn, cs;
	rn_sincos(angle, &sn, &cs);
	const float p1 = radius * cs;
	float p2 = radius * sn;
	const float s = 0.5f * (1.0f + stretched.z);
	p2 = (1.0f - s) * sqrtf(fmaxf(1.0f - p1 * p1, 0.0f)) + s * p2;
	const V3 normal = t1 * p1 + t2 * p2 + stretched * sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f));
	return normalize(v3(alpha * normal.x, alpha * normal.y, fmaxf(normal.z, 0.0f)));
}

// fs_specular.sc:70-74
__device__ __forceinline__ float smithG1(float cosine, float alpha)
{
	const float alphaSquared = alpha * alpha;
	return 2.0f * cosine / (cosine + sqrtf(alphaSquared + (1.0f - alphaSquared) * cosine * cosine));
}

// brdf.sh:29-37
__device__ __forceinline__ V3 fresnelSchlick(V3 halfway, V3 view, V3 f0)
{
	const float cosine = clampf(dot(halfway, view), 0.0f, 1.0f);
	return f0 + (v3s(1.0f) - f0) * rn_pow5(1.0f - cosine);
}

// The split-sum specular albedo, brdf.sh:68-76 (Karis' analytic fit).
__device__ __forceinline__ V3 specularAlbedo(V3 f0, float roughness, float normalView)
{
	const float rx = -1.0f * roughness + 1.0f, ry = -0.0275f * roughness + 0.0425f;
	const float rz = -0.572f * roughness + 1.04f, rw = 0.022f * roughness + -0.04f;
	const float a004 = fminf(rx * rx, rn_exp2(-9.28f * normalView)) * rx + ry;
	const float scale = -1.04f * a004 + rz, bias = 1.04f * a004 + rw;
	return f0 * scale + bias;
}

// Radiance leaving a ray's hit point back along the ray, fs_specular.sc:77-125.
__device__ inline V3 specularHitRadiance(const GiPass& g, const uint16_t* __restrict__ previousHdr, V3 hitPosition,
	float hitId, V3 rayDirection)
{
	const RestirParams& P = g.P;
	if (isSkySample(hitId))
	{
		return skyRadiance(P, rayDirection);
	}
	V2 uv;
	float viewDepth;
	bool visibleSurface = false;
	if (g.projectToScreen(hitPosition, uv, viewDepth))
	{
		const float depth = g.depthAt(uv);
		visibleSurface = depth < kSkyDepth && distance(reconstructWorldPosition(P, uv, depth), hitPosition) <= g.kSampleTolerance();
	}
	if (visibleSurface)
	{
		const V4 clip = mul(P.prev_view_proj, v4(hitPosition, 1.0f));
		if (P.history_valid > 0.5f && clip.w > 0.0001f)
		{
			const V2 previousUv = clipToUv(P, clip);
			const V4 previous = loadH4(previousHdr, g.full(previousUv));
			if (isOnScreen(previousUv) && previous.w > 0.5f)
			{
				return previous.xyz();
			}
		}
		const V3 normal = g.decode(uv);
		return g.directFromLight(g.diffuseAlbedo(uv), hitPosition, normal) + g.previousIndirect(hitPosition, normal, g.diffuseAlbedo(uv))
			+ loadH4(g.surfaceLight, g.full(uv)).xyz() * P.surface_light_scale;
	}
	const int triangleIndex = int(fabsf(hitId) + 0.5f) - 1;
	if (triangleIndex < 0 || !g.bvh.available())
	{
		return v3s(0.0f);
	}
	const V3 v0 = g.bvh.vertex(triangleIndex, 0);
	V3 normal = normalize(cross(g.bvh.vertex(triangleIndex, 1) - v0, g.bvh.vertex(triangleIndex, 2) - v0));
	if (dot(normal, -rayDirection) < 0.0f)
	{
		normal = -normal;
	}
	const V3 albedo = g.bvh.albedo(triangleIndex);
	return g.directFromLight(albedo, hitPosition, normal) + g.previousIndirect(hitPosition, normal, albedo)
		+ g.bvh.emission(triangleIndex) * P.emission_scale;
}

// Blocks per SM the specular kernel is compiled for: capped at 64 registers (8
// blocks of 128 threads) it takes 1.84 ms at 1080p (GI 960x540) against 2.10 ms
// at its natural 88 registers (5 blocks); the traversal is latency-bound.
#ifndef RESTIR_SPECULAR_MIN_BLOCKS
#define RESTIR_SPECULAR_MIN_BLOCKS 8
#endif

// The pixel's surface and its reflection ray, fs_specular.sc:127-160.
struct SpecularRay
{
	bool surface;
	V3 position, normal, viewDirection, f0, halfway, direction, origin;
	float roughness, alpha, normalView, normalLight;
};

__device__ __forceinline__ SpecularRay specularRay(const GiPass& g, V2 uv)
{
	const RestirParams& P = g.P;
	SpecularRay r;
	const float depth = g.depthAt(uv);
	r.surface = depth < kSkyDepth;
	if (!r.surface)
	{
		return r;
	}
	r.position = reconstructWorldPosition(P, uv, depth);
	r.normal = g.decode(uv);
	const V4 albedoRoughness = loadU8(g.albedoTex, g.full(uv));
	const float metallic = loadU8(g.normalTex, g.full(uv)).w;
	r.roughness = fmaxf(albedoRoughness.w, 0.02f);
	r.alpha = r.roughness * r.roughness;
	const V3 camera = v3(P.camera_position[0], P.camera_position[1], P.camera_position[2]);
	r.viewDirection = normalize(camera - r.position);
	r.normalView = fmaxf(dot(r.normal, r.viewDirection), 0.001f);
	r.f0 = mix(v3s(0.04f), albedoRoughness.xyz(), metallic);
	const V2 pixel = v2(floorf(uv.x * g.giSize.x), floorf(uv.y * g.giSize.y));
	uint32_t rng = pcg(uint32_t(pixel.x) + pcg(uint32_t(pixel.y) + pcg(uint32_t(P.frame_index) ^ 0x2545f491u)));

	V3 tangent, bitangent;
	tangentFrame(r.normal, tangent, bitangent);
	const V3 localView = v3(dot(r.viewDirection, tangent), dot(r.viewDirection, bitangent), r.normalView);
	const float random0 = nextRandom(rng);
	const float random1 = nextRandom(rng);
	const V3 localHalfway = sampleVisibleNormal(localView, r.alpha, random0, random1);
	r.halfway = tangent * localHalfway.x + bitangent * localHalfway.y + r.normal * localHalfway.z;
	const V3 incident = -r.viewDirection;
	r.direction = incident - r.halfway * (2.0f * dot(r.halfway, incident));
	r.normalLight = dot(r.normal, r.direction);
	r.origin = r.position + r.normal * g.kRayBias();
	return r;
}

// The hit of a BVH ray of the pass: the triangle, or the sky when enabled.
__device__ __forceinline__ bool specularBvhHit(const GiPass& g, const SpecularRay& r, int triangleIndex, float hitDistance,
	V3& hitPosition, float& hitId)
{
	if (triangleIndex >= 0)
	{
		hitPosition = r.origin + r.direction * hitDistance;
		hitId = g.encodeSampleId(triangleIndex, r.direction);
		return true;
	}
	if (skyEnabled(g.P))
	{
		hitId = kSkySampleId;
		return true;
	}
	return false;
}

// fs_specular.sc:160-226 from the ray's hit: radiance, demodulation by the
// split-sum albedo, the outlier clamp and the reprojected history.
__device__ inline void specularFinish(const GiPass& g, const SpecularRay& r, bool hit, V3 hitPosition, float hitId,
	const uint16_t* __restrict__ previousHdr, const uint16_t* __restrict__ specularHistory, uint16_t* out, int i)
{
	const RestirParams& P = g.P;
	V3 estimate = v3s(0.0f);
	if (hit)
	{
		const V3 fresnel = fresnelSchlick(r.halfway, r.viewDirection, r.f0);
		estimate = specularHitRadiance(g, previousHdr, hitPosition, hitId, r.direction) * fresnel * smithG1(r.normalLight, r.alpha);
	}
	V3 demodulated = estimate / vmax(specularAlbedo(r.f0, r.roughness, r.normalView), v3s(0.001f));
	if (P.outlier_clamp > 0.0f)
	{
		demodulated = vmin(demodulated, v3s(P.outlier_clamp));
	}

	V3 history = v3s(0.0f);
	float historyLength = 0.0f;
	const V4 clipPrevious = mul(P.prev_view_proj, v4(r.position, 1.0f));
	if (P.history_valid > 0.5f && clipPrevious.w > 0.0001f)
	{
		const V2 projected = clipToUv(P, clipPrevious);
		const V2 previousUv = v2((floorf(projected.x * g.giSize.x) + 0.5f) * g.giTexel.x,
			(floorf(projected.y * g.giSize.y) + 0.5f) * g.giTexel.y);
		const int h = g.gi(previousUv);
		const float4 rp = __ldg(g.historyReceiver + h);
		const float4 rn = __ldg(g.historyNormal + h);
		const V3 receiverPosition = v3(rp.x, rp.y, rp.z);
		const V3 receiverNormal = v3(rn.x, rn.y, rn.z);
		const V3 offset = receiverPosition - r.position;
		if (isOnScreen(previousUv) && dot(receiverNormal, receiverNormal) > 0.5f
			&& dot(offset, offset) <= g.kBounceRadius() * g.kBounceRadius() && fabsf(dot(offset, r.normal)) <= g.kReceiverPlane()
			&& dot(normalize(receiverNormal), r.normal) >= 0.9f)
		{
			const V4 previous = loadH4(specularHistory, h);
			history = previous.xyz();
			historyLength = previous.w;
		}
	}
	const float maxHistory = mixf(4.0f, 32.0f, clampf(r.roughness * 1.5f, 0.0f, 1.0f));
	historyLength = fminf(historyLength + 1.0f, maxHistory);
	storeH4(out, i, v4(mix(history, demodulated, 1.0f / historyLength), historyLength));
}

// fs_specular.sc:127-226, one thread per GI pixel in 16x8 tiles.
__global__ void __launch_bounds__(128, RESTIR_SPECULAR_MIN_BLOCKS) giSpecularKernel(const RestirParams P, BvhView bvh, GiBindings b,
	const uint16_t* __restrict__ previousHdr, const uint16_t* __restrict__ specularHistory, uint16_t* out)
{
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	if (px >= g.w || py >= g.h)
	{
		return;
	}
	const int i = py * g.w + px;
	const SpecularRay r = specularRay(g, pixelUv(px, py, g.giTexel));
	if (!r.surface)
	{
		storeH4(out, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	V3 hitPosition = v3s(0.0f);
	float hitId = 0.0f;
	bool hit = false;
	if (r.normalLight > 0.0f)
	{
		if (P.ray_mode != RESTIR_RAY_MODE_BVH)
		{
			hit = g.traceScreenSpaceRay(r.origin, r.direction, g.kMaxRayDistance(), hitPosition);
		}
		if (!hit && P.ray_mode != RESTIR_RAY_MODE_SCREEN)
		{
			float hitDistance = 0.0f;
			// A fragment shader: no shared-memory stack, the stackless walk (bvh.sh:298-319).
			const int triangleIndex = traceBvh(g.bvh, r.origin, r.direction, g.kMaxBvhRayDistance(), false, hitDistance, nullptr, 0);
			hit = specularBvhHit(g, r, triangleIndex, hitDistance, hitPosition, hitId);
		}
	}
	specularFinish(g, r, hit, hitPosition, hitId, previousHdr, specularHistory, out, i);
}

// The pass as a wavefront (restir_gi_specular_wavefront), step 1: rays and
// depth-buffer marches; the rays the march does not answer go to the queue.
// records[i] = (screen-space hit position, tag): tag (the float's bits) -1 no
// hit, -2 the march's hit, else the ray's queue slot.
__global__ void __launch_bounds__(128) specularRaysKernel(const RestirParams P, BvhView bvh, GiBindings b, float4* records,
	RayQueue queue)
{
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	const bool inside = px < g.w && py < g.h;
	SpecularRay r = {};
	V3 hitPosition = v3s(0.0f);
	int tag = -1;
	bool push = false;
	if (inside)
	{
		r = specularRay(g, pixelUv(px, py, g.giTexel));
		if (r.surface && r.normalLight > 0.0f)
		{
			bool hit = false;
			if (P.ray_mode != RESTIR_RAY_MODE_BVH)
			{
				hit = g.traceScreenSpaceRay(r.origin, r.direction, g.kMaxRayDistance(), hitPosition);
			}
			tag = hit ? -2 : -1;
			push = !hit && P.ray_mode != RESTIR_RAY_MODE_SCREEN;
		}
	}
	// Every lane votes in the push, pixels outside the image included.
	const int slot = queuePush(queue, push, r.origin, g.kMaxBvhRayDistance(), r.direction);
	if (inside)
	{
		records[py * g.w + px] = make_float4(hitPosition.x, hitPosition.y, hitPosition.z, __int_as_float(push ? slot : tag));
	}
}

// Step 3: the rest of the pass from the recorded hits, replaying step 1's
// ray (the same two random numbers), so every value is giSpecularKernel's.
__global__ void __launch_bounds__(128, RESTIR_SPECULAR_MIN_BLOCKS) specularShadeKernel(const RestirParams P, BvhView bvh,
	GiBindings b, const float4* __restrict__ records, RayQueue queue, const uint16_t* __restrict__ previousHdr,
	const uint16_t* __restrict__ specularHistory, uint16_t* out)
{
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const int px = int(blockIdx.x * 16 + threadIdx.x % 16);
	const int py = int(blockIdx.y * 8 + threadIdx.x / 16);
	if (px >= g.w || py >= g.h)
	{
		return;
	}
	const int i = py * g.w + px;
	const SpecularRay r = specularRay(g, pixelUv(px, py, g.giTexel));
	if (!r.surface)
	{
		storeH4(out, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	V3 hitPosition = v3s(0.0f);
	float hitId = 0.0f;
	bool hit = false;
	if (r.normalLight > 0.0f)
	{
		const float4 record = __ldg(records + i);
		const int tag = __float_as_int(record.w);
		if (tag == -2)
		{
			hit = true;
			hitPosition = v3(record.x, record.y, record.z);
		}
		else if (tag >= 0)
		{
			hit = specularBvhHit(g, r, queue.hitTriangle[tag], queue.hitDistance[tag], hitPosition, hitId);
		}
	}
	specularFinish(g, r, hit, hitPosition, hitId, previousHdr, specularHistory, out, i);
}

__global__ void __launch_bounds__(128) traceQueueWalkKernel(BvhView bvh, RayQueue queue)
{
	traceQueueClosest<128, true>(bvh, queue, nullptr);
}

GiBindings bindings(const RestirGBuffer* gb, const RestirGiHistory* history, const uint32_t* grid, const float* shadowAtlas,
	const uint16_t* surfaceLight)
{
	GiBindings b = {};
	b.albedo = gb->albedo;
	b.normal = gb->normal;
	b.depth = gb->depth;
	b.historySample = reinterpret_cast<const float4*>(history->sample);
	b.historyReceiver = reinterpret_cast<const float4*>(history->receiver);
	b.historyNormal = reinterpret_cast<const float4*>(history->normal);
	b.historyColor = history->color;
	b.historyMoments = history->moments;
	b.surfaceLight = surfaceLight;
	b.shadowAtlas = shadowAtlas;
	b.grid = grid;
	return b;
}

bool validCommon(const RestirParams* p, const RestirScene* s, const RestirGBuffer* gb, const RestirGiHistory* h,
	const uint32_t* grid, const float* atlas)
{
	return p != nullptr && s != nullptr && gb != nullptr && h != nullptr && grid != nullptr && atlas != nullptr
		&& gb->albedo != nullptr && gb->normal != nullptr && gb->depth != nullptr && h->receiver != nullptr
		&& h->normal != nullptr && h->color != nullptr && p->gi_width > 0 && p->gi_height > 0 && p->trace_steps > 0
		&& p->grid_table_size >= 4u && (p->grid_table_size & (p->grid_table_size - 1u)) == 0u;
}

} // namespace
} // namespace restir

using namespace restir;

extern "C" int restir_gi_temporal(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas, const uint16_t* surface_light,
	const RestirGiReservoirs* output, void* stream)
{
	if (!validCommon(params, scene, gbuffer, history, previous_grid, shadow_atlas) || history->sample == nullptr
		|| output == nullptr || output->sample == nullptr || output->receiver == nullptr || output->normal == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	GiBindings b = bindings(gbuffer, history, previous_grid, shadow_atlas, surface_light);
	b.outSample = reinterpret_cast<float4*>(output->sample);
	b.outReceiver = reinterpret_cast<float4*>(output->receiver);
	b.outNormal = reinterpret_cast<float4*>(output->normal);
	const int groups = int((params->gi_width + 3) / 4 * ((params->gi_height + 7) / 8));
	giTemporalKernel<<<(groups + kGiWarps - 1) / kGiWarps, kGiThreads, 0, asStream(stream)>>>(*params, makeBvhView(scene), b);
	return launchStatus();
}

extern "C" int restir_gi_spatial(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiReservoirs* current, const uint32_t* current_grid, const RestirGiHistory* history, const float* shadow_atlas,
	const uint16_t* surface_light, uint16_t* color, uint16_t* moments, void* stream)
{
	if (!validCommon(params, scene, gbuffer, history, current_grid, shadow_atlas) || current == nullptr
		|| current->sample == nullptr || current->receiver == nullptr || current->normal == nullptr || color == nullptr
		|| moments == nullptr || history->moments == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	GiBindings b = bindings(gbuffer, history, current_grid, shadow_atlas, surface_light);
	b.reservoirSample = reinterpret_cast<const float4*>(current->sample);
	b.reservoirReceiver = reinterpret_cast<const float4*>(current->receiver);
	b.reservoirNormal = reinterpret_cast<const float4*>(current->normal);
	b.outColor = color;
	b.outMoments = moments;
	dim3 grid((params->gi_width + 15) / 16, (params->gi_height + 7) / 8);
	giSpatialKernel<<<grid, 128, 0, asStream(stream)>>>(*params, makeBvhView(scene), b);
	return launchStatus();
}

extern "C" int restir_gi_specular(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const float* shadow_atlas, const uint16_t* surface_light, const uint16_t* previous_hdr,
	const uint16_t* specular_history, uint16_t* specular, void* stream)
{
	if (params == nullptr || scene == nullptr || gbuffer == nullptr || history == nullptr || shadow_atlas == nullptr
		|| gbuffer->albedo == nullptr || gbuffer->normal == nullptr || gbuffer->depth == nullptr || history->receiver == nullptr
		|| history->normal == nullptr || history->color == nullptr || previous_hdr == nullptr || specular_history == nullptr
		|| specular == nullptr || specular == specular_history || params->gi_width == 0 || params->gi_height == 0
		|| params->trace_steps <= 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	GiBindings b = bindings(gbuffer, history, nullptr, shadow_atlas, surface_light);
	dim3 grid((params->gi_width + 15) / 16, (params->gi_height + 7) / 8);
	giSpecularKernel<<<grid, 128, 0, asStream(stream)>>>(*params, makeBvhView(scene), b, previous_hdr, specular_history,
		specular);
	return launchStatus();
}


namespace restir
{
namespace
{

// The radiance cache's share of the workspace: query rows and their values
// for the candidates then the reused reservoirs, and the training batch.
struct CacheWorkspace
{
	float4* queries;        // 4 float4 per row
	uint16_t* values;       // half4 per row
	uint32_t rows;
	RayQueue trainQueue;    // one suffix ray per training sample (no counter)
	float4* trainQueries;   // at the training points
	float4* hitQueries;     // at the suffixes' hit points
	uint16_t* hitValues;
	float4* partial;        // direct + emission at the hit (rgb), training weight
	float4* hitAlbedo;
	float4* targets;
	uint32_t samples;
};

struct TemporalWorkspace
{
	RayQueue queue;
	CandidateRecords records;
	CacheWorkspace cache;
	uint64_t bytes;
};

// [2 counters][rays 32 B x n][hit triangles 4 B x n][hit distances 4 B x n][screen hits 16 B x n]
// [slots 4 B x n], each region starting on 256 bytes; n = GI pixels x initial candidates. With the
// radiance cache: [queries 64 B x r][values 8 B x r], r = n + GI pixels, then the training batch of
// s samples: [rays 32 B][hit triangles 4 B][hit distances 4 B][2 counters][training queries 64 B]
// [hit queries 64 B][hit values 8 B][partial 16 B][hit albedo 16 B][targets 16 B], each x s.
TemporalWorkspace layoutTemporalWorkspace(const RestirParams* p, void* base)
{
	const uint64_t n = uint64_t(p->gi_width) * p->gi_height * uint64_t(p->initial_candidates > 0 ? p->initial_candidates : 0);
	char* at = static_cast<char*>(base);
	uint64_t offset = 0;
	auto region = [&](uint64_t bytes) -> char*
	{
		char* start = at + offset;
		offset += (bytes + 255u) & ~uint64_t(255u);
		return start;
	};
	TemporalWorkspace w = {};
	uint32_t* counters = reinterpret_cast<uint32_t*>(region(2 * sizeof(uint32_t)));
	w.queue.count = counters;
	w.queue.claimed = counters + 1;
	w.queue.rays = reinterpret_cast<float4*>(region(n * 32));
	w.queue.hitTriangle = reinterpret_cast<int*>(region(n * 4));
	w.queue.hitDistance = reinterpret_cast<float*>(region(n * 4));
	w.records.screenHit = reinterpret_cast<float4*>(region(n * 16));
	w.records.slot = reinterpret_cast<int*>(region(n * 4));
	w.queue.capacity = uint32_t(n);
	w.records.candidates = p->initial_candidates;
	if (p->radiance_cache > 0.5f)
	{
		CacheWorkspace& c = w.cache;
		c.rows = uint32_t(n + uint64_t(p->gi_width) * p->gi_height);
		c.queries = reinterpret_cast<float4*>(region(uint64_t(c.rows) * 64));
		c.values = reinterpret_cast<uint16_t*>(region(uint64_t(c.rows) * 8));
		c.samples = p->cache_training_samples;
		const uint64_t s = c.samples;
		c.trainQueue.rays = reinterpret_cast<float4*>(region(s * 32));
		c.trainQueue.hitTriangle = reinterpret_cast<int*>(region(s * 4));
		c.trainQueue.hitDistance = reinterpret_cast<float*>(region(s * 4));
		c.trainQueue.claimed = reinterpret_cast<uint32_t*>(region(2 * sizeof(uint32_t)));
		c.trainQueue.count = nullptr;
		c.trainQueue.capacity = c.samples;
		c.trainQueries = reinterpret_cast<float4*>(region(s * 64));
		c.hitQueries = reinterpret_cast<float4*>(region(s * 64));
		c.hitValues = reinterpret_cast<uint16_t*>(region(s * 8));
		c.partial = reinterpret_cast<float4*>(region(s * 16));
		c.hitAlbedo = reinterpret_cast<float4*>(region(s * 16));
		c.targets = reinterpret_cast<float4*>(region(s * 16));
	}
	w.bytes = offset;
	return w;
}

// One resident grid of a queue tracer of 128 threads per block: SMs x blocks
// that fit on one SM.
int residentBlocks(const void* kernel)
{
	int device = 0, sms = 148, perSm = 0;
	if (cudaGetDevice(&device) == cudaSuccess)
	{
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	}
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, 128, 0) != cudaSuccess || perSm < 1)
	{
		perSm = 1;
	}
	return sms * perSm;
}

int persistentBlocks()
{
	static int blocks = 0;
	if (blocks == 0)
	{
		blocks = residentBlocks(reinterpret_cast<const void*>(traceQueueKernel));
	}
	return blocks;
}

int walkBlocks()
{
	static int blocks = 0;
	if (blocks == 0)
	{
		blocks = residentBlocks(reinterpret_cast<const void*>(traceQueueWalkKernel));
	}
	return blocks;
}

// The specular wavefront's workspace: [2 counters][rays 32 B x n][hit triangles
// 4 B x n][hit distances 4 B x n][records 16 B x n], each region starting on 256
// bytes; n = GI pixels.
struct SpecularWorkspace
{
	RayQueue queue;
	float4* records;
	uint64_t bytes;
};

SpecularWorkspace layoutSpecularWorkspace(const RestirParams* p, void* base)
{
	const uint64_t n = uint64_t(p->gi_width) * p->gi_height;
	char* at = static_cast<char*>(base);
	uint64_t offset = 0;
	auto region = [&](uint64_t bytes) -> char*
	{
		char* start = at + offset;
		offset += (bytes + 255u) & ~uint64_t(255u);
		return start;
	};
	SpecularWorkspace w = {};
	uint32_t* counters = reinterpret_cast<uint32_t*>(region(2 * sizeof(uint32_t)));
	w.queue.count = counters;
	w.queue.claimed = counters + 1;
	w.queue.rays = reinterpret_cast<float4*>(region(n * 32));
	w.queue.hitTriangle = reinterpret_cast<int*>(region(n * 4));
	w.queue.hitDistance = reinterpret_cast<float*>(region(n * 4));
	w.records = reinterpret_cast<float4*>(region(n * 16));
	w.queue.capacity = uint32_t(n);
	w.bytes = offset;
	return w;
}

} // namespace
} // namespace restir

extern "C" uint64_t restir_gi_temporal_workspace_bytes(const RestirParams* params)
{
	if (params == nullptr)
	{
		return 0;
	}
	return layoutTemporalWorkspace(params, nullptr).bytes;
}

extern "C" int restir_gi_temporal_wavefront(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas, const uint16_t* surface_light,
	const RestirGiReservoirs* output, void* workspace, uint64_t workspace_bytes, void* stream)
{
	if (!validCommon(params, scene, gbuffer, history, previous_grid, shadow_atlas) || history->sample == nullptr
		|| output == nullptr || output->sample == nullptr || output->receiver == nullptr || output->normal == nullptr
		|| workspace == nullptr || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0u || params->initial_candidates < 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	TemporalWorkspace w = layoutTemporalWorkspace(params, workspace);
	if (workspace_bytes < w.bytes)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	GiBindings b = bindings(gbuffer, history, previous_grid, shadow_atlas, surface_light);
	b.outSample = reinterpret_cast<float4*>(output->sample);
	b.outReceiver = reinterpret_cast<float4*>(output->receiver);
	b.outNormal = reinterpret_cast<float4*>(output->normal);
	const BvhView bvh = makeBvhView(scene);
	cudaStream_t s = asStream(stream);
	const int groups = int((params->gi_width + 3) / 4 * ((params->gi_height + 7) / 8));
	const int blocks = (groups + kGiWarps - 1) / kGiWarps;
	cudaMemsetAsync(workspace, 0, 2 * sizeof(uint32_t), s);
	giCandidatesKernel<<<blocks, kGiThreads, 0, s>>>(*params, bvh, b, w.records, w.queue);
	traceQueueKernel<<<persistentBlocks(), 128, 0, s>>>(bvh, w.queue);
	giTemporalShadeKernel<<<blocks, kGiThreads, 0, s>>>(*params, bvh, b, w.records, w.queue);
	return launchStatus();
}

extern "C" uint64_t restir_gi_specular_workspace_bytes(const RestirParams* params)
{
	if (params == nullptr)
	{
		return 0;
	}
	return layoutSpecularWorkspace(params, nullptr).bytes;
}

extern "C" int restir_gi_specular_wavefront(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const float* shadow_atlas, const uint16_t* surface_light, const uint16_t* previous_hdr,
	const uint16_t* specular_history, uint16_t* specular, void* workspace, uint64_t workspace_bytes, void* stream)
{
	if (params == nullptr || scene == nullptr || gbuffer == nullptr || history == nullptr || shadow_atlas == nullptr
		|| gbuffer->albedo == nullptr || gbuffer->normal == nullptr || gbuffer->depth == nullptr || history->receiver == nullptr
		|| history->normal == nullptr || history->color == nullptr || previous_hdr == nullptr || specular_history == nullptr
		|| specular == nullptr || specular == specular_history || params->gi_width == 0 || params->gi_height == 0
		|| params->trace_steps <= 0 || workspace == nullptr || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0u)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	SpecularWorkspace w = layoutSpecularWorkspace(params, workspace);
	if (workspace_bytes < w.bytes)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	GiBindings b = bindings(gbuffer, history, nullptr, shadow_atlas, surface_light);
	const BvhView bvh = makeBvhView(scene);
	cudaStream_t s = asStream(stream);
	dim3 grid((params->gi_width + 15) / 16, (params->gi_height + 7) / 8);
	cudaMemsetAsync(workspace, 0, 2 * sizeof(uint32_t), s);
	specularRaysKernel<<<grid, 128, 0, s>>>(*params, bvh, b, w.records, w.queue);
	traceQueueWalkKernel<<<walkBlocks(), 128, 0, s>>>(bvh, w.queue);
	specularShadeKernel<<<grid, 128, 0, s>>>(*params, bvh, b, w.records, w.queue, previous_hdr, specular_history, specular);
	return launchStatus();
}

// --- the wavefront's three steps with a caller-owned, shareable ray queue ---------
//
// Several views (or frames) can append to one queue and have it traced by a
// single persistent launch: restir_gi_temporal_candidates for each, one
// restir_trace_queue, restir_gi_temporal_shade for each.

namespace restir
{
namespace
{

// [2 counters][rays 32 B x c][hit triangles 4 B x c][hit distances 4 B x c], each on 256 bytes.
RayQueue layoutQueue(void* base, uint32_t capacity, uint64_t* bytes)
{
	char* at = static_cast<char*>(base);
	uint64_t offset = 0;
	auto region = [&](uint64_t size) -> char*
	{
		char* start = at + offset;
		offset += (size + 255u) & ~uint64_t(255u);
		return start;
	};
	RayQueue q;
	uint32_t* counters = reinterpret_cast<uint32_t*>(region(2 * sizeof(uint32_t)));
	q.count = counters;
	q.claimed = counters + 1;
	q.rays = reinterpret_cast<float4*>(region(uint64_t(capacity) * 32));
	q.hitTriangle = reinterpret_cast<int*>(region(uint64_t(capacity) * 4));
	q.hitDistance = reinterpret_cast<float*>(region(uint64_t(capacity) * 4));
	q.capacity = capacity;
	if (bytes != nullptr)
	{
		*bytes = offset;
	}
	return q;
}

// [screen hits 16 B x n][slots 4 B x n], n = GI pixels x initial candidates.
CandidateRecords layoutRecords(const RestirParams* p, void* base, uint64_t* bytes)
{
	const uint64_t n = uint64_t(p->gi_width) * p->gi_height * uint64_t(p->initial_candidates > 0 ? p->initial_candidates : 0);
	CandidateRecords r;
	r.screenHit = static_cast<float4*>(base);
	r.slot = reinterpret_cast<int*>(static_cast<char*>(base) + ((n * 16 + 255u) & ~uint64_t(255u)));
	r.candidates = p->initial_candidates;
	if (bytes != nullptr)
	{
		*bytes = ((n * 16 + 255u) & ~uint64_t(255u)) + ((n * 4 + 255u) & ~uint64_t(255u));
	}
	return r;
}

bool aligned(const void* p)
{
	return p != nullptr && (reinterpret_cast<uintptr_t>(p) & 255u) == 0u;
}

template<int kThreads>
int launchQueueTracer(const BvhView& bvh, const RayQueue& q, uint32_t blocksPerSm, cudaStream_t s)
{
	// SM count and resident blocks, queried once (not inside a stream capture on later calls).
	static int sms = 0, fit = 0;
	if (sms == 0)
	{
		int device = 0;
		sms = 148;
		if (cudaGetDevice(&device) == cudaSuccess)
		{
			cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
		}
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, traceQueueSizedKernel<kThreads>, kThreads, 0) != cudaSuccess
			|| fit < 1)
		{
			fit = 1;
		}
	}
	int perSm = fit;
	if (blocksPerSm > 0u && int(blocksPerSm) < perSm)
	{
		perSm = int(blocksPerSm);
	}
	traceQueueSizedKernel<kThreads><<<sms * perSm, kThreads, 0, s>>>(bvh, q);
	return launchStatus();
}

} // namespace
} // namespace restir

extern "C" uint64_t restir_ray_queue_bytes(uint32_t capacity)
{
	uint64_t bytes = 0;
	layoutQueue(nullptr, capacity, &bytes);
	return bytes;
}

extern "C" int restir_ray_queue_reset(void* queue, void* stream)
{
	if (!aligned(queue))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return cudaMemsetAsync(queue, 0, 2 * sizeof(uint32_t), asStream(stream)) == cudaSuccess ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
}

extern "C" uint64_t restir_gi_candidate_records_bytes(const RestirParams* params)
{
	if (params == nullptr)
	{
		return 0;
	}
	uint64_t bytes = 0;
	layoutRecords(params, nullptr, &bytes);
	return bytes;
}

extern "C" int restir_gi_temporal_candidates(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas, const uint16_t* surface_light,
	void* records, uint64_t records_bytes, void* queue, uint32_t queue_capacity, void* stream)
{
	if (!validCommon(params, scene, gbuffer, history, previous_grid, shadow_atlas) || params->initial_candidates < 0
		|| !aligned(records) || !aligned(queue))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	uint64_t needed = 0;
	CandidateRecords r = layoutRecords(params, records, &needed);
	if (records_bytes < needed)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const RayQueue q = layoutQueue(queue, queue_capacity, nullptr);
	GiBindings b = bindings(gbuffer, history, previous_grid, shadow_atlas, surface_light);
	const int groups = int((params->gi_width + 3) / 4 * ((params->gi_height + 7) / 8));
	giCandidatesKernel<<<(groups + kGiWarps - 1) / kGiWarps, kGiThreads, 0, asStream(stream)>>>(*params, makeBvhView(scene), b,
		r, q);
	return launchStatus();
}

extern "C" int restir_trace_queue(const RestirScene* scene, void* queue, uint32_t queue_capacity, uint32_t threads,
	uint32_t blocks_per_sm, void* stream)
{
	if (scene == nullptr || !aligned(queue))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const RayQueue q = layoutQueue(queue, queue_capacity, nullptr);
	const BvhView bvh = makeBvhView(scene);
	cudaStream_t s = asStream(stream);
	switch (threads)
	{
	case 64:
		return launchQueueTracer<64>(bvh, q, blocks_per_sm, s);
	case 128:
		return launchQueueTracer<128>(bvh, q, blocks_per_sm, s);
	case 256:
		return launchQueueTracer<256>(bvh, q, blocks_per_sm, s);
	default:
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
}

extern "C" int restir_gi_temporal_shade(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas, const uint16_t* surface_light,
	const RestirGiReservoirs* output, const void* records, uint64_t records_bytes, const void* queue,
	uint32_t queue_capacity, void* stream)
{
	if (!validCommon(params, scene, gbuffer, history, previous_grid, shadow_atlas) || history->sample == nullptr
		|| output == nullptr || output->sample == nullptr || output->receiver == nullptr || output->normal == nullptr
		|| params->initial_candidates < 0 || !aligned(records) || !aligned(queue))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	uint64_t needed = 0;
	CandidateRecords r = layoutRecords(params, const_cast<void*>(records), &needed);
	if (records_bytes < needed)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const RayQueue q = layoutQueue(const_cast<void*>(queue), queue_capacity, nullptr);
	GiBindings b = bindings(gbuffer, history, previous_grid, shadow_atlas, surface_light);
	b.outSample = reinterpret_cast<float4*>(output->sample);
	b.outReceiver = reinterpret_cast<float4*>(output->receiver);
	b.outNormal = reinterpret_cast<float4*>(output->normal);
	const int groups = int((params->gi_width + 3) / 4 * ((params->gi_height + 7) / 8));
	giTemporalShadeKernel<<<(groups + kGiWarps - 1) / kGiWarps, kGiThreads, 0, asStream(stream)>>>(*params, makeBvhView(scene),
		b, r, q);
	return launchStatus();
}

// --- the radiance cache in the GI passes -----------------------------------------
//
// restir_gi_temporal_cached and restir_gi_spatial_cached are the GI passes
// with the cache standing in for previousIndirect: before shading, one query
// row per sample point the pass may shade (the candidates' hits, the reused
// reservoirs' samples) is filled with the point's surface as evaluateSample
// finds it, the cache answers all rows in one tensor-core launch, and the
// shading reads the answers by slot. restir_cache_train_frame traces the
// training batch: path suffixes from G-buffer points, each target the light
// leaving the suffix's first hit, with the cache's own value there standing
// for everything beyond it.

namespace restir
{
namespace
{

__device__ __forceinline__ void writeQuery(float4* q, V3 position, float roughness, V3 normal, bool valid, V3 direction,
	V3 albedo)
{
	q[0] = make_float4(position.x, position.y, position.z, roughness);
	q[1] = make_float4(normal.x, normal.y, normal.z, valid ? 1.0f : 0.0f);
	q[2] = make_float4(direction.x, direction.y, direction.z, 0.0f);
	q[3] = make_float4(albedo.x, albedo.y, albedo.z, 0.0f);
}

// The query for a sample point shaded for a receiver: its surface as
// evaluateSample finds it (restir.sh:466-495), the direction toward the
// receiver; a padding row when the point is the sky or cannot be shaded.
__device__ inline void sampleQuery(const GiPass& g, V3 receiver, V3 samplePosition, float sampleId, bool present, float4* q)
{
	bool visible = false;
	V2 uv = v2(0.0f, 0.0f);
	int triangle = -1;
	V3 normal = v3(0.0f, 0.0f, 1.0f);
	if (!present || isSkySample(sampleId) || !g.sampleSurface(samplePosition, sampleId, visible, uv, triangle, normal))
	{
		writeQuery(q, samplePosition, 0.0f, normal, false, normal, v3s(0.0f));
		return;
	}
	const V3 albedo = visible ? g.diffuseAlbedo(uv) : g.bvh.albedo(triangle);
	const float roughness = visible ? loadU8(g.albedoTex, g.full(uv)).w : 1.0f;
	const V3 toReceiver = receiver - samplePosition;
	const float distanceSquared = dot(toReceiver, toReceiver);
	const V3 direction = distanceSquared > 0.0f ? toReceiver * inversesqrt(distanceSquared) : normal;
	writeQuery(q, samplePosition, roughness, normal, true, direction, albedo);
}

// One row per candidate: its hit resolved as giTemporalShadeKernel resolves it.
__global__ void __launch_bounds__(128) candidateQueryKernel(const RestirParams P, BvhView bvh, GiBindings b,
	CandidateRecords records, RayQueue queue, float4* queries)
{
	const int r = int(blockIdx.x * blockDim.x + threadIdx.x);
	const int w = int(P.gi_width), h = int(P.gi_height);
	if (r >= w * h * records.candidates)
	{
		return;
	}
	GiPass g = makePass(P, bvh, b, P.prev_camera_position, nullptr, 0);
	const int pixel = r / records.candidates;
	const V2 uv = pixelUv(pixel % w, pixel / w, g.giTexel);
	const float depth = g.depthAt(uv);
	const V3 receiver = reconstructWorldPosition(P, uv, depth);
	const float4 screen = records.screenHit[r];
	const int slot = records.slot[r];
	V3 hitPosition = v3(screen.x, screen.y, screen.z);
	float hitId = 0.0f;
	bool present = false;
	if (slot >= 0)
	{
		const int triangle = queue.hitTriangle[slot];
		if (triangle >= 0)
		{
			const float4 o = queue.rays[2 * slot];
			const float4 d = queue.rays[2 * slot + 1];
			const V3 direction = v3(d.x, d.y, d.z);
			hitPosition = v3(o.x, o.y, o.z) + direction * queue.hitDistance[slot];
			hitId = g.encodeSampleId(triangle, direction);
			present = true;
		}
	}
	else if (slot == -2)
	{
		present = screen.w > 0.5f;
	}
	sampleQuery(g, receiver, hitPosition, hitId, present && depth < kSkyDepth, queries + size_t(r) * 4);
}

// One row per reservoir of a GI-resolution set (last frame's, or this frame's
// for the spatial pass).
__global__ void __launch_bounds__(128) reservoirQueryKernel(const RestirParams P, BvhView bvh, GiBindings b,
	const float4* sample, const float4* receiver, const float4* normal, float4* queries)
{
	const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
	if (i >= int(P.gi_width * P.gi_height))
	{
		return;
	}
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const float4 s = __ldg(sample + i);
	const float4 r = __ldg(receiver + i);
	const float4 n = __ldg(normal + i);
	sampleQuery(g, v3(r.x, r.y, r.z), v3(s.x, s.y, s.z), n.w, s.w > 0.0f, queries + size_t(i) * 4);
}

// The cache-only form: one row per GI pixel at its own G-buffer surface, the
// query the training points use (trainingRaysKernel): the view direction,
// the surface's roughness and diffuse albedo.
__global__ void __launch_bounds__(128) primaryQueryKernel(const RestirParams P, BvhView bvh, GiBindings b, float4* queries)
{
	const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
	if (i >= int(P.gi_width * P.gi_height))
	{
		return;
	}
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const V2 uv = pixelUv(i % g.w, i / g.w, g.giTexel);
	const float depth = g.depthAt(uv);
	const V3 position = reconstructWorldPosition(P, uv, depth);
	const V3 normal = g.decode(uv);
	const V3 camera = v3(P.camera_position[0], P.camera_position[1], P.camera_position[2]);
	const V3 toCamera = camera - position;
	const float distanceSquared = dot(toCamera, toCamera);
	const V3 view = distanceSquared > 0.0f ? toCamera * inversesqrt(distanceSquared) : normal;
	writeQuery(queries + size_t(i) * 4, position, loadU8(g.albedoTex, g.full(uv)).w, normal, depth < kSkyDepth, view,
		g.diffuseAlbedo(uv));
}

// The GI targets from the cache's values: demodulated irradiance (clamped as
// the spatial pass clamps, albedo x irradiance <= the outlier clamp), its
// moments for the denoiser, and the receiver rows the later passes read.
__global__ void __launch_bounds__(128) giFromCacheKernel(const RestirParams P, BvhView bvh, GiBindings b,
	const uint16_t* __restrict__ values, float4* outSample, float4* outReceiver, float4* outNormal, uint16_t* color,
	uint16_t* moments)
{
	const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
	if (i >= int(P.gi_width * P.gi_height))
	{
		return;
	}
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const V2 uv = pixelUv(i % g.w, i / g.w, g.giTexel);
	const float depth = g.depthAt(uv);
	outSample[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	if (depth >= kSkyDepth)
	{
		outReceiver[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		outNormal[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		storeH4(color, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		storeH4(moments, i, v4(0.0f, 0.0f, 0.0f, 0.0f));
		return;
	}
	const V3 position = reconstructWorldPosition(P, uv, depth);
	const V3 normal = g.decode(uv);
	const V4 value = loadH4(values, i);
	V3 irradiance = value.w > 0.5f ? vmax(value.xyz(), v3s(0.0f)) : v3s(0.0f);
	if (P.outlier_clamp > 0.0f)
	{
		const V3 albedo = g.diffuseAlbedo(uv);
		irradiance = v3(fminf(irradiance.x, P.outlier_clamp / fmaxf(albedo.x, 1e-4f)),
			fminf(irradiance.y, P.outlier_clamp / fmaxf(albedo.y, 1e-4f)), fminf(irradiance.z, P.outlier_clamp / fmaxf(albedo.z, 1e-4f)));
	}
	const float l = luminance(irradiance);
	outReceiver[i] = make_float4(position.x, position.y, position.z, 1.0f);
	outNormal[i] = make_float4(normal.x, normal.y, normal.z, 0.0f);
	storeH4(color, i, v4(irradiance, 1.0f));
	storeH4(moments, i, v4(l, l * l, 1.0f, 0.0f));
}

// Training: sample j < count starts at a seeded GI pixel's G-buffer surface
// and traces one cosine-distributed suffix ray.
__global__ void __launch_bounds__(128) trainingRaysKernel(const RestirParams P, BvhView bvh, GiBindings b, CacheWorkspace c,
	uint32_t count)
{
	const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= count)
	{
		return;
	}
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const uint32_t pixels = P.gi_width * P.gi_height;
	uint32_t rng = pcg(j + pcg(uint32_t(P.frame_index) ^ 0x2545f491u));
	const uint32_t pixel = pcg(rng) % pixels;
	const V2 uv = pixelUv(int(pixel % P.gi_width), int(pixel / P.gi_width), g.giTexel);
	const float depth = g.depthAt(uv);
	const bool valid = depth < kSkyDepth;
	const V3 position = reconstructWorldPosition(P, uv, depth);
	const V3 normal = g.decode(uv);
	const float r0 = nextRandom(rng);
	const float r1 = nextRandom(rng);
	const V3 direction = GiPass::cosineHemisphere(normal, r0, r1);
	const V3 origin = position + normal * g.kRayBias();
	c.trainQueue.rays[2 * j] = make_float4(origin.x, origin.y, origin.z, valid ? g.kMaxBvhRayDistance() : 0.0f);
	c.trainQueue.rays[2 * j + 1] = make_float4(direction.x, direction.y, direction.z, 0.0f);
	const V3 camera = v3(P.camera_position[0], P.camera_position[1], P.camera_position[2]);
	const V3 toCamera = camera - position;
	const float distanceSquared = dot(toCamera, toCamera);
	const V3 view = distanceSquared > 0.0f ? toCamera * inversesqrt(distanceSquared) : normal;
	writeQuery(c.trainQueries + size_t(j) * 4, position, loadU8(g.albedoTex, g.full(uv)).w, normal, valid, view,
		g.diffuseAlbedo(uv));
}

// The suffix's first hit (rows begin..end-1): its direct light and emission
// now, a query for the cache's value there.
__global__ void __launch_bounds__(128) trainingHitsKernel(const RestirParams P, BvhView bvh, GiBindings b, CacheWorkspace c,
	uint32_t begin, uint32_t end)
{
	const uint32_t j = begin + blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= end)
	{
		return;
	}
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const float weight = c.trainQueries[size_t(j) * 4 + 1].w;
	const int triangle = c.trainQueue.hitTriangle[j];
	const float4 o = c.trainQueue.rays[2 * j];
	const float4 d = c.trainQueue.rays[2 * j + 1];
	const V3 direction = v3(d.x, d.y, d.z);
	V3 light = v3s(0.0f);
	V3 albedo = v3s(0.0f);
	float4* q = c.hitQueries + size_t(j) * 4;
	if (weight > 0.0f && triangle >= 0)
	{
		const V3 hit = v3(o.x, o.y, o.z) + direction * c.trainQueue.hitDistance[j];
		const float id = g.encodeSampleId(triangle, direction);
		const V3 v0 = bvh.vertex(triangle, 0);
		const V3 normal = normalize(cross(bvh.vertex(triangle, 1) - v0, bvh.vertex(triangle, 2) - v0)) * (id < 0.0f ? -1.0f : 1.0f);
		albedo = bvh.albedo(triangle);
		light = g.directFromLight(albedo, hit, normal) + bvh.emission(triangle) * P.emission_scale;
		writeQuery(q, hit, 1.0f, normal, true, -direction, albedo);
	}
	else
	{
		if (weight > 0.0f && skyEnabled(P))
		{
			light = skyRadiance(P, direction);
		}
		writeQuery(q, v3s(0.0f), 0.0f, v3(0.0f, 0.0f, 1.0f), false, v3(0.0f, 0.0f, 1.0f), v3s(0.0f));
	}
	// The row's frame, so that the next frame's call can tell these hits from
	// any other content of the workspace (an unused word of the query row).
	q[3].w = __uint_as_float(uint32_t(P.frame_index) + 1u);
	c.partial[j] = make_float4(light.x, light.y, light.z, weight);
	c.hitAlbedo[j] = make_float4(albedo.x, albedo.y, albedo.z, 0.0f);
}

// The second half of the training rows: row first + j starts where row j's
// suffix hit in the previous frame's call (the point a GI sample of a visible
// surface lands on, and where the GI passes query the cache), with that
// hit's query (its surface, the direction back toward row j's point), and
// traces its own cosine-distributed suffix. The previous frame's rows are
// read from the workspace before this call's hits replace them, so both
// halves trace in one launch. Rows whose suffix left the scene, and any row
// not written by the previous frame's call (the tag in the query row's last
// word is that frame's index + 1), are padding (weight 0).
__global__ void __launch_bounds__(128) trainingSecondRaysKernel(const RestirParams P, BvhView bvh, GiBindings b,
	CacheWorkspace c, uint32_t first, uint32_t count)
{
	const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= count)
	{
		return;
	}
	GiPass g = makePass(P, bvh, b, P.camera_position, nullptr, 0);
	const uint32_t row = first + j;
	const float4* hit = c.hitQueries + size_t(j) * 4;
	float4* query = c.trainQueries + size_t(row) * 4;
	const bool valid = hit[1].w > 0.5f && __float_as_uint(hit[3].w) == uint32_t(P.frame_index);
	if (!valid)
	{
		// A padding row: a clean query (whatever the workspace held) and an empty ray.
		writeQuery(query, v3s(0.0f), 0.0f, v3(0.0f, 0.0f, 1.0f), false, v3(0.0f, 0.0f, 1.0f), v3s(0.0f));
		c.trainQueue.rays[2 * row] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		c.trainQueue.rays[2 * row + 1] = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
		return;
	}
	for (int k = 0; k < 4; ++k)
	{
		query[k] = hit[k];
	}
	uint32_t rng = pcg(row + pcg(uint32_t(P.frame_index) ^ 0x2545f491u));
	const float r0 = nextRandom(rng);
	const float r1 = nextRandom(rng);
	const V3 position = v3(hit[0].x, hit[0].y, hit[0].z);
	const V3 normal = v3(hit[1].x, hit[1].y, hit[1].z);
	const V3 direction = GiPass::cosineHemisphere(normal, r0, r1);
	const V3 origin = position + normal * g.kRayBias();
	c.trainQueue.rays[2 * row] = make_float4(origin.x, origin.y, origin.z, g.kMaxBvhRayDistance());
	c.trainQueue.rays[2 * row + 1] = make_float4(direction.x, direction.y, direction.z, 0.0f);
}

// The training target: the light arriving along the suffix, i.e. its hit's
// direct light and emission plus its albedo times the cache's value there.
// With the outlier clamp on, the target is held to what the spatial pass
// lets through at the training point (albedo x irradiance <= clamp,
// cs_restir_spatial.sc:188-192): the same bias as the plain method, and a
// bound on the loop through which the cache trains on its own values.
__global__ void __launch_bounds__(128) trainingTargetsKernel(CacheWorkspace c, float outlierClamp)
{
	const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= c.samples)
	{
		return;
	}
	const float4 partial = c.partial[j];
	const float4 albedo = c.hitAlbedo[j];
	const V4 cached = loadH4(c.hitValues, int(j));
	const float beyond = cached.w > 0.5f ? 1.0f : 0.0f;
	V3 target = v3(partial.x + albedo.x * cached.x * beyond, partial.y + albedo.y * cached.y * beyond,
		partial.z + albedo.z * cached.z * beyond);
	if (outlierClamp > 0.0f)
	{
		const float4 receiver = c.trainQueries[size_t(j) * 4 + 3];
		target = v3(fminf(target.x, outlierClamp / fmaxf(receiver.x, 1e-4f)), fminf(target.y, outlierClamp / fmaxf(receiver.y, 1e-4f)),
			fminf(target.z, outlierClamp / fmaxf(receiver.z, 1e-4f)));
	}
	c.targets[j] = make_float4(target.x, target.y, target.z, partial.w);
}

bool validCache(const RestirCacheConfig* cfg, const void* state)
{
	return cfg != nullptr && state != nullptr && (reinterpret_cast<uintptr_t>(state) & 255u) == 0u;
}

int gridFor(uint32_t n)
{
	return int((n + 127u) / 128u);
}

} // namespace
} // namespace restir

extern "C" int restir_gi_temporal_cached(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas, const uint16_t* surface_light,
	const RestirGiReservoirs* output, const RestirCacheConfig* cache_config, const void* cache_state, void* workspace,
	uint64_t workspace_bytes, void* stream)
{
	if (!validCommon(params, scene, gbuffer, history, previous_grid, shadow_atlas) || history->sample == nullptr
		|| output == nullptr || output->sample == nullptr || output->receiver == nullptr || output->normal == nullptr
		|| workspace == nullptr || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0u || params->initial_candidates < 0
		|| params->radiance_cache <= 0.5f || !validCache(cache_config, cache_state))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	TemporalWorkspace w = layoutTemporalWorkspace(params, workspace);
	if (workspace_bytes < w.bytes)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	GiBindings b = bindings(gbuffer, history, previous_grid, shadow_atlas, surface_light);
	b.outSample = reinterpret_cast<float4*>(output->sample);
	b.outReceiver = reinterpret_cast<float4*>(output->receiver);
	b.outNormal = reinterpret_cast<float4*>(output->normal);
	const BvhView bvh = makeBvhView(scene);
	cudaStream_t s = asStream(stream);
	const int groups = int((params->gi_width + 3) / 4 * ((params->gi_height + 7) / 8));
	const int blocks = (groups + kGiWarps - 1) / kGiWarps;
	const uint32_t candidates = w.queue.capacity;
	const uint32_t pixels = params->gi_width * params->gi_height;
	cudaMemsetAsync(workspace, 0, 2 * sizeof(uint32_t), s);
	giCandidatesKernel<<<blocks, kGiThreads, 0, s>>>(*params, bvh, b, w.records, w.queue);
	traceQueueKernel<<<persistentBlocks(), 128, 0, s>>>(bvh, w.queue);
	if (candidates > 0u)
	{
		candidateQueryKernel<<<gridFor(candidates), 128, 0, s>>>(*params, bvh, b, w.records, w.queue, w.cache.queries);
	}
	reservoirQueryKernel<<<gridFor(pixels), 128, 0, s>>>(*params, bvh, b, b.historySample, b.historyReceiver,
		b.historyNormal, w.cache.queries + size_t(candidates) * 4);
	int status = restir_cache_query(cache_config, cache_state, reinterpret_cast<const float*>(w.cache.queries), w.cache.rows,
		w.cache.values, stream);
	if (status != RESTIR_OK)
	{
		return status;
	}
	b.cache = w.cache.values;
	b.cacheNeighbourBase = int(candidates);
	giTemporalShadeKernel<<<blocks, kGiThreads, 0, s>>>(*params, bvh, b, w.records, w.queue);
	return launchStatus();
}

extern "C" int restir_gi_spatial_cached(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiReservoirs* current, const uint32_t* current_grid, const RestirGiHistory* history, const float* shadow_atlas,
	const uint16_t* surface_light, uint16_t* color, uint16_t* moments, const RestirCacheConfig* cache_config,
	const void* cache_state, void* workspace, uint64_t workspace_bytes, void* stream)
{
	if (!validCommon(params, scene, gbuffer, history, current_grid, shadow_atlas) || current == nullptr
		|| current->sample == nullptr || current->receiver == nullptr || current->normal == nullptr || color == nullptr
		|| moments == nullptr || history->moments == nullptr || workspace == nullptr
		|| (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0u || params->radiance_cache <= 0.5f
		|| !validCache(cache_config, cache_state))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	TemporalWorkspace w = layoutTemporalWorkspace(params, workspace);
	if (workspace_bytes < w.bytes)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	GiBindings b = bindings(gbuffer, history, current_grid, shadow_atlas, surface_light);
	b.reservoirSample = reinterpret_cast<const float4*>(current->sample);
	b.reservoirReceiver = reinterpret_cast<const float4*>(current->receiver);
	b.reservoirNormal = reinterpret_cast<const float4*>(current->normal);
	b.outColor = color;
	b.outMoments = moments;
	const BvhView bvh = makeBvhView(scene);
	cudaStream_t s = asStream(stream);
	const uint32_t pixels = params->gi_width * params->gi_height;
	reservoirQueryKernel<<<gridFor(pixels), 128, 0, s>>>(*params, bvh, b, b.reservoirSample, b.reservoirReceiver,
		b.reservoirNormal, w.cache.queries);
	int status = restir_cache_query(cache_config, cache_state, reinterpret_cast<const float*>(w.cache.queries), pixels,
		w.cache.values, stream);
	if (status != RESTIR_OK)
	{
		return status;
	}
	b.cache = w.cache.values;
	b.cacheNeighbourBase = 0;
	dim3 grid((params->gi_width + 15) / 16, (params->gi_height + 7) / 8);
	giSpatialKernel<<<grid, 128, 0, s>>>(*params, bvh, b);
	return launchStatus();
}

extern "C" int restir_gi_from_cache(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirCacheConfig* cache_config, const void* cache_state, void* workspace, uint64_t workspace_bytes,
	const RestirGiReservoirs* output, uint16_t* color, uint16_t* moments, void* stream)
{
	if (params == nullptr || scene == nullptr || gbuffer == nullptr || gbuffer->albedo == nullptr || gbuffer->normal == nullptr
		|| gbuffer->depth == nullptr || output == nullptr || output->sample == nullptr || output->receiver == nullptr
		|| output->normal == nullptr || color == nullptr || moments == nullptr || workspace == nullptr
		|| (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0u || params->radiance_cache <= 0.5f
		|| params->gi_width == 0u || params->gi_height == 0u || !validCache(cache_config, cache_state))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	TemporalWorkspace w = layoutTemporalWorkspace(params, workspace);
	if (workspace_bytes < w.bytes)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	GiBindings b = {};
	b.albedo = gbuffer->albedo;
	b.normal = gbuffer->normal;
	b.depth = gbuffer->depth;
	const BvhView bvh = makeBvhView(scene);
	cudaStream_t s = asStream(stream);
	const uint32_t pixels = params->gi_width * params->gi_height;
	primaryQueryKernel<<<gridFor(pixels), 128, 0, s>>>(*params, bvh, b, w.cache.queries);
	int status = restir_cache_query(cache_config, cache_state, reinterpret_cast<const float*>(w.cache.queries), pixels,
		w.cache.values, stream);
	if (status != RESTIR_OK)
	{
		return status;
	}
	giFromCacheKernel<<<gridFor(pixels), 128, 0, s>>>(*params, bvh, b, w.cache.values,
		reinterpret_cast<float4*>(output->sample), reinterpret_cast<float4*>(output->receiver),
		reinterpret_cast<float4*>(output->normal), color, moments);
	return launchStatus();
}

extern "C" int restir_cache_train_frame(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const float* shadow_atlas, const RestirCacheConfig* cache_config, void* cache_state, void* workspace,
	uint64_t workspace_bytes, void* stream)
{
	if (params == nullptr || scene == nullptr || gbuffer == nullptr || shadow_atlas == nullptr || gbuffer->albedo == nullptr
		|| gbuffer->normal == nullptr || gbuffer->depth == nullptr || workspace == nullptr
		|| (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0u || params->radiance_cache <= 0.5f
		|| params->gi_width == 0u || params->gi_height == 0u || !validCache(cache_config, cache_state))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	TemporalWorkspace w = layoutTemporalWorkspace(params, workspace);
	if (workspace_bytes < w.bytes)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const CacheWorkspace& c = w.cache;
	if (c.samples == 0u)
	{
		return RESTIR_OK;
	}
	GiBindings b = {};
	b.albedo = gbuffer->albedo;
	b.normal = gbuffer->normal;
	b.depth = gbuffer->depth;
	b.shadowAtlas = shadow_atlas;
	const BvhView bvh = makeBvhView(scene);
	cudaStream_t s = asStream(stream);
	// Rows [0, first): points on visible surfaces; rows [first, samples): the
	// previous frame's first suffix hits of rows [0, samples - first), so the
	// cache also learns at the points the GI passes query it (the GI samples'
	// surfaces, mostly off screen), which a cache trained on visible surfaces
	// alone only extrapolates to. Each row traces one ray, all in one launch:
	// the frame's ray budget is the same as with visible-surface rows only.
	const uint32_t first = (c.samples + 1u) / 2u;
	const uint32_t second = c.samples - first;
	cudaMemsetAsync(c.trainQueue.claimed, 0, sizeof(uint32_t), s);
	if (second > 0u)
	{
		trainingSecondRaysKernel<<<gridFor(second), 128, 0, s>>>(*params, bvh, b, c, first, second);
	}
	trainingRaysKernel<<<gridFor(first), 128, 0, s>>>(*params, bvh, b, c, first);
	traceQueueKernel<<<persistentBlocks(), 128, 0, s>>>(bvh, c.trainQueue);
	trainingHitsKernel<<<gridFor(c.samples), 128, 0, s>>>(*params, bvh, b, c, 0u, c.samples);
	int status = restir_cache_query(cache_config, cache_state, reinterpret_cast<const float*>(c.hitQueries), c.samples,
		c.hitValues, stream);
	if (status != RESTIR_OK)
	{
		return status;
	}
	trainingTargetsKernel<<<gridFor(c.samples), 128, 0, s>>>(c, params->outlier_clamp);
	status = launchStatus();
	if (status != RESTIR_OK)
	{
		return status;
	}
	return restir_cache_train(cache_config, cache_state, reinterpret_cast<const float*>(c.trainQueries),
		reinterpret_cast<const float*>(c.targets), c.samples, stream);
}
