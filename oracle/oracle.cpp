/*
 * ORACLE (test infrastructure, never linked into the product).
 *
 * CPU restatement of the reference's per-frame passes, one function per
 * pass of include/restir_gpu.h. Each follows its shader line by line:
 *   oracle_grid_clear            shaders/cs_grid_clear.sc:12-21
 *   oracle_grid_insert           shaders/cs_grid_insert.sc:40-73
 *   oracle_gi_temporal           shaders/cs_restir_temporal.sc:57-297
 *   oracle_gi_spatial            shaders/cs_restir_spatial.sc:49-246
 *   oracle_di_temporal           shaders/cs_di_temporal.sc:32-180
 *   oracle_di_spatial            shaders/cs_di_spatial.sc:30-169
 *   oracle_svgf_variance         shaders/fs_svgf_variance.sc:29-76
 *   oracle_svgf_atrous           shaders/fs_svgf_atrous.sc:29-95
 *   oracle_composite             shaders/fs_composite.sc:48-143
 *   oracle_reference_accumulate  shaders/fs_reference.sc:18-25 (in FP64)
 *   oracle_error                 shaders/cs_error.sc:35-93 (in FP64)
 *   oracle_trace                 shaders/bvh.sh:140-319
 * and, for the two raster passes the ABI restates as ray casts:
 *   oracle_gbuffer_primary       shaders/fs_gbuffer.sc:22-95 (targets and
 *                                back-face discard) at pixel centres
 *   oracle_shadow_atlas          shaders/fs_shadow.sc:13-23 at texel centres
 * Pixels are independent except where the shader shares a group (the GI
 * temporal pass's 4x8 group sum), and are spread over std::thread workers
 * (parallel.h).
 */
#include "oracle.h"
#include "oracle_gi.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <vector>

#include "parallel.h"

using namespace oracle;

namespace
{

std::atomic<uint64_t> g_counts[5];
std::atomic<uint32_t> g_status(0);

void resetCounts()
{
	for (auto& c : g_counts)
	{
		c = 0;
	}
}

void addCounts(const Bvh& b, uint64_t screenRays, uint64_t pixels)
{
	g_counts[0] += b.rays;
	g_counts[1] += screenRays;
	g_counts[2] += b.nodeVisits;
	g_counts[3] += b.triangleTests;
	g_counts[4] += pixels;
}

Bvh makeBvh(const RestirScene* _scene)
{
	Bvh b;
	if (_scene)
	{
		b.data = _scene->bvh;
		b.nodeCount = int(_scene->node_count);
		b.triangleOffset = int(_scene->triangle_offset);
	}
	b.status = &g_status;
	return b;
}

Grid makeGrid(const RestirParams* _p, const uint32_t* _data, const float* _camera)
{
	Grid g;
	g.minCell = _p->grid_min_cell;
	g.pixelSize = _p->grid_pixel_size;
	g.cellPixels = _p->grid_cell_pixels;
	g.worldSpace = _p->world_space_reuse > 0.5f;
	g.camera = vec3(_camera[0], _camera[1], _camera[2]);
	g.tableSize = _p->grid_table_size;
	g.capacity = _p->grid_cell_capacity;
	g.data = const_cast<uint32_t*>(_data);
	return g;
}

/* The resources a GI pass binds (renderer.cpp:772-802). */
GiPass makeGiPass(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiHistory* history, const float* shadowAtlas, const uint16_t* surfaceLight)
{
	GiPass g;
	g.P = P;
	g.screen.init(P);
	g.shadow.init(P, shadowAtlas);
	g.sky.init(P);
	g.bvh = makeBvh(scene);
	int W = int(P->width), H = int(P->height);
	int w = int(P->gi_width), h = int(P->gi_height);
	g.albedoTex = { gb->albedo, W, H };
	g.normalTex = { gb->normal, W, H };
	g.depthTex = { gb->depth, W, H };
	g.surfaceLight = { surfaceLight, W, H };
	g.historyColor = { history->color, w, h };
	g.historyNormal = { history->normal, w, h };
	g.historyReceiver = { history->receiver, w, h };
	g.giSize = vec2(float(w), float(h));
	g.giTexel = vec2(1.0f / float(w), 1.0f / float(h));
	return g;
}


} // namespace

/* --- BVH ---------------------------------------------------------------- */

extern "C" int oracle_trace(const RestirParams* params, const RestirScene* scene, const float* rays,
	int32_t* hit_triangle, float* hit_distance, uint32_t n, int kind)
{
	(void)params;
	resetCounts();
	Bvh base = makeBvh(scene);
	const int threadCount = threads();
	std::vector<Bvh> perThread(size_t(threadCount), base);
	if (kind == RESTIR_TRACE_ANY_WAVE)
	{
		// Rays 32w .. 32w + 31 are the lanes of wave w.
		const int64_t waves = (int64_t(n) + 31) / 32;
		parallelFor(waves, 16, [&](int64_t wave, int thread)
		{
			Bvh& b = perThread[size_t(thread)];
			const int64_t first = wave * 32;
			const int count = int(std::min<int64_t>(32, int64_t(n) - first));
			vec3 origin[32], direction[32];
			float distance[32];
			int hit[32];
			for (int lane = 0; lane < count; ++lane)
			{
				const float* r = rays + 8 * (first + lane);
				origin[lane] = vec3(r[0], r[1], r[2]);
				direction[lane] = vec3(r[4], r[5], r[6]);
				distance[lane] = r[3];
				hit[lane] = -1;
			}
			if (b.available())
			{
				traceBvhWave(b, count, origin, direction, true, distance, hit);
			}
			for (int lane = 0; lane < count; ++lane)
			{
				hit_triangle[first + lane] = hit[lane];
				hit_distance[first + lane] = distance[lane];
			}
		});
		for (int t = 0; t < threadCount; ++t)
		{
			addCounts(perThread[size_t(t)], 0, 0);
		}
		return RESTIR_OK;
	}
	parallelFor(int64_t(n), 256, [&](int64_t i, int thread)
	{
		Bvh& b = perThread[size_t(thread)];
		const float* r = rays + 8 * i;
		vec3 origin(r[0], r[1], r[2]);
		vec3 direction(r[4], r[5], r[6]);
		float distance = r[3];
		int hit = -1;
		// The queued closest-hit kind differs only in scheduling.
		if (kind == RESTIR_TRACE_CLOSEST || kind == RESTIR_TRACE_CLOSEST_QUEUE)
		{
			hit = traceBvh(b, origin, direction, r[3], false, distance, true);
		}
		else if (kind == RESTIR_TRACE_ANY)
		{
			hit = traceBvh(b, origin, direction, r[3], true, distance, false);
		}
		else if (kind == RESTIR_TRACE_CLOSEST_STACKLESS)
		{
			hit = traceBvh(b, origin, direction, r[3], false, distance, false);
		}
		else
		{
			hit = b.available() ? traceWatertight(b, origin, direction, distance) : -1;
		}
		hit_triangle[i] = hit;
		hit_distance[i] = distance;
	});
	for (int t = 0; t < threadCount; ++t)
	{
		addCounts(perThread[size_t(t)], 0, 0);
	}
	return RESTIR_OK;
}

/* --- primary rays: the G-buffer and the shadow atlas --------------------- */

namespace
{

/* Moeller-Trumbore nearest hit in (0, tmax) among the triangles _accept
 * lets through (the raster passes' ray casts). */
template<typename Accept>
int traceNearestFiltered(const Bvh& b, vec3 _origin, vec3 _direction, float& _distance, Accept _accept)
{
	return traceNearestFirst(b, _origin, _direction, _distance, false,
		[&](int t, float) { return intersectTriangle(_origin, _direction, b.vertex(t, 0), b.vertex(t, 1), b.vertex(t, 2)); },
		_accept);
}

vec3 clipToWorld(const mat4& _inverse, vec3 _clip)
{
	vec4 world = mul(_inverse, vec4(_clip, 1.0f));
	return world.xyz() / world.w;
}

} // namespace

extern "C" int oracle_gbuffer_primary(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb)
{
	Bvh b = makeBvh(scene);
	Screen screen;
	screen.init(P);
	const int W = int(P->width), H = int(P->height);
	const vec3 camera(P->camera_position[0], P->camera_position[1], P->camera_position[2]);
	const vec2 texel(1.0f / float(W), 1.0f / float(H));
parallelFor(int64_t(H), 16, [&](int64_t y_, int)
	{
		int y = int(y_);
		for (int x = 0; x < W; ++x)
		{
			int i = y * W + x;
			vec2 uv = (vec2(float(x), float(y)) + 0.5f) * texel;
			float ndcY = screen.toClipSpaceY(uv.y * 2.0f - 1.0f);
			vec3 nearPoint = clipToWorld(screen.invViewProj, vec3(uv.x * 2.0f - 1.0f, ndcY, 0.0f));
			vec3 farPoint = clipToWorld(screen.invViewProj, vec3(uv.x * 2.0f - 1.0f, ndcY, 1.0f));
			vec3 span = farPoint - nearPoint;
			float rayLength = length(span);
			vec3 direction = span / rayLength;
			float distance_ = rayLength;
			/* fs_gbuffer.sc:45-55: back faces are discarded unless two-sided. */
			int hit = traceNearestFiltered(b, nearPoint, direction, distance_, [&](int t)
			{
				const float* n = scene->triangle_normals + 4 * size_t(t);
				vec3 normal(n[0], n[1], n[2]);
				return n[3] > 0.5f || dot(normal, camera - b.vertex(t, 0)) > 0.0f;
			});
			if (hit < 0)
			{
				storeU8(gb->albedo, i, vec4_splat(0.0f));
				storeU8(gb->normal, i, vec4_splat(0.0f));
				storeH4(gb->emissive, i, vec4_splat(0.0f));
				storeU8(gb->shading_normal, i, vec4_splat(0.0f));
				gb->depth[i] = 1.0f;
				continue;
			}
			vec3 position = nearPoint + direction * distance_;
			vec4 clip = mul(screen.viewProj, vec4(position, 1.0f));
			const float* n = scene->triangle_normals + 4 * size_t(hit);
			vec3 worldNormal = normalize(vec3(n[0], n[1], n[2]));
			vec3 toCamera = normalize(camera - position);
			float facing = dot(worldNormal, camera - b.vertex(hit, 0)) > 0.0f ? 1.0f : -1.0f;
			vec3 normal = worldNormal * facing;
			float normalView = dot(normal, toCamera);
			if (normalView < 0.05f)
			{
				normal = normalize(normal + toCamera * (0.05f - normalView));
			}
			int material = int(b.row(b.triangleOffset + hit * 4).w + 0.5f);
			const float* m = scene->materials + 8 * size_t(material);
			storeU8(gb->albedo, i, vec4(m[0], m[1], m[2], m[3]));
			storeU8(gb->normal, i, vec4(worldNormal * facing * 0.5f + 0.5f, m[7]));
			storeH4(gb->emissive, i, vec4(m[4], m[5], m[6], 1.0f));
			storeU8(gb->shading_normal, i, vec4(normal * 0.5f + 0.5f, 1.0f));
			gb->depth[i] = clip.z / clip.w;
		}
	});
	return RESTIR_OK;
}

extern "C" int oracle_shadow_atlas(const RestirParams* P, const RestirScene* scene, float* atlas)
{
	Bvh b = makeBvh(scene);
	const int f = int(P->shadow_face_size);
	const int W = 3 * f, H = 2 * f;
	const vec3 light(P->light_position[0], P->light_position[1], P->light_position[2]);
	const bool originBottomLeft = P->origin_bottom_left > 0.5f;
	const float inverseFace = 1.0f / float(f);
parallelFor(int64_t(H), 8, [&](int64_t y_, int)
	{
		int y = int(y_);
		for (int x = 0; x < W; ++x)
		{
			int column = x / f;
			int row = y / f;
			int face = column + 3 * (originBottomLeft ? 1 - row : row);
			vec2 local = (vec2(float(x - column * f), float(y - row * f)) + 0.5f) * inverseFace;
			float ndcX = local.x * 2.0f - 1.0f;
			float ndcY = originBottomLeft ? local.y * 2.0f - 1.0f : 1.0f - local.y * 2.0f;
			mat4 inverse = make_mat4(P->shadow_inv_view_proj[face]);
			vec3 nearPoint = clipToWorld(inverse, vec3(ndcX, ndcY, 0.0f));
			vec3 farPoint = clipToWorld(inverse, vec3(ndcX, ndcY, 1.0f));
			vec3 span = farPoint - nearPoint;
			float rayLength = length(span);
			vec3 direction = span / rayLength;
			float distance_ = rayLength;
			int hit = traceNearestFiltered(b, nearPoint, direction, distance_, [](int) { return true; });
			float value = 1.0f;
			if (hit >= 0)
			{
				value = length(nearPoint + direction * distance_ - light) / P->shadow_far;
			}
			atlas[y * W + x] = value;
		}
	});
	return RESTIR_OK;
}

/* --- hash grid ---------------------------------------------------------- */

extern "C" int oracle_grid_clear(const RestirParams* P, uint32_t* grid)
{
	size_t T = P->grid_table_size;
	std::fill(grid, grid + 2 * T, 0u);
	std::fill(grid + 2 * T, grid + (2 + P->grid_cell_capacity) * T, 0xffffffffu);
	return RESTIR_OK;
}

extern "C" int oracle_grid_insert(const RestirParams* P, const RestirGBuffer* gb, uint32_t* grid)
{
	Screen screen;
	screen.init(P);
	Grid g = makeGrid(P, grid, P->camera_position);
	const int W = int(P->width), H = int(P->height);
	const int w = int(P->gi_width), h = int(P->gi_height);
	TexF1 depthTex = { gb->depth, W, H };
	TexU8 normalTex = { gb->normal, W, H };
	const vec2 texel(1.0f / float(w), 1.0f / float(h));
	/* Keys in parallel, insertion in pixel order (the deterministic mode). */
	std::vector<uint32_t> slots(size_t(w) * h), checksums(size_t(w) * h, 0u);
parallelFor(int64_t(h), 64, [&](int64_t y_, int)
	{
		int y = int(y_);
		for (int x = 0; x < w; ++x)
		{
			vec2 uv = (vec2(float(x), float(y)) + 0.5f) * texel;
			float depth = depthTex.sample(uv);
			if (depth >= kSkyDepth)
			{
				continue;
			}
			vec3 position = screen.reconstructWorldPosition(uv, depth);
			vec3 normal = normalize(normalTex.sample(uv).xyz() * 2.0f - 1.0f);
			uint rng = pcg(uint(x) + pcg(uint(y) + pcg(uint(P->frame_index) ^ 0x5bd1e995u)));
			float cellSize = g.cellSize(position);
			float r0 = nextRandom(rng);
			float r1 = nextRandom(rng);
			vec3 jittered = Grid::jitter(position, normal, cellSize, r0, r1);
			uint slot, checksum;
			g.key(jittered, normal, cellSize, slot, checksum);
			slots[size_t(y) * w + x] = slot;
			checksums[size_t(y) * w + x] = checksum;
		}
	});
	for (size_t i = 0; i < slots.size(); ++i)
	{
		if (checksums[i] != 0u && !g.insert(slots[i], checksums[i], uint(i)))
		{
			g_status |= 2u;
		}
	}
	return RESTIR_OK;
}

/* --- ReSTIR GI temporal (cs_restir_temporal.sc) -------------------------- */

namespace
{

struct TemporalThread
{
	bool inside = false, working = false;
	vec3 position, normal, albedo;
	vec2 previousUv;
	bool historyValid = false;
	Reservoir canonical;
	float canonicalWeight = 0.0f;
	PairwiseMis mis;
	float combinedWeight = 0.0f;
	float estimate = 0.0f;
};

} // namespace

/* The largest reservoir weight the temporal pass with the radiance cache
 * stores (restir_gi_temporal_cached's cap). */
static const float kCachedReservoirWeightCap = 64.0f;

/* cache_values (half4 per slot, null for the plain pass): the radiance
 * cache's values for the candidates (slot pixel * initial_candidates + k)
 * then last frame's reservoirs (slot GI pixels * initial_candidates + pixel),
 * standing in for previousIndirect as in restir_gi_temporal_cached. */
extern "C" int oracle_gi_temporal_cached(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, const RestirGiReservoirs* out, const uint16_t* cache_values)
{
	resetCounts();
	GiPass base = makeGiPass(P, scene, gb, history, shadow_atlas, surface_light);
	base.sharedStack = true;
	base.grid = makeGrid(P, previous_grid, P->prev_camera_position);
	const int w = int(P->gi_width), h = int(P->gi_height);
	base.cache = cache_values;
	base.cacheNeighbourBase = w * h * P->initial_candidates;
	TexF4 historySample = { history->sample, w, h };
	const int groupsX = (w + 3) / 4, groupsY = (h + 7) / 8;
const int threadCount = threads();
	std::vector<GiPass> gs_(size_t(threadCount), base);
	std::vector<uint64_t> screenRayss_(size_t(threadCount), 0);
	std::vector<uint64_t> pixelss_(size_t(threadCount), 0);
	parallelFor(int64_t(groupsX * groupsY), 4, [&](int64_t group_, int thread_)
	{
		GiPass& g = gs_[size_t(thread_)];
		uint64_t& screenRays = screenRayss_[size_t(thread_)];
		uint64_t& pixels = pixelss_[size_t(thread_)];
		int group = int(group_);
			TemporalThread th[32];
			for (int thread = 0; thread < 32; ++thread)
			{
				TemporalThread& t = th[thread];
				int px = (group % groupsX) * 4 + (thread & 3);
				int py = (group / groupsX) * 8 + (thread >> 2);
				t.inside = px < w && py < h;
				vec2 uv = (vec2(float(px), float(py)) + 0.5f) * g.giTexel;
				float depth = t.inside ? g.depthTex.sample(uv) : 1.0f;
				t.working = t.inside && depth < kSkyDepth;
				pixels += t.working ? 1 : 0;
				t.position = g.reconstructWorldPosition(uv, depth);
				t.normal = g.decodeNormal(uv);
				t.albedo = g.diffuseAlbedo(uv);
				vec3 rayOrigin = t.position + t.normal * g.kRayBias();
				vec2 giPixelCoord = g.giPixel(uv);
				uint rng = pcg(uint(giPixelCoord.x) + pcg(uint(giPixelCoord.y) + pcg(uint(P->frame_index))));

				Reservoir& canonical = t.canonical;
				for (int sampleIndex = 0; sampleIndex < P->initial_candidates; ++sampleIndex)
				{
					float random0 = nextRandom(rng);
					float random1 = nextRandom(rng);
					float randomSelect = nextRandom(rng);
					vec3 direction = GiPass::cosineHemisphere(t.normal, random0, random1);
					canonical.count += 1.0f;
					vec3 hitPosition = vec3_splat(0.0f);
					float hitId = 0.0f;
					bool hit = false;
					if (t.working && P->ray_mode != RESTIR_RAY_MODE_BVH)
					{
						++screenRays;
						hit = g.traceScreenSpaceRay(rayOrigin, direction, g.kMaxRayDistance(), hitPosition);
					}
					bool needBvh = t.working && !hit && P->ray_mode != RESTIR_RAY_MODE_SCREEN;
					if (needBvh)
					{
						float queueDistance;
						int queueTriangle = traceBvh(g.bvh, rayOrigin, direction, g.kMaxBvhRayDistance(), false, queueDistance, true);
						if (queueTriangle >= 0)
						{
							hit = true;
							hitPosition = rayOrigin + direction * queueDistance;
							hitId = g.encodeSampleId(queueTriangle, direction);
						}
						else if (g.sky.enabled())
						{
							hit = true;
							hitPosition = direction;
							hitId = kSkySampleId;
						}
					}
					vec3 contribution = vec3_splat(0.0f);
					vec3 hitNormal = vec3_splat(0.0f);
					bool evaluated = false;
					if (hit)
					{
						const int cacheSlot = g.cache != nullptr ? (py * w + px) * P->initial_candidates + sampleIndex : -1;
						evaluated = g.evaluateSample(t.position, t.normal, t.albedo, hitPosition, hitId, contribution, hitNormal,
							cacheSlot);
					}
					if (evaluated)
					{
						float target = luminance(contribution);
						float sourcePdf = dot(t.normal, direction) / kPi;
						if (!isSkySample(hitId))
						{
							vec3 fromReceiver = hitPosition - t.position;
							vec3 fromOrigin = hitPosition - rayOrigin;
							float receiverSquared = max(dot(fromReceiver, fromReceiver), g.kMinDistanceSquared() * 0.01f);
							float originSquared = max(dot(fromOrigin, fromOrigin), g.kMinDistanceSquared() * 0.01f);
							float hitCosineOrigin = max(-dot(hitNormal, fromOrigin), 0.0f) * inversesqrt(originSquared);
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

				t.canonicalWeight = canonical.target > 0.000001f
					? canonical.weightSum / (canonical.count * canonical.target)
					: 0.0f;
				t.historyValid = P->history_valid > 0.5f;
				t.previousUv = vec2_splat(0.0f);
				vec4 clipPrevious = mul(g.screen.prevViewProj, vec4(t.position, 1.0f));
				if (clipPrevious.w > 0.0001f)
				{
					t.previousUv = g.screen.clipToUv(clipPrevious);
				}
				float radius = g.reuseRadius(t.position);
				t.mis = g.beginPairwiseMis(t.position, t.normal, canonical, canonical.count, P->temporal_taps);
				t.combinedWeight = 0.0f;
				if (t.working)
				{
					for (int tapIndex = 0; tapIndex < P->temporal_taps; ++tapIndex)
					{
						float random0 = nextRandom(rng);
						float random1 = nextRandom(rng);
						float random2 = nextRandom(rng);
						float randomSelect = nextRandom(rng);
						vec2 historyUv = vec2_splat(-1.0f);
						if (t.historyValid)
						{
							if (g.grid.worldSpace)
							{
								uint entry = g.grid.pickEntry(t.position, t.normal, random0, random1, random2);
								if (entry != kGridInvalid)
								{
									historyUv = g.giPixelUv(entry);
								}
							}
							else if (tapIndex == 0 && clipPrevious.w > 0.0001f)
							{
								historyUv = t.previousUv;
							}
						}
						NeighbourReservoir neighbour;
						if (!isOnScreen(historyUv)
							|| !g.acceptNeighbour(historySample.sample(historyUv), g.historyReceiver.sample(historyUv),
								g.historyNormal.sample(historyUv), t.position, t.normal, radius, neighbour))
						{
							GiPass::skipNeighbour(t.mis);
							continue;
						}
						neighbour.cacheSlot = g.cache != nullptr ? g.cacheNeighbourBase + texelIndex(historyUv, w, h) : -1;
						g.addNeighbour(t.mis, t.position, t.normal, t.albedo, neighbour, randomSelect);
					}
					t.combinedWeight = g.finishPairwiseMis(t.mis, t.position, t.normal, canonical, t.canonicalWeight, nextRandom(rng));
				}
				t.estimate = t.working ? t.mis.combined.target * t.combinedWeight : 0.0f;
			}

			/* groupSum (compute.sh:356-390): a tree over gl_LocalInvocationIndex. */
			vec2 sums[32];
			for (int i = 0; i < 32; ++i)
			{
				sums[i] = vec2(th[i].estimate, th[i].working ? 1.0f : 0.0f);
			}
			for (int stride = 16; stride > 0; stride >>= 1)
			{
				for (int i = 0; i < stride; ++i)
				{
					sums[i] += sums[i + stride];
				}
			}
			vec2 tileSum = sums[0];
			float tileMean = tileSum.x / max(tileSum.y, 1.0f);

			for (int thread = 0; thread < 32; ++thread)
			{
				TemporalThread& t = th[thread];
				if (t.working && P->boiling_filter > 0.0f && t.combinedWeight > 0.0f)
				{
					float reference = t.canonical.target * t.canonicalWeight;
					vec3 historyColor;
					if (t.historyValid && g.historyIrradiance(t.previousUv, t.position, t.normal, historyColor))
					{
						reference = max(reference, luminance(historyColor * t.albedo));
					}
					else
					{
						reference = max(reference, tileMean);
					}
					float limit = P->boiling_filter * reference;
					if (t.estimate > limit)
					{
						t.combinedWeight *= limit / t.estimate;
					}
				}
				if (g.cache != nullptr)
				{
					// The form with the radiance cache (no reference counterpart) caps
					// the stored reservoir weight, as restir_gi_temporal_cached does.
					t.combinedWeight = fminf(t.combinedWeight, kCachedReservoirWeightCap);
				}
				if (t.inside)
				{
					int px = (group % groupsX) * 4 + (thread & 3);
					int py = (group / groupsX) * 8 + (thread >> 2);
					int i = py * w + px;
					storeF4(out->sample, i, t.working ? vec4(t.mis.combined.position, t.mis.totalCount) : vec4_splat(0.0f));
					storeF4(out->receiver, i, t.working ? vec4(t.position, t.combinedWeight) : vec4_splat(0.0f));
					storeF4(out->normal, i, t.working ? vec4(t.normal, t.mis.combined.id) : vec4_splat(0.0f));
				}
			}
		});
	for (int t_ = 0; t_ < threadCount; ++t_)
	{
		addCounts(gs_[size_t(t_)].bvh, screenRayss_[size_t(t_)], pixelss_[size_t(t_)]);
	}
	return RESTIR_OK;
}

extern "C" int oracle_gi_temporal(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, const RestirGiReservoirs* out)
{
	return oracle_gi_temporal_cached(P, scene, gb, history, previous_grid, shadow_atlas, surface_light, out, nullptr);
}

/* --- ReSTIR GI spatial (cs_restir_spatial.sc) ---------------------------- */

/* cache_values: the radiance cache's values for this frame's reservoirs
 * (slot = pixel), as in restir_gi_spatial_cached; null for the plain pass. */
extern "C" int oracle_gi_spatial_cached(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiReservoirs* current, const uint32_t* current_grid, const RestirGiHistory* history,
	const float* shadow_atlas, const uint16_t* surface_light, uint16_t* color_out, uint16_t* moments_out,
	const uint16_t* cache_values)
{
	resetCounts();
	GiPass base = makeGiPass(P, scene, gb, history, shadow_atlas, surface_light);
	base.sharedStack = false;
	base.grid = makeGrid(P, current_grid, P->camera_position);
	const int w = int(P->gi_width), h = int(P->gi_height);
	base.cache = cache_values;
	base.cacheNeighbourBase = 0;
	TexF4 reservoirSample = { current->sample, w, h };
	TexF4 reservoirReceiver = { current->receiver, w, h };
	TexF4 reservoirNormal = { current->normal, w, h };
	TexH4 historyMoments = { history->moments, w, h };
const int threadCount = threads();
	std::vector<GiPass> gs_(size_t(threadCount), base);
	std::vector<uint64_t> pixelss_(size_t(threadCount), 0);
	parallelFor(int64_t(h), 4, [&](int64_t py_, int thread_)
	{
		GiPass& g = gs_[size_t(thread_)];
		uint64_t& pixels = pixelss_[size_t(thread_)];
		int py = int(py_);
			for (int px = 0; px < w; ++px)
			{
				int outIndex = py * w + px;
				vec2 v_texcoord0 = (vec2(float(px), float(py)) + 0.5f) * g.giTexel;
				float depth = g.depthTex.sample(v_texcoord0);
				if (depth >= kSkyDepth)
				{
					storeH4(color_out, outIndex, vec4_splat(0.0f));
					storeH4(moments_out, outIndex, vec4_splat(0.0f));
					continue;
				}
				++pixels;
				vec3 position = g.reconstructWorldPosition(v_texcoord0, depth);
				vec3 normal = g.decodeNormal(v_texcoord0);
				vec3 albedo = g.diffuseAlbedo(v_texcoord0);
				vec2 pixel = g.giPixel(v_texcoord0);
				uint pixelIndex = g.giPixelIndex(pixel);
				uint rng = pcg(uint(pixel.x) + pcg(uint(pixel.y) + pcg(uint(P->frame_index) ^ 0x68e31da4u)));

				vec4 ownSample = reservoirSample.sample(v_texcoord0);
				float canonicalWeight = reservoirReceiver.sample(v_texcoord0).w;
				float canonicalCount = max(min(ownSample.w, 20.0f), 1.0f);
				Reservoir canonical;
				vec3 canonicalContribution = vec3_splat(0.0f);
				vec3 canonicalNormal = vec3(0.0f, 0.0f, 1.0f);
				bool canonicalValid = false;
				if (canonicalWeight > 0.0f)
				{
					canonicalValid = g.evaluateSample(position, normal, albedo, ownSample.xyz(),
						reservoirNormal.sample(v_texcoord0).w, canonicalContribution, canonicalNormal,
						g.cache != nullptr ? texelIndex(v_texcoord0, w, h) : -1);
				}
				if (canonicalValid)
				{
					canonical.contribution = canonicalContribution;
					canonical.position = ownSample.xyz();
					canonical.normal = canonicalNormal;
					canonical.id = reservoirNormal.sample(v_texcoord0).w;
					canonical.target = luminance(canonicalContribution);
				}

				float radius = g.reuseRadius(position);
				PairwiseMis mis = g.beginPairwiseMis(position, normal, canonical, canonicalCount, P->spatial_taps);
				for (int tapIndex = 0; tapIndex < P->spatial_taps; ++tapIndex)
				{
					float random0 = nextRandom(rng);
					float random1 = nextRandom(rng);
					float random2 = nextRandom(rng);
					float randomSelect = nextRandom(rng);
					vec2 neighbourUv = vec2_splat(-1.0f);
					if (g.grid.worldSpace)
					{
						uint entry = g.grid.pickEntry(position, normal, random0, random1, random2);
						if (entry != kGridInvalid && entry != pixelIndex)
						{
							neighbourUv = g.giPixelUv(entry);
						}
					}
					else
					{
						float diskRadius = 12.0f * sqrt(random0);
						float angle = 2.0f * kPi * random1;
						vec2 neighbourPixel = floor(pixel + vec2(cos(angle), sin(angle)) * diskRadius);
						if (neighbourPixel.x != pixel.x || neighbourPixel.y != pixel.y)
						{
							neighbourUv = (neighbourPixel + 0.5f) * g.giTexel;
						}
					}
					NeighbourReservoir neighbour;
					if (!isOnScreen(neighbourUv)
						|| !g.acceptNeighbour(reservoirSample.sample(neighbourUv), reservoirReceiver.sample(neighbourUv),
							reservoirNormal.sample(neighbourUv), position, normal, radius, neighbour))
					{
						GiPass::skipNeighbour(mis);
						continue;
					}
					neighbour.cacheSlot = g.cache != nullptr ? texelIndex(neighbourUv, w, h) : -1;
					g.addNeighbour(mis, position, normal, albedo, neighbour, randomSelect);
				}

				float combinedWeight = g.finishPairwiseMis(mis, position, normal, canonical, canonicalWeight, nextRandom(rng));
				vec3 estimate = mis.combined.contribution * combinedWeight;
				if (P->outlier_clamp > 0.0f)
				{
					estimate = min(estimate, vec3_splat(P->outlier_clamp));
				}
				vec3 irradiance = estimate / max(albedo, vec3_splat(0.001f));
				float irradianceLuminance = luminance(irradiance);

				vec3 previousColor = vec3_splat(0.0f);
				vec3 previousMoments = vec3_splat(0.0f);
				vec4 clipPrevious = mul(g.screen.prevViewProj, vec4(position, 1.0f));
				if (P->history_valid > 0.5f && clipPrevious.w > 0.0001f)
				{
					/* reprojectHistory (cs_restir_spatial.sc:49-93) */
					vec2 previousUv = g.screen.clipToUv(clipPrevious);
					vec3 c = vec3_splat(0.0f);
					vec3 m = vec3_splat(0.0f);
					vec2 texelCoord = previousUv * g.giSize - 0.5f;
					vec2 baseCoord = floor(texelCoord);
					vec2 blend = texelCoord - baseCoord;
					float weightSum = 0.0f;
					for (int tapIndex = 0; tapIndex < 4; ++tapIndex)
					{
						vec2 offset = vec2(float(tapIndex & 1), float(tapIndex >> 1));
						vec2 uv = (baseCoord + offset + 0.5f) * g.giTexel;
						if (!isOnScreen(uv))
						{
							continue;
						}
						if (!g.sameHistorySurface(uv, position, normal))
						{
							continue;
						}
						vec2 bilinear = mix(vec2_splat(1.0f) - blend, blend, offset);
						float weight = bilinear.x * bilinear.y;
						c += g.historyColor.sample(uv).xyz() * weight;
						m += historyMoments.sample(uv).xyz() * weight;
						weightSum += weight;
					}
					if (weightSum < 0.01f)
					{
						c = vec3_splat(0.0f);
						m = vec3_splat(0.0f);
					}
					else
					{
						c /= weightSum;
						m /= weightSum;
					}
					previousColor = c;
					previousMoments = m;
				}

				float historyLength = min(previousMoments.z + 1.0f, 16.0f);
				float blendWeight = 1.0f / historyLength;
				vec3 color = mix(previousColor, irradiance, blendWeight);
				vec2 moments = mix(vec2(previousMoments.x, previousMoments.y),
					vec2(irradianceLuminance, irradianceLuminance * irradianceLuminance), blendWeight);
				storeH4(color_out, outIndex, vec4(color, historyLength));
				storeH4(moments_out, outIndex, vec4(moments.x, moments.y, historyLength, 0.0f));
			}
		});
	for (int t_ = 0; t_ < threadCount; ++t_)
	{
		addCounts(gs_[size_t(t_)].bvh, 0, pixelss_[size_t(t_)]);
	}
	return RESTIR_OK;
}

extern "C" int oracle_gi_spatial(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiReservoirs* current, const uint32_t* current_grid, const RestirGiHistory* history,
	const float* shadow_atlas, const uint16_t* surface_light, uint16_t* color_out, uint16_t* moments_out)
{
	return oracle_gi_spatial_cached(P, scene, gb, current, current_grid, history, shadow_atlas, surface_light, color_out,
		moments_out, nullptr);
}

/* --- ReSTIR DI (di.sh, cs_di_temporal.sc, cs_di_spatial.sc) -------------- */

namespace
{

struct Surface
{
	vec3 position;
	vec3 normal;
	vec3 surfaceNormal;
	vec3 albedo;
	float roughness = 0.0f;
	float metallic = 0.0f;
	vec3 eye;
	bool valid = false;
};

/* brdf.sh:14-62 */
float distributionGGX(vec3 _normal, vec3 _halfway, float _roughness)
{
	float alpha = _roughness * _roughness;
	float alphaSquared = alpha * alpha;
	float normalHalfway = max(dot(_normal, _halfway), 0.0f);
	float denominator = normalHalfway * normalHalfway * (alphaSquared - 1.0f) + 1.0f;
	return alphaSquared / max(kPi * denominator * denominator, 0.0001f);
}

float geometrySchlickGGX(float _normalDirection, float _roughness)
{
	float k = (_roughness + 1.0f) * (_roughness + 1.0f) / 8.0f;
	return _normalDirection / max(_normalDirection * (1.0f - k) + k, 0.0001f);
}

vec3 fresnelSchlick(vec3 _halfway, vec3 _viewDirection, vec3 _f0)
{
	float cosine = clamp(dot(_halfway, _viewDirection), 0.0f, 1.0f);
	return _f0 + (vec3_splat(1.0f) - _f0) * rn_pow5(1.0f - cosine);
}

void evaluateBrdf(vec3 _normal, vec3 _viewDirection, vec3 _lightDirection, vec3 _albedo, float _roughness,
	float _metallic, vec3& _diffuse, vec3& _specular)
{
	float normalLight = max(dot(_normal, _lightDirection), 0.0f);
	float normalView = max(dot(_normal, _viewDirection), 0.0f);
	vec3 halfway = normalize(_viewDirection + _lightDirection);
	vec3 f0 = mix(vec3_splat(0.04f), _albedo, _metallic);
	vec3 fresnel = fresnelSchlick(halfway, _viewDirection, f0);
	float roughness = max(_roughness, 0.05f);
	float distribution = distributionGGX(_normal, halfway, roughness);
	float geometry = geometrySchlickGGX(normalLight, roughness) * geometrySchlickGGX(normalView, roughness);
	_specular = distribution * geometry * fresnel / max(4.0f * normalLight * normalView, 0.001f) * normalLight;
	_diffuse = (vec3_splat(1.0f) - fresnel) * (1.0f - _metallic) * _albedo / kPi * normalLight;
}

struct DiPass
{
	const RestirParams* P = nullptr;
	Screen screen;
	Bvh bvh;
	const float* lights = nullptr;
	TexU8 albedoTex, normalTex, shadingNormalTex;
	TexF1 depthTex;
	vec3 camera;
	vec2 texel;

	float s() const { return P->scene_scale; }
	float kDiRayBias() const { return 0.01f * s(); }
	float kDiReceiverRadius() const { return 0.1f * s(); }
	float kDiReceiverPlane() const { return 0.03f * s(); }
	float kDiMinDistanceSquared() const { return 0.0001f * s() * s(); }

	Surface loadSurface(vec2 _uv) const
	{
		Surface surface;
		float depth = depthTex.sample(_uv);
		vec4 albedoRoughness = albedoTex.sample(_uv);
		vec4 normalMetallic = normalTex.sample(_uv);
		surface.valid = depth < kSkyDepth;
		surface.position = screen.reconstructWorldPosition(_uv, min(depth, kSkyDepth));
		surface.surfaceNormal = normalize(normalMetallic.xyz() * 2.0f - 1.0f);
		surface.normal = normalize(shadingNormalTex.sample(_uv).xyz() * 2.0f - 1.0f);
		surface.albedo = albedoRoughness.xyz();
		surface.roughness = albedoRoughness.w;
		surface.metallic = normalMetallic.w;
		surface.eye = camera;
		return surface;
	}

	int lightCount() const { return P->di_light_count; }
	vec4 lightData(int _light, int _row) const
	{
		const float* q = lights + 4 * size_t(_light * 4 + _row);
		return vec4(q[0], q[1], q[2], q[3]);
	}
	bool isPointLight(int _light) const { return lightData(_light, 0).w > 0.5f; }

	int selectLight(float _random, float& _pmf) const
	{
		int low = 0;
		int high = lightCount() - 1;
		for (int step = 0; step < 24 && low < high; ++step)
		{
			int middle = (low + high) >> 1;
			if (lightData(middle, 2).w < _random)
			{
				low = middle + 1;
			}
			else
			{
				high = middle;
			}
		}
		_pmf = lightData(low, 3).w;
		return low;
	}

	float triangleArea(int _light) const
	{
		vec3 v0 = lightData(_light, 0).xyz();
		return 0.5f * length(cross(lightData(_light, 1).xyz() - v0, lightData(_light, 2).xyz() - v0));
	}

	vec3 sampleLightPoint(int _light, float _random0, float _random1, float& _density) const
	{
		vec3 v0 = lightData(_light, 0).xyz();
		if (isPointLight(_light))
		{
			_density = 1.0f;
			return v0;
		}
		float root = sqrt(_random0);
		float u = 1.0f - root;
		float v = _random1 * root;
		_density = 1.0f / max(triangleArea(_light), 1e-12f);
		return v0 + (lightData(_light, 1).xyz() - v0) * u + (lightData(_light, 2).xyz() - v0) * v;
	}

	void evaluateLightSample(const Surface& _surface, int _light, vec3 _point, vec3& _diffuse, vec3& _specular) const
	{
		_diffuse = vec3_splat(0.0f);
		_specular = vec3_splat(0.0f);
		if (_light < 0 || _light >= lightCount())
		{
			return;
		}
		vec3 toLight = _point - _surface.position;
		float distanceSquared = max(dot(toLight, toLight), kDiMinDistanceSquared());
		vec3 direction = toLight * inversesqrt(distanceSquared);
		if (dot(_surface.surfaceNormal, direction) <= 0.0f)
		{
			return;
		}
		vec3 radiance = lightData(_light, 3).xyz() / distanceSquared;
		if (!isPointLight(_light))
		{
			vec3 v0 = lightData(_light, 0).xyz();
			vec3 lightNormal = normalize(cross(lightData(_light, 1).xyz() - v0, lightData(_light, 2).xyz() - v0));
			radiance *= abs(dot(lightNormal, direction));
		}
		vec3 diffuse, specular;
		evaluateBrdf(_surface.normal, normalize(_surface.eye - _surface.position), direction,
			_surface.albedo, _surface.roughness, _surface.metallic, diffuse, specular);
		_diffuse = diffuse * radiance;
		_specular = specular * radiance;
	}

	float lightTarget(const Surface& _surface, int _light, vec3 _point) const
	{
		vec3 diffuse, specular;
		evaluateLightSample(_surface, _light, _point, diffuse, specular);
		return luminance(diffuse + specular);
	}

	bool lightVisible(const Surface& _surface, vec3 _point) const
	{
		vec3 origin = _surface.position + _surface.surfaceNormal * kDiRayBias();
		vec3 toPoint = _point - origin;
		float pointDistance = length(toPoint);
		float occluderDistance = 0.0f;
		return traceBvh(bvh, origin, toPoint / max(pointDistance, 0.0001f),
			pointDistance * 0.999f - kDiRayBias(), true, occluderDistance, false) < 0;
	}

	bool sameSurface(vec3 _position, vec3 _normal, vec3 _otherPosition, vec3 _otherNormal, float _radius) const
	{
		vec3 offset = _otherPosition - _position;
		return dot(_otherNormal, _otherNormal) > 0.5f
			&& dot(offset, offset) <= _radius * _radius
			&& abs(dot(offset, _normal)) <= kDiReceiverPlane()
			&& dot(normalize(_otherNormal), _normal) >= 0.9f;
	}
};

DiPass makeDiPass(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb)
{
	DiPass d;
	d.P = P;
	d.screen.init(P);
	d.bvh = makeBvh(scene);
	d.lights = scene->lights;
	int W = int(P->width), H = int(P->height);
	d.albedoTex = { gb->albedo, W, H };
	d.normalTex = { gb->normal, W, H };
	d.shadingNormalTex = { gb->shading_normal, W, H };
	d.depthTex = { gb->depth, W, H };
	d.camera = vec3(P->camera_position[0], P->camera_position[1], P->camera_position[2]);
	d.texel = vec2(1.0f / float(W), 1.0f / float(H));
	return d;
}

} // namespace

extern "C" int oracle_di_temporal(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirDiReservoirs* previous, const RestirDiReservoirs* out)
{
	resetCounts();
	DiPass base = makeDiPass(P, scene, gb);
	const int W = int(P->width), H = int(P->height);
	TexF4 previousSample = { previous->sample, W, H };
	TexF4 previousReceiver = { previous->receiver, W, H };
	TexH4 previousNormal = { previous->normal, W, H };
	const vec3 previousEye(P->prev_camera_position[0], P->prev_camera_position[1], P->prev_camera_position[2]);
const int threadCount = threads();
	std::vector<DiPass> ds_(size_t(threadCount), base);
	std::vector<uint64_t> pixelss_(size_t(threadCount), 0);
	parallelFor(int64_t(H), 4, [&](int64_t py_, int thread_)
	{
		DiPass& d = ds_[size_t(thread_)];
		uint64_t& pixels = pixelss_[size_t(thread_)];
		int py = int(py_);
			for (int px = 0; px < W; ++px)
			{
				int i = py * W + px;
				vec2 v_texcoord0 = (vec2(float(px), float(py)) + 0.5f) * d.texel;
				Surface surface = d.loadSurface(v_texcoord0);
				if (!surface.valid || d.lightCount() == 0)
				{
					storeF4(out->sample, i, vec4(0.0f, 0.0f, 0.0f, -1.0f));
					storeF4(out->receiver, i, vec4_splat(0.0f));
					storeH4(out->normal, i, vec4_splat(0.0f));
					continue;
				}
				++pixels;
				uint rng = pcg(uint(px) + pcg(uint(py) + pcg(uint(P->frame_index) ^ 0x3c6ef372u)));
				int candidates = P->di_candidates;
				float weightSum = 0.0f;
				vec3 chosenPoint = vec3_splat(0.0f);
				int chosenLight = -1;
				float chosenTarget = 0.0f;
				for (int candidate = 0; candidate < candidates; ++candidate)
				{
					float pmf;
					int light = d.selectLight(nextRandom(rng), pmf);
					float density;
					float r0 = nextRandom(rng);
					float r1 = nextRandom(rng);
					vec3 lightPoint = d.sampleLightPoint(light, r0, r1, density);
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
				float canonicalCount = float(candidates);
				float canonicalWeight = chosenTarget > 0.0f ? weightSum / (canonicalCount * chosenTarget) : 0.0f;
				vec3 canonicalPoint = chosenPoint;
				int canonicalLight = chosenLight;
				float canonicalTarget = chosenTarget;

				float temporalCount = 0.0f;
				float temporalWeight = 0.0f;
				vec3 temporalPoint = vec3_splat(0.0f);
				int temporalLight = -1;
				Surface prev = surface;
				vec4 clip = mul(d.screen.prevViewProj, vec4(surface.position, 1.0f));
				if (P->di_history_valid > 0.5f && clip.w > 0.0001f)
				{
					vec2 uv = vec2(clip.x, P->origin_bottom_left > 0.5f ? clip.y : -clip.y) / clip.w * 0.5f + 0.5f;
					if (uv.x > 0.0f && uv.x < 1.0f && uv.y > 0.0f && uv.y < 1.0f)
					{
						vec4 sampleData = previousSample.sample(uv);
						vec4 receiver = previousReceiver.sample(uv);
						vec4 normal = previousNormal.sample(uv);
						int light = int(sampleData.w + 0.5f);
						if (sampleData.w >= 0.0f && light < d.lightCount()
							&& d.sameSurface(surface.position, surface.normal, receiver.xyz(), normal.xyz(), d.kDiReceiverRadius()))
						{
							temporalCount = min(normal.w, 20.0f);
							temporalWeight = receiver.w;
							temporalPoint = sampleData.xyz();
							temporalLight = light;
							prev.position = receiver.xyz();
							prev.normal = normalize(normal.xyz());
							prev.eye = previousEye;
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
					float weight = denominator > 0.0f
						? temporalCount * previousTarget / denominator * target * temporalWeight
						: 0.0f;
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
				storeF4(out->sample, i, vec4(chosenPoint, float(chosenLight)));
				storeF4(out->receiver, i, vec4(surface.position, combinedWeight));
				storeH4(out->normal, i, vec4(surface.normal, canonicalCount + temporalCount));
			}
		});
	for (int t_ = 0; t_ < threadCount; ++t_)
	{
		addCounts(ds_[size_t(t_)].bvh, 0, pixelss_[size_t(t_)]);
	}
	return RESTIR_OK;
}

extern "C" int oracle_di_spatial(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirDiReservoirs* current, uint16_t* diffuse_out, uint16_t* specular_out)
{
	resetCounts();
	DiPass base = makeDiPass(P, scene, gb);
	const int W = int(P->width), H = int(P->height);
	TexF4 reservoirSample = { current->sample, W, H };
	TexF4 reservoirReceiver = { current->receiver, W, H };
	TexH4 reservoirNormal = { current->normal, W, H };
const int threadCount = threads();
	std::vector<DiPass> ds_(size_t(threadCount), base);
	std::vector<uint64_t> pixelss_(size_t(threadCount), 0);
	parallelFor(int64_t(H), 4, [&](int64_t py_, int thread_)
	{
		DiPass& d = ds_[size_t(thread_)];
		uint64_t& pixels = pixelss_[size_t(thread_)];
		int py = int(py_);
			for (int px = 0; px < W; ++px)
			{
				int i = py * W + px;
				vec2 v_texcoord0 = (vec2(float(px), float(py)) + 0.5f) * d.texel;
				Surface surface = d.loadSurface(v_texcoord0);
				vec4 ownSample = reservoirSample.sample(v_texcoord0);
				vec4 ownReceiver = reservoirReceiver.sample(v_texcoord0);
				vec4 ownNormal = reservoirNormal.sample(v_texcoord0);
				if (!surface.valid || d.lightCount() == 0)
				{
					storeH4(diffuse_out, i, vec4_splat(0.0f));
					storeH4(specular_out, i, vec4_splat(0.0f));
					continue;
				}
				++pixels;
				uint rng = pcg(uint(px) + pcg(uint(py) + pcg(uint(P->frame_index) ^ 0x9e3779b9u)));
				int taps = P->di_spatial_taps;
				float canonicalCount = max(min(ownNormal.w, 20.0f), 1.0f);
				int canonicalLight = ownSample.w >= 0.0f ? int(ownSample.w + 0.5f) : -1;
				vec3 canonicalPoint = ownSample.xyz();
				float canonicalTarget = canonicalLight >= 0 && ownReceiver.w > 0.0f
					? d.lightTarget(surface, canonicalLight, canonicalPoint)
					: 0.0f;
				float pairCanonical = canonicalCount / float(max(taps, 1));
				float totalCount = canonicalCount;
				float canonicalShare = taps > 0 ? 0.0f : canonicalCount;
				float weightSum = 0.0f;
				vec3 chosenPoint = canonicalPoint;
				int chosenLight = -1;
				float chosenTarget = 0.0f;
				bool neighbourSelected = false;
				for (int tap = 0; tap < taps; ++tap)
				{
					float radius = 16.0f * sqrt(nextRandom(rng));
					float angle = 2.0f * kPi * nextRandom(rng);
					float randomSelect = nextRandom(rng);
					vec2 uv = v_texcoord0 + vec2(cos(angle), sin(angle)) * radius * d.texel;
					Surface neighbour = d.loadSurface(uv);
					vec4 sampleData = reservoirSample.sample(uv);
					vec4 receiver = reservoirReceiver.sample(uv);
					vec4 normal = reservoirNormal.sample(uv);
					int light = sampleData.w >= 0.0f ? int(sampleData.w + 0.5f) : -1;
					if (uv.x <= 0.0f || uv.x >= 1.0f || uv.y <= 0.0f || uv.y >= 1.0f || !neighbour.valid
						|| !d.sameSurface(surface.position, surface.normal, neighbour.position, neighbour.normal, 4.0f * d.kDiReceiverRadius()))
					{
						canonicalShare += pairCanonical;
						continue;
					}
					float neighbourCount = min(normal.w, 20.0f);
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
						float weight = denominator > 0.0f
							? pairWeight * neighbourDensity / denominator * target * receiver.w
							: 0.0f;
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
				vec3 diffuse, specular;
				d.evaluateLightSample(surface, chosenLight, chosenPoint, diffuse, specular);
				storeH4(diffuse_out, i, vec4(diffuse * combinedWeight, 1.0f));
				storeH4(specular_out, i, vec4(specular * combinedWeight, 1.0f));
			}
		});
	for (int t_ = 0; t_ < threadCount; ++t_)
	{
		addCounts(ds_[size_t(t_)].bvh, 0, pixelss_[size_t(t_)]);
	}
	return RESTIR_OK;
}

/* --- SVGF (svgf.sh, fs_svgf_variance.sc, fs_svgf_atrous.sc) -------------- */

namespace
{

float geometryWeight(float _sceneScale, vec3 _position, vec3 _normal, vec3 _neighbourPosition, vec3 _neighbourNormal)
{
	if (dot(_neighbourNormal, _neighbourNormal) < 0.5f)
	{
		return 0.0f;
	}
	float planeDistance = abs(dot(_normal, _neighbourPosition - _position)) / (0.02f * _sceneScale);
	float normalWeight = rn_pow64(max(dot(_normal, normalize(_neighbourNormal)), 0.0f));
	return exp(-planeDistance) * normalWeight;
}

bool isInside(vec2 _uv)
{
	return _uv.x >= 0.0f && _uv.x <= 1.0f && _uv.y >= 0.0f && _uv.y <= 1.0f;
}

} // namespace

extern "C" int oracle_svgf_variance(const RestirParams* P, const uint16_t* color, const uint16_t* moments,
	const float* receiver, const float* normal, uint16_t* output)
{
	const int w = int(P->gi_width), h = int(P->gi_height);
	TexH4 giColor = { color, w, h }, giMoments = { moments, w, h };
	TexF4 giReceiver = { receiver, w, h }, giNormal = { normal, w, h };
	const vec2 texel(1.0f / float(w), 1.0f / float(h));
parallelFor(int64_t(h), 8, [&](int64_t py_, int)
	{
		int py = int(py_);
		for (int px = 0; px < w; ++px)
		{
			int i = py * w + px;
			vec2 v_texcoord0 = (vec2(float(px), float(py)) + 0.5f) * texel;
			vec3 n = giNormal.sample(v_texcoord0).xyz();
			if (dot(n, n) < 0.5f)
			{
				storeH4(output, i, vec4_splat(0.0f));
				continue;
			}
			n = normalize(n);
			vec3 c = giColor.sample(v_texcoord0).xyz();
			vec4 m4 = giMoments.sample(v_texcoord0);
			vec3 m(m4.x, m4.y, m4.z);
			float historyLength = m.z;
			if (historyLength >= 4.0f)
			{
				storeH4(output, i, vec4(c, max(m.y - m.x * m.x, 0.0f)));
				continue;
			}
			vec3 position = giReceiver.sample(v_texcoord0).xyz();
			vec2 momentSum = vec2_splat(0.0f);
			float weightSum = 0.0f;
			for (int y = -3; y <= 3; ++y)
			{
				for (int x = -3; x <= 3; ++x)
				{
					vec2 uv = v_texcoord0 + vec2(float(x), float(y)) * texel;
					if (!isInside(uv))
					{
						continue;
					}
					float weight = geometryWeight(P->scene_scale, position, n, giReceiver.sample(uv).xyz(), giNormal.sample(uv).xyz());
					momentSum += giMoments.sample(uv).xy() * weight;
					weightSum += weight;
				}
			}
			vec2 spatialMoments = momentSum / max(weightSum, 0.0001f);
			float variance = max(spatialMoments.y - spatialMoments.x * spatialMoments.x, 0.0f)
				* (4.0f / max(historyLength, 1.0f));
			storeH4(output, i, vec4(c, variance));
		}
	});
	return RESTIR_OK;
}

extern "C" int oracle_svgf_atrous(const RestirParams* P, int step, const uint16_t* input,
	const float* receiver, const float* normal, uint16_t* output)
{
	const int w = int(P->gi_width), h = int(P->gi_height);
	TexH4 filterInput = { input, w, h };
	TexF4 giReceiver = { receiver, w, h }, giNormal = { normal, w, h };
	const vec2 texel(1.0f / float(w), 1.0f / float(h));
	const float stepSize = float(step);
	auto splineWeight = [](int _offset)
	{
		int d = _offset < 0 ? -_offset : _offset;
		return d == 0 ? 0.375f : (d == 1 ? 0.25f : 0.0625f);
	};
parallelFor(int64_t(h), 8, [&](int64_t py_, int)
	{
		int py = int(py_);
		for (int px = 0; px < w; ++px)
		{
			int i = py * w + px;
			vec2 v_texcoord0 = (vec2(float(px), float(py)) + 0.5f) * texel;
			vec3 n = giNormal.sample(v_texcoord0).xyz();
			if (dot(n, n) < 0.5f)
			{
				storeH4(output, i, vec4_splat(0.0f));
				continue;
			}
			n = normalize(n);
			vec3 position = giReceiver.sample(v_texcoord0).xyz();
			vec4 center = filterInput.sample(v_texcoord0);
			float centerLuminance = luminance(center.xyz());
			float variance = 0.0f;
			for (int by = -1; by <= 1; ++by)
			{
				for (int bx = -1; bx <= 1; ++bx)
				{
					float weight = (bx == 0 ? 0.5f : 0.25f) * (by == 0 ? 0.5f : 0.25f);
					variance += filterInput.sample(v_texcoord0 + vec2(float(bx), float(by)) * texel).w * weight;
				}
			}
			float luminanceScale = 1.0f / (4.0f * sqrt(max(variance, 0.0f)) + 0.0001f);
			vec3 colorSum = vec3_splat(0.0f);
			float varianceSum = 0.0f;
			float weightSum = 0.0f;
			for (int y = -2; y <= 2; ++y)
			{
				for (int x = -2; x <= 2; ++x)
				{
					vec2 uv = v_texcoord0 + vec2(float(x), float(y)) * (stepSize * texel);
					if (!isInside(uv))
					{
						continue;
					}
					vec4 tap = filterInput.sample(uv);
					float weight = splineWeight(x) * splineWeight(y);
					if (x != 0 || y != 0)
					{
						weight *= geometryWeight(P->scene_scale, position, n, giReceiver.sample(uv).xyz(), giNormal.sample(uv).xyz());
						weight *= exp(-abs(luminance(tap.xyz()) - centerLuminance) * luminanceScale);
					}
					colorSum += tap.xyz() * weight;
					varianceSum += tap.w * weight * weight;
					weightSum += weight;
				}
			}
			storeH4(output, i, vec4(colorSum / weightSum, varianceSum / (weightSum * weightSum)));
		}
	});
	return RESTIR_OK;
}

/* --- composite (fs_composite.sc), reference, error ----------------------- */

/* brdf.sh:68-76 */
vec3 specularAlbedo(vec3 _f0, float _roughness, float _normalView)
{
	const vec4 c0(-1.0f, -0.0275f, -0.572f, 0.022f);
	const vec4 c1(1.0f, 0.0425f, 1.04f, -0.04f);
	const vec4 r(c0.x * _roughness + c1.x, c0.y * _roughness + c1.y, c0.z * _roughness + c1.z, c0.w * _roughness + c1.w);
	const float a004 = min(r.x * r.x, rn_exp2(-9.28f * _normalView)) * r.x + r.y;
	const vec2 scaleBias(-1.04f * a004 + r.z, 1.04f * a004 + r.w);
	return _f0 * scaleBias.x + scaleBias.y;
}

extern "C" int oracle_composite_specular(const RestirParams* P, const RestirGBuffer* gb, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, const uint16_t* specular_target,
	uint16_t* hdr);

extern "C" int oracle_composite(const RestirParams* P, const RestirGBuffer* gb, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, uint16_t* hdr)
{
	return oracle_composite_specular(P, gb, shadow_atlas, gi, di_diffuse, di_specular, nullptr, hdr);
}

/* fs_composite.sc:48-143; the indirect specular term when specular_target is given. */
extern "C" int oracle_composite_specular(const RestirParams* P, const RestirGBuffer* gb, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, const uint16_t* specular_target,
	uint16_t* hdr)
{
	TexH4 specularTex = { specular_target, int(P->gi_width), int(P->gi_height) };
	const int W = int(P->width), H = int(P->height);
	const int w = int(P->gi_width), h = int(P->gi_height);
	Screen screen;
	screen.init(P);
	Shadow shadow;
	shadow.init(P, shadow_atlas);
	Sky sky;
	sky.init(P);
	TexU8 albedoTex = { gb->albedo, W, H }, normalTex = { gb->normal, W, H }, shadingTex = { gb->shading_normal, W, H };
	TexF1 depthTex = { gb->depth, W, H };
	TexH4 emissiveTex = { gb->emissive, W, H };
	TexH4 giTex = { gi, w, h };
	TexH4 diDiffuseTex = { di_diffuse, W, H }, diSpecularTex = { di_specular, W, H };
	const vec2 texel(1.0f / float(W), 1.0f / float(H));
	const vec2 giSize = vec2(float(w), float(h));
	const vec2 giTexel(1.0f / float(w), 1.0f / float(h));
	const vec3 camera(P->camera_position[0], P->camera_position[1], P->camera_position[2]);
	const vec3 lightPosition(P->light_position[0], P->light_position[1], P->light_position[2]);
	const vec3 lightColor(P->light_color[0], P->light_color[1], P->light_color[2]);
	const float s = P->scene_scale;
	const float* options = P->composite_options;
parallelFor(int64_t(H), 8, [&](int64_t py_, int)
	{
		int py = int(py_);
		for (int px = 0; px < W; ++px)
		{
			int i = py * W + px;
			vec2 v_texcoord0 = (vec2(float(px), float(py)) + 0.5f) * texel;
			float depth = depthTex.sample(v_texcoord0);
			if (depth >= 0.99999f)
			{
				vec3 farPosition = screen.reconstructWorldPosition(v_texcoord0, 1.0f);
				vec3 direction = normalize(farPosition - camera);
				storeH4(hdr, i, sky.enabled() ? vec4(sky.radiance(direction), 1.0f) : vec4_splat(0.0f));
				continue;
			}
			vec4 albedoRoughness = albedoTex.sample(v_texcoord0);
			vec4 normalMetallic = normalTex.sample(v_texcoord0);
			vec3 albedo = albedoRoughness.xyz();
			float roughness = max(albedoRoughness.w, 0.05f);
			float metallic = normalMetallic.w;
			vec3 surfaceNormal = normalize(normalMetallic.xyz() * 2.0f - 1.0f);
			vec3 normal = normalize(shadingTex.sample(v_texcoord0).xyz() * 2.0f - 1.0f);
			vec4 emissiveOcclusion = emissiveTex.sample(v_texcoord0);
			vec3 position = screen.reconstructWorldPosition(v_texcoord0, depth);
			vec3 viewDirection = normalize(camera - position);
			vec3 toLight = lightPosition - position;
			float distanceSquared = max(dot(toLight, toLight), 0.01f * s * s);
			vec3 lightDirection = toLight * inversesqrt(distanceSquared);
			vec3 diffuse, specular;
			evaluateBrdf(normal, viewDirection, lightDirection, albedo, roughness, metallic, diffuse, specular);
			float visibility = 0.0f;
			if (dot(normal, lightDirection) > 0.0f)
			{
				visibility = shadow.visibilitySoft(position, surfaceNormal);
			}
			vec3 direct = (diffuse + specular) * (lightColor / distanceSquared) * visibility
				+ diDiffuseTex.sample(v_texcoord0).xyz() + diSpecularTex.sample(v_texcoord0).xyz();

			/* upsampleIndirect (fs_composite.sc:48-80), diffuse part. */
			vec2 texelCoord = v_texcoord0 * giSize - 0.5f;
			vec2 baseCoord = floor(texelCoord);
			vec2 blend = texelCoord - baseCoord;
			vec3 sum = vec3_splat(0.0f);
			vec3 specularSum = vec3_splat(0.0f);
			float weightSum = 0.0f;
			for (int tapIndex = 0; tapIndex < 4; ++tapIndex)
			{
				vec2 offset = vec2(float(tapIndex & 1), float(tapIndex >> 1));
				vec2 tapUv = (baseCoord + offset + 0.5f) * giTexel;
				float tapDepth = depthTex.sample(tapUv);
				if (tapDepth >= 0.99999f)
				{
					continue;
				}
				vec3 tapPosition = screen.reconstructWorldPosition(tapUv, tapDepth);
				vec3 tapNormal = normalize(normalTex.sample(tapUv).xyz() * 2.0f - 1.0f);
				vec2 bilinear = mix(vec2_splat(1.0f) - blend, blend, offset);
				float weight = (bilinear.x * bilinear.y + 0.01f)
					* step(abs(dot(tapPosition - position, surfaceNormal)), 0.03f * s)
					* step(0.9f, dot(tapNormal, surfaceNormal));
				sum += giTex.sample(tapUv).xyz() * weight;
				if (specular_target != nullptr)
				{
					specularSum += specularTex.sample(tapUv).xyz() * weight;
				}
				weightSum += weight;
			}
			vec3 irradiance = weightSum > 0.0f ? sum / weightSum : giTex.sample(v_texcoord0).xyz();
			vec3 indirect = irradiance
				* (options[2] > 0.5f ? albedo * (1.0f - metallic) * emissiveOcclusion.w : vec3_splat(1.0f));
			if (specular_target != nullptr)
			{
				/* fs_composite.sc:131-136 */
				vec3 specularRadiance = weightSum > 0.0f ? specularSum / weightSum : specularTex.sample(v_texcoord0).xyz();
				vec3 f0 = mix(vec3_splat(0.04f), albedo, metallic);
				indirect += specularRadiance * specularAlbedo(f0, roughness, max(dot(normal, viewDirection), 0.001f))
					* emissiveOcclusion.w * P->composite_specular;
			}
			vec3 result = direct * options[0] + indirect * options[1] + emissiveOcclusion.xyz() * options[3];
			storeH4(hdr, i, vec4(result, 1.0f));
		}
	});
	return RESTIR_OK;
}

extern "C" int oracle_reference_accumulate(const RestirParams* P, const uint16_t* hdr, double* mean,
	uint8_t* alpha, uint32_t frames)
{
	const size_t n = size_t(P->width) * P->height;
	const double weight = 1.0 / double(frames + 1);
parallelFor(int64_t(int64_t(n)), 64, [&](int64_t i_, int)
	{
		int64_t i = int64_t(i_);
		float c[4];
		for (int k = 0; k < 4; ++k)
		{
			c[k] = rn_half_to_float(hdr[4 * i + k]);
		}
		bool nan = c[0] != c[0] || c[1] != c[1] || c[2] != c[2];
		for (int k = 0; k < 3; ++k)
		{
			double history = mean[k * n + i];
			double color = nan ? history : double(c[k]);
			mean[k * n + i] = history * (1.0 - weight) + color * weight;
		}
		alpha[i] = c[3] >= 0.5f ? 1 : 0;
	});
	return RESTIR_OK;
}

extern "C" int oracle_error(const RestirParams* P, const uint16_t* display, const double* mean,
	const uint8_t* alpha, double* out)
{
	const size_t n = size_t(P->width) * P->height;
	double relative = 0.0, image = 0.0, reference = 0.0, count = 0.0;
	for (size_t i = 0; i < n; ++i)
	{
		if (alpha[i] == 0)
		{
			continue;
		}
		double r = rn_half_to_float(display[4 * i + 0]);
		double g = rn_half_to_float(display[4 * i + 1]);
		double b = rn_half_to_float(display[4 * i + 2]);
		double imageLuminance = 0.2126 * r + 0.7152 * g + 0.0722 * b;
		double referenceLuminance = 0.2126 * mean[i] + 0.7152 * mean[n + i] + 0.0722 * mean[2 * n + i];
		double difference = imageLuminance - referenceLuminance;
		relative += difference * difference / (referenceLuminance * referenceLuminance + 0.01);
		image += imageLuminance;
		reference += referenceLuminance;
		count += 1.0;
	}
	double total = count > 1.0 ? count : 1.0;
	out[0] = relative / total;
	out[1] = image / total;
	out[2] = reference / total;
	out[3] = count;
	return RESTIR_OK;
}

extern "C" void oracle_grid_keys(const float* camera, const float* constants, uint32_t table_size, const float* positions,
	const float* normals, const float* randoms, uint32_t n, uint32_t* cell_bits, uint32_t* slots, uint32_t* checksums)
{
	Grid g;
	g.minCell = constants[0];
	g.pixelSize = constants[1];
	g.cellPixels = constants[2];
	g.camera = vec3(camera[0], camera[1], camera[2]);
	g.tableSize = table_size;
	for (uint32_t i = 0; i < n; ++i)
	{
		vec3 p(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
		vec3 nrm(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]);
		float size = g.cellSize(p);
		vec3 jittered = Grid::jitter(p, nrm, size, randoms[2 * i], randoms[2 * i + 1]);
		g.key(jittered, nrm, size, slots[i], checksums[i]);
		cell_bits[i] = floatBitsToUint(size);
	}
}

/* --- indirect specular (fs_specular.sc) ---------------------------------- */

namespace
{

void tangentFrame(vec3 _normal, vec3& _tangent, vec3& _bitangent)
{
	_tangent = normalize(abs(_normal.y) < 0.99f
		? cross(_normal, vec3(0.0f, 1.0f, 0.0f))
		: cross(_normal, vec3(1.0f, 0.0f, 0.0f)));
	_bitangent = cross(_normal, _tangent);
}

vec3 sampleVisibleNormal(vec3 _view, float _alpha, float _random0, float _random1)
{
	vec3 stretched = normalize(vec3(_alpha * _view.x, _alpha * _view.y, _view.z));
	float lengthSquared = stretched.x * stretched.x + stretched.y * stretched.y;
	vec3 t1 = lengthSquared > 0.0f
		? vec3(-stretched.y, stretched.x, 0.0f) * inversesqrt(lengthSquared)
		: vec3(1.0f, 0.0f, 0.0f);
	vec3 t2 = cross(stretched, t1);
	float radius = sqrt(_random0);
	float angle = 2.0f * kPi * _random1;
	float p1 = radius * cos(angle);
	float p2 = radius * sin(angle);
	float s = 0.5f * (1.0f + stretched.z);
	p2 = (1.0f - s) * sqrt(max(1.0f - p1 * p1, 0.0f)) + s * p2;
	vec3 normal = p1 * t1 + p2 * t2 + sqrt(max(1.0f - p1 * p1 - p2 * p2, 0.0f)) * stretched;
	return normalize(vec3(_alpha * normal.x, _alpha * normal.y, max(normal.z, 0.0f)));
}

float smithG1(float _cosine, float _alpha)
{
	float alphaSquared = _alpha * _alpha;
	return 2.0f * _cosine / (_cosine + sqrt(alphaSquared + (1.0f - alphaSquared) * _cosine * _cosine));
}

vec3 reflect(vec3 _incident, vec3 _normal)
{
	return _incident - 2.0f * dot(_normal, _incident) * _normal;
}

/* fs_specular.sc:77-125 */
vec3 hitRadiance(const GiPass& g, const TexH4& previousHdr, vec3 _hitPosition, float _hitId, vec3 _rayDirection)
{
	if (isSkySample(_hitId))
	{
		return g.sky.radiance(_rayDirection);
	}
	vec2 uv;
	float viewDepth;
	bool visibleSurface = false;
	if (g.projectToScreen(_hitPosition, uv, viewDepth))
	{
		float depth = g.depthTex.sample(uv);
		visibleSurface = depth < kSkyDepth
			&& distance(g.reconstructWorldPosition(uv, depth), _hitPosition) <= g.kSampleTolerance();
	}
	if (visibleSurface)
	{
		vec4 clip = mul(g.screen.prevViewProj, vec4(_hitPosition, 1.0f));
		if (g.P->history_valid > 0.5f && clip.w > 0.0001f)
		{
			vec2 previousUv = g.screen.clipToUv(clip);
			vec4 previous = previousHdr.sample(previousUv);
			if (isOnScreen(previousUv) && previous.w > 0.5f)
			{
				return previous.xyz();
			}
		}
		vec3 normal = g.decodeNormal(uv);
		return g.evaluateSecondaryDirect(uv, _hitPosition, normal)
			+ g.previousIndirect(_hitPosition, normal, g.diffuseAlbedo(uv))
			+ g.surfaceLight.sample(uv).xyz() * g.P->surface_light_scale;
	}
	int triangleIndex = int(abs(_hitId) + 0.5f) - 1;
	if (triangleIndex < 0 || !g.bvh.available())
	{
		return vec3_splat(0.0f);
	}
	vec3 v0 = g.bvh.vertex(triangleIndex, 0);
	vec3 normal = normalize(cross(g.bvh.vertex(triangleIndex, 1) - v0, g.bvh.vertex(triangleIndex, 2) - v0));
	normal = dot(normal, -_rayDirection) < 0.0f ? -normal : normal;
	vec3 albedo = bvhTriangleAlbedo(g.bvh, triangleIndex);
	return g.evaluateWorldDirect(albedo, _hitPosition, normal)
		+ g.previousIndirect(_hitPosition, normal, albedo)
		+ bvhTriangleEmission(g.bvh, triangleIndex) * g.P->emission_scale;
}

} // namespace

/* fs_specular.sc:127-226 at GI resolution. */
extern "C" int oracle_gi_specular(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiHistory* history, const float* shadow_atlas, const uint16_t* surface_light, const uint16_t* previous_hdr,
	const uint16_t* specular_history, uint16_t* specular)
{
	resetCounts();
	const GiPass base = makeGiPass(P, scene, gb, history, shadow_atlas, surface_light);
	const int W = int(P->width), H = int(P->height);
	const int w = int(P->gi_width), h = int(P->gi_height);
	const TexH4 previousHdr = { previous_hdr, W, H };
	const TexH4 specularHistory = { specular_history, w, h };
	const vec3 camera(P->camera_position[0], P->camera_position[1], P->camera_position[2]);
	parallelFor(int64_t(h), 4, [&](int64_t py_, int)
	{
		const GiPass& g = base;
		const int py = int(py_);
		for (int px = 0; px < w; ++px)
		{
			const int outIndex = py * w + px;
			vec2 v_texcoord0 = (vec2(float(px), float(py)) + 0.5f) * g.giTexel;
			float depth = g.depthTex.sample(v_texcoord0);
			if (depth >= kSkyDepth)
			{
				storeH4(specular, outIndex, vec4_splat(0.0f));
				continue;
			}
			vec3 position = g.reconstructWorldPosition(v_texcoord0, depth);
			vec3 normal = g.decodeNormal(v_texcoord0);
			vec4 albedoRoughness = g.albedoTex.sample(v_texcoord0);
			float metallic = g.normalTex.sample(v_texcoord0).w;
			float roughness = max(albedoRoughness.w, 0.02f);
			float alpha = roughness * roughness;
			vec3 viewDirection = normalize(camera - position);
			float normalView = max(dot(normal, viewDirection), 0.001f);
			vec3 f0 = mix(vec3_splat(0.04f), albedoRoughness.xyz(), metallic);
			vec2 pixel = g.giPixel(v_texcoord0);
			uint rng = pcg(uint(pixel.x) + pcg(uint(pixel.y) + pcg(uint(P->frame_index) ^ 0x2545f491u)));

			vec3 tangent, bitangent;
			tangentFrame(normal, tangent, bitangent);
			vec3 localView = vec3(dot(viewDirection, tangent), dot(viewDirection, bitangent), normalView);
			float random0 = nextRandom(rng);
			float random1 = nextRandom(rng);
			vec3 localHalfway = sampleVisibleNormal(localView, alpha, random0, random1);
			vec3 halfway = tangent * localHalfway.x + bitangent * localHalfway.y + normal * localHalfway.z;
			vec3 direction = reflect(-viewDirection, halfway);
			float normalLight = dot(normal, direction);

			vec3 estimate = vec3_splat(0.0f);
			if (normalLight > 0.0f)
			{
				vec3 rayOrigin = position + normal * g.kRayBias();
				vec3 hitPosition = vec3_splat(0.0f);
				float hitId = 0.0f;
				bool hit = false;
				if (P->ray_mode != RESTIR_RAY_MODE_BVH)
				{
					hit = g.traceScreenSpaceRay(rayOrigin, direction, g.kMaxRayDistance(), hitPosition);
				}
				if (!hit && P->ray_mode != RESTIR_RAY_MODE_SCREEN)
				{
					float hitDistance = 0.0f;
					int triangleIndex = traceBvh(g.bvh, rayOrigin, direction, g.kMaxBvhRayDistance(), false, hitDistance, false);
					if (triangleIndex >= 0)
					{
						hit = true;
						hitPosition = rayOrigin + direction * hitDistance;
						hitId = g.encodeSampleId(triangleIndex, direction);
					}
					else if (g.sky.enabled())
					{
						hit = true;
						hitId = kSkySampleId;
					}
				}
				if (hit)
				{
					vec3 fresnel = fresnelSchlick(halfway, viewDirection, f0);
					estimate = hitRadiance(g, previousHdr, hitPosition, hitId, direction) * fresnel * smithG1(normalLight, alpha);
				}
			}

			vec3 demodulated = estimate / max(specularAlbedo(f0, roughness, normalView), vec3_splat(0.001f));
			if (P->outlier_clamp > 0.0f)
			{
				demodulated = min(demodulated, vec3_splat(P->outlier_clamp));
			}

			vec3 pastColor = vec3_splat(0.0f);
			float historyLength = 0.0f;
			vec4 clipPrevious = mul(g.screen.prevViewProj, vec4(position, 1.0f));
			if (P->history_valid > 0.5f && clipPrevious.w > 0.0001f)
			{
				vec2 previousUv = (floor(g.screen.clipToUv(clipPrevious) * g.giSize) + 0.5f) * g.giTexel;
				vec3 receiverPosition = g.historyReceiver.sample(previousUv).xyz();
				vec3 receiverNormal = g.historyNormal.sample(previousUv).xyz();
				vec3 offset = receiverPosition - position;
				if (isOnScreen(previousUv)
					&& dot(receiverNormal, receiverNormal) > 0.5f
					&& dot(offset, offset) <= g.kBounceRadius() * g.kBounceRadius()
					&& abs(dot(offset, normal)) <= g.kReceiverPlane()
					&& dot(normalize(receiverNormal), normal) >= 0.9f)
				{
					vec4 previous = specularHistory.sample(previousUv);
					pastColor = previous.xyz();
					historyLength = previous.w;
				}
			}
			float maxHistory = mix(4.0f, 32.0f, clamp(roughness * 1.5f, 0.0f, 1.0f));
			historyLength = min(historyLength + 1.0f, maxHistory);
			storeH4(specular, outIndex, vec4(mix(pastColor, demodulated, 1.0f / historyLength), historyLength));
		}
	});
	return RESTIR_OK;
}

extern "C" void oracle_numeric_eval(int fn, const float* input, float* output, uint32_t n)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		const float x = input[i];
		float y = x;
		switch (fn)
		{
		case 0: y = rn_sin(x); break;
		case 1: y = rn_cos(x); break;
		case 2: y = rn_exp(x); break;
		case 3:
		case 4: y = rn_half_to_float(rn_float_to_half(x)); break;
		case 5: y = float(rn_unorm8(x)); break;
		case 6: y = float(rn_floor_log2(x)); break;
		case 7: y = rn_pow64(x); break;
		case 8: y = rn_bits_float(pcg(rn_float_bits(x))); break;
		case 9: y = rn_bits_float(gridChecksumHash(rn_float_bits(x))); break;
		case 10: y = rn_half_to_float(uint16_t(rn_float_bits(x) & 0xffffu)); break;
		case 11: y = rn_log2(x); break;
		case 12: y = rn_exp2(x); break;
		case 13: y = rn_pow(x, 2.2f); break;
		case 14: y = rn_pow(x, 1.0f / 2.2f); break;
		default: break;
		}
		output[i] = y;
	}
}

extern "C" void oracle_last_counts(uint64_t* counts)
{
	for (int i = 0; i < 5; ++i)
	{
		counts[i] = g_counts[i];
	}
}

int& oracle::threadSetting()
{
	static int s_threads = 0;
	return s_threads;
}

extern "C" void oracle_set_threads(int count)
{
	threadSetting() = count;
}

extern "C" int oracle_get_threads(void)
{
	return threads();
}
