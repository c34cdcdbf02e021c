// The frame driver: the reference's Renderer (src/renderer.h:73-125,
// src/renderer.cpp:365-1166) over the CUDA passes of include/restir_gpu.h.
//
// It owns every device buffer of a frame and its history with the
// reference's ping-pong by frame parity (renderer.h:218-219), derives the
// uniforms with restir_frame_params, and enqueues the passes in the
// reference's order on its own stream. render_graph records a frame with
// stream capture and replays it as one CUDA graph launch; later frames are
// captured again and patched into the instantiated graph
// (cudaGraphExecUpdate), since their uniforms and ping-pong buffers change.
#include "../../include/restir_cache.h"
#include "../../include/restir_display.h"
#include "../../include/restir_frame.h"
#include "bvh_build.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

namespace restir
{

// The no-allocation error pass shares this launcher (csrc/reference.cu).
int launchError(const RestirParams* params, const uint16_t* display, const double* mean, const uint8_t* alpha, double* out,
	double* partials, cudaStream_t stream);
uint64_t errorScratchBytes();

namespace
{

struct Buffer
{
	void* pointer = nullptr;
	uint64_t bytes = 0;
};

// A scene's host data and device buffers (BVH, normals, materials, light
// list, radiance cache), shared by every renderer drawing it.
struct SceneState
{
	Mesh mesh;
	BvhResult bvh;
	LightListResult lights;
	std::string lightsKey;
	std::map<std::string, Buffer> buffers;
	RestirCacheConfig cacheConfig = {};
	bool has = false;

	SceneState() = default;
	SceneState(const SceneState&) = delete;
	SceneState& operator=(const SceneState&) = delete;
	~SceneState()
	{
		for (auto& kv : buffers)
		{
			cudaFree(kv.second.pointer);
		}
	}
};

class Batch;

class Renderer
{
	friend class Batch;

public:
	explicit Renderer(const RestirSettings& settings) : m_settings(settings)
	{
		std::memset(&m_state, 0, sizeof(m_state));
		for (int i = 0; i < 4; ++i)
		{
			m_state.previous_view_proj[i * 5] = 1.0f;
		}
		// The main chain of passes at the device's highest stream priority: the
		// block scheduler then fills what it leaves free with the passes on
		// the side streams, instead of stretching the chain.
		int leastPriority = 0, greatestPriority = 0;
		cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority);
		cudaStreamCreateWithPriority(&m_stream, cudaStreamNonBlocking, greatestPriority);
		cudaStreamCreateWithFlags(&m_side, cudaStreamNonBlocking);
		cudaEventCreateWithFlags(&m_fork, cudaEventDisableTiming);
		cudaEventCreateWithFlags(&m_join, cudaEventDisableTiming);
		cudaStreamCreateWithFlags(&m_aside, cudaStreamNonBlocking);
		cudaEventCreateWithFlags(&m_asideFork, cudaEventDisableTiming);
		cudaEventCreateWithFlags(&m_shadowJoin, cudaEventDisableTiming);
		cudaEventCreateWithFlags(&m_specularJoin, cudaEventDisableTiming);
		for (auto& frame : m_events)
		{
			for (auto& pass : frame)
			{
				cudaEventCreate(&pass[0]);
				cudaEventCreate(&pass[1]);
			}
		}
		cudaMallocHost(&m_errorHost, 4 * sizeof(double));
		for (int k = 0; k < 2; ++k)
		{
			cudaEventCreateWithFlags(&m_orbitCopied[k], cudaEventDisableTiming);
		}
	}

	~Renderer()
	{
		cudaStreamSynchronize(m_stream);
		releaseGraph();
		releaseTargets();
		releaseScene();
		for (auto& frame : m_events)
		{
			for (auto& pass : frame)
			{
				cudaEventDestroy(pass[0]);
				cudaEventDestroy(pass[1]);
			}
		}
		cudaFreeHost(m_errorHost);
		for (int k = 0; k < 2; ++k)
		{
			cudaEventDestroy(m_orbitCopied[k]);
			cudaFreeHost(m_orbitHost[k]);
		}
		cudaStreamSynchronize(m_side);
		cudaEventDestroy(m_fork);
		cudaEventDestroy(m_join);
		cudaStreamDestroy(m_side);
		cudaStreamSynchronize(m_aside);
		cudaEventDestroy(m_asideFork);
		cudaEventDestroy(m_shadowJoin);
		cudaEventDestroy(m_specularJoin);
		cudaStreamDestroy(m_aside);
		cudaStreamDestroy(m_stream);
	}

	int setScene(const Mesh& mesh, bool useSceneDefaults)
	{
		cudaStreamSynchronize(m_stream);
		releaseGraph();
		releaseScene();
		m_scene->mesh = mesh;
		if (useSceneDefaults)
		{
			std::memcpy(m_settings.light_position, mesh.lightPosition, sizeof(m_settings.light_position));
			m_settings.sky_enabled = mesh.sky ? 1 : 0;
		}
		int status = 0;
		if (m_settings.bvh_on_device)
		{
			// Built on the device; the rows and normals stay there.
			DeviceBvh device;
			const int built = buildBvhGpu(mesh, m_stream, m_scene->bvh, &device);
			if (built != RESTIR_OK)
			{
				m_scene->has = false;
				return built;
			}
			m_scene->buffers["bvh"] = Buffer{ device.rows, device.rowsBytes };
			m_scene->buffers["normals"] = Buffer{ device.normals, device.normalsBytes };
		}
		else
		{
			m_scene->bvh = buildBvh(mesh, 8);
			status |= upload(m_scene->buffers["bvh"], m_scene->bvh.data.data(), m_scene->bvh.data.size() * sizeof(float));
			status |= upload(m_scene->buffers["normals"], m_scene->bvh.triangleNormals.data(),
				m_scene->bvh.triangleNormals.size() * sizeof(float));
		}
		status |= upload(m_scene->buffers["materials"], mesh.materialData.data(), mesh.materialData.size() * sizeof(float));
		m_scene->lightsKey.clear();
		status |= updateLights();
		status |= initCache(mesh);
		m_state.history_valid = 0;
		m_state.di_valid = 0;
		m_state.reference_frames = 0;
		m_state.taa_valid = 0;
		m_state.exposure_valid = 0;
		m_scene->has = status == 0;
		return status == 0 ? RESTIR_OK : RESTIR_ERROR_OUT_OF_MEMORY;
	}

	// The radiance cache over the scene's box (1% of the radius wider), fresh
	// for every scene.
	int initCache(const Mesh& mesh)
	{
		restir_cache_config_default(&m_scene->cacheConfig);
		for (int i = 0; i < 3; ++i)
		{
			m_scene->cacheConfig.bounds_min[i] = mesh.boundsMin[i] - 0.01f * mesh.radius;
			m_scene->cacheConfig.bounds_max[i] = mesh.boundsMax[i] + 0.01f * mesh.radius;
		}
		const uint64_t bytes = restir_cache_state_bytes(&m_scene->cacheConfig);
		Buffer& b = m_scene->buffers["cache.state"];
		b.bytes = bytes;
		if (bytes == 0 || cudaMalloc(&b.pointer, bytes) != cudaSuccess)
		{
			b.pointer = nullptr;
			return 1;
		}
		applyCacheSettings();
		return restir_cache_init(&m_scene->cacheConfig, b.pointer, m_stream) == RESTIR_OK ? 0 : 1;
	}

	int setSettings(const RestirSettings& settings)
	{
		m_settings = settings;
		applyCacheSettings();
		return updateLights();
	}

	// The settings the cache's training reads on every step.
	void applyCacheSettings()
	{
		RestirCacheConfig defaults;
		restir_cache_config_default(&defaults);
		m_scene->cacheConfig.learning_rate = m_settings.cache_learning_rate > 0.0f ? m_settings.cache_learning_rate
			: defaults.learning_rate;
	}

	const RestirSettings& settings() const { return m_settings; }

	// The frame's uniforms, targets and workspace (the first part of render).
	int prepare(const RestirFrameInput& input)
	{
		if (!m_scene->has)
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		int status = updateLights();
		if (status == RESTIR_OK)
		{
			status = orbitLights(input.delta_time);
		}
		if (status != RESTIR_OK)
		{
			return status;
		}
		RestirMeshDesc desc = describe();
		RestirBvhDesc bvhDesc = {};
		bvhDesc.node_count = m_scene->bvh.nodeCount;
		bvhDesc.triangle_offset = m_scene->bvh.triangleOffset;
		bvhDesc.triangle_count = m_scene->bvh.triangleCount;
		// Reference mode: a moved camera starts the reference again (renderer.cpp:1050-1060).
		// The frame time is not part of the view.
		RestirFrameInput view = input;
		view.delta_time = 0.0f;
		if (m_state.reference_accumulating && m_state.reference_frames > 0
			&& (std::memcmp(&m_referenceInput, &view, sizeof(view)) != 0))
		{
			m_state.reference_frames = 0;
		}
		m_referenceInput = view;
		m_deltaTime = input.delta_time;
		status = restir_frame_params(&m_settings, &desc, m_scene->lights.count, &bvhDesc, &input, &m_state, &m_params, &m_plan);
		if (status != RESTIR_OK)
		{
			return status;
		}
		if (!targetsMatch(m_params))
		{
			// New targets start a new history: derive the uniforms again from the reset state.
			status = ensureTargets(m_params);
			if (status == RESTIR_OK)
			{
				status = restir_frame_params(&m_settings, &desc, m_scene->lights.count, &bvhDesc, &input, &m_state, &m_params, &m_plan);
			}
			if (status != RESTIR_OK)
			{
				return status;
			}
		}
		return ensureWorkspace(m_params);
	}

	// What the frame carries to the next: state and the ping-pong (the last part of render).
	void advance(const RestirFrameInput& input)
	{
		restir_frame_advance(&m_params, &m_plan, &input, &m_state);
		m_historyRead = 1 - m_historyRead;
		m_displayTaa = m_plan.display && m_plan.taa;
		if (m_plan.specular)
		{
			m_specularRead = 1 - m_specularRead;
		}
		if (m_displayTaa)
		{
			m_taaRead = 1 - m_taaRead;
		}
		if (m_plan.di_active)
		{
			m_diRead = 1 - m_diRead;
		}
	}

	int render(const RestirFrameInput& input, bool graph)
	{
		int status = prepare(input);
		if (status != RESTIR_OK)
		{
			return status;
		}
		if (graph)
		{
			status = renderGraph();
			m_timedFrames = 0;
		}
		else
		{
			status = enqueue(true);
			m_lastSlot = m_slot;
			m_slot = (m_slot + 1) % kEventRing;
			m_timedFrames = m_timedFrames < kEventRing ? m_timedFrames + 1 : kEventRing;
		}
		if (status != RESTIR_OK)
		{
			return status;
		}
		advance(input);
		m_timed = !graph;
		return RESTIR_OK;
	}

	// --- batch views (restir_batch_*) ---

	// Draws another renderer's scene (no copy; the scene lives while either holds it).
	void shareScene(const Renderer& owner)
	{
		cudaStreamSynchronize(m_stream);
		releaseGraph();
		m_scene = owner.m_scene;
		m_state.history_valid = 0;
		m_state.di_valid = 0;
		m_state.reference_frames = 0;
		m_state.taa_valid = 0;
		m_state.exposure_valid = 0;
	}

	// The batch's shadow atlas and ray queue (null: the renderer's own).
	void setBatch(float* atlas, void* queue, uint32_t capacity)
	{
		m_sharedAtlas = atlas;
		m_batchQueue = queue;
		m_batchQueueCapacity = capacity;
	}

	// The candidate records of this view's share of the batch's ray queue.
	int ensureRecords()
	{
		const uint64_t needed = restir_gi_candidate_records_bytes(&m_params);
		auto found = m_targets.find("gi.records");
		if (found != m_targets.end() && found->second.bytes >= needed)
		{
			return RESTIR_OK;
		}
		cudaStreamSynchronize(m_stream);
		if (found != m_targets.end())
		{
			cudaFree(found->second.pointer);
			m_targets.erase(found);
		}
		Buffer b;
		b.bytes = needed;
		if (cudaMalloc(&b.pointer, needed) != cudaSuccess)
		{
			return RESTIR_ERROR_OUT_OF_MEMORY;
		}
		m_targets["gi.records"] = b;
		return RESTIR_OK;
	}

	uint32_t candidateRays() const
	{
		return m_params.gi_width * m_params.gi_height * uint32_t(m_params.initial_candidates > 0 ? m_params.initial_candidates : 0);
	}

	const RestirParams& params() const { return m_params; }

	RestirScene deviceScene()
	{
		RestirScene scene = {};
		scene.bvh = static_cast<const float*>(m_scene->buffers["bvh"].pointer);
		scene.node_count = m_scene->bvh.nodeCount;
		scene.triangle_offset = m_scene->bvh.triangleOffset;
		scene.triangle_count = m_scene->bvh.triangleCount;
		scene.lights = static_cast<const float*>(m_scene->buffers["lights"].pointer);
		scene.light_count = m_scene->lights.count;
		scene.triangle_normals = static_cast<const float*>(m_scene->buffers["normals"].pointer);
		scene.materials = static_cast<const float*>(m_scene->buffers["materials"].pointer);
		scene.material_count = uint32_t(m_scene->mesh.materials.size());
		return scene;
	}

	int measure(RestirMetrics* metrics)
	{
		std::memset(metrics, 0, sizeof(*metrics));
		if (m_targets.empty())
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		// The error pass compares the displayed image: the TAA output when TAA ran (renderer.cpp:1078-1094).
		int status = launchError(&m_params, displayedHdr(), p<double>("reference.mean"), p<uint8_t>("reference.alpha"),
			p<double>("error.out"), p<double>("error.scratch"), m_stream);
		if (status != RESTIR_OK)
		{
			return status;
		}
		cudaMemcpyAsync(m_errorHost, p<double>("error.out"), 4 * sizeof(double), cudaMemcpyDeviceToHost, m_stream);
		if (cudaStreamSynchronize(m_stream) != cudaSuccess)
		{
			return RESTIR_ERROR_LAUNCH;
		}
		std::memcpy(metrics->error, m_errorHost, sizeof(metrics->error));
		metrics->valid = m_state.reference_frames > 0 ? 1 : 0;
		metrics->relative_mse = m_errorHost[0];
		metrics->bias = m_errorHost[2] > 0.0 ? m_errorHost[1] / m_errorHost[2] - 1.0 : 0.0;
		metrics->reference_frames = m_state.reference_frames;
		passTimes(metrics->pass_ms);
		return RESTIR_OK;
	}

	void passTimes(float* ms)
	{
		for (int i = 0; i < RESTIR_PASS_COUNT; ++i)
		{
			ms[i] = 0.0f;
			if (m_timed && m_passRan[m_lastSlot][i])
			{
				cudaEventElapsedTime(&ms[i], m_events[m_lastSlot][i][0], m_events[m_lastSlot][i][1]);
			}
		}
	}

	// Per-pass times of the last `frames` stream-launched frames, oldest
	// first (ms[f * RESTIR_PASS_COUNT + pass]); returns how many there were.
	int passHistory(uint32_t frames, float* ms)
	{
		if (cudaStreamSynchronize(m_stream) != cudaSuccess)
		{
			return RESTIR_ERROR_LAUNCH;
		}
		const uint32_t available = frames < m_timedFrames ? frames : m_timedFrames;
		for (uint32_t f = 0; f < available; ++f)
		{
			const uint32_t slot = (m_slot + kEventRing - available + f) % kEventRing;
			for (int i = 0; i < RESTIR_PASS_COUNT; ++i)
			{
				float t = 0.0f;
				if (m_passRan[slot][i])
				{
					cudaEventElapsedTime(&t, m_events[slot][i][0], m_events[slot][i][1]);
				}
				ms[f * RESTIR_PASS_COUNT + i] = t;
			}
		}
		return int(available);
	}

	void setReferenceAccumulation(bool accumulate)
	{
		if (accumulate == (m_state.reference_accumulating != 0))
		{
			return;
		}
		m_state.reference_accumulating = accumulate ? 1 : 0;
		if (accumulate)
		{
			m_state.reference_frames = 0;
		}
		// The history means something else with and without the shortcuts (renderer.cpp:1139-1141).
		m_state.history_valid = 0;
		m_state.taa_valid = 0;
	}

	void invalidateHistory()
	{
		m_state.history_valid = 0;
		m_state.di_valid = 0;
	}

	cudaStream_t stream() const { return m_stream; }

	// One frame with the work counters on, gathered per pass.
	int profile(const RestirFrameInput& input, uint64_t* counts)
	{
		std::memset(counts, 0, sizeof(uint64_t) * 8 * RESTIR_PASS_COUNT);
		restir_counters(1, nullptr);
		m_profile = counts;
		int status = render(input, false);
		m_profile = nullptr;
		restir_counters(0, nullptr);
		return status;
	}

	void lastFrame(RestirParams* params, RestirFramePlan* plan, RestirFrameState* state) const
	{
		if (params)
		{
			*params = m_params;
		}
		if (plan)
		{
			*plan = m_plan;
		}
		if (state)
		{
			*state = m_state;
		}
	}

	// The last frame's displayed HDR image: its TAA output, or the composite.
	uint16_t* displayedHdr()
	{
		return m_displayTaa ? p<uint16_t>("taa" + std::to_string(m_taaRead)) : p<uint16_t>("hdr");
	}

	int buffer(const std::string& name, void** pointer, uint64_t* bytes)
	{
		if (name == "display.hdr" && !m_targets.empty())
		{
			*pointer = displayedHdr();
			*bytes = m_targets["hdr"].bytes;
			return RESTIR_OK;
		}
		auto it = m_targets.find(name);
		if (it == m_targets.end())
		{
			it = m_scene->buffers.find(name);
			if (it == m_scene->buffers.end())
			{
				return RESTIR_ERROR_INVALID_ARGUMENT;
			}
		}
		*pointer = it->second.pointer;
		*bytes = it->second.bytes;
		return RESTIR_OK;
	}

private:
	template<typename T>
	T* p(const std::string& name)
	{
		return static_cast<T*>(m_targets[name].pointer);
	}

	static int upload(Buffer& b, const void* data, size_t bytes)
	{
		b.bytes = bytes;
		if (bytes == 0)
		{
			return 0;
		}
		if (cudaMalloc(&b.pointer, bytes) != cudaSuccess)
		{
			b.pointer = nullptr;
			return 1;
		}
		return cudaMemcpy(b.pointer, data, bytes, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : 1;
	}

	RestirMeshDesc describe() const
	{
		RestirMeshDesc d = {};
		d.triangle_count = m_scene->mesh.triangleCount();
		d.material_count = uint32_t(m_scene->mesh.materials.size());
		std::memcpy(d.bounds_min, m_scene->mesh.boundsMin, sizeof(d.bounds_min));
		std::memcpy(d.bounds_max, m_scene->mesh.boundsMax, sizeof(d.bounds_max));
		std::memcpy(d.center, m_scene->mesh.center, sizeof(d.center));
		d.radius = m_scene->mesh.radius;
		return d;
	}

	// Renderer::updateLightList (renderer.cpp:1170-1207): rebuilt when its inputs change.
	int updateLights()
	{
		if (!m_scene->has && m_scene->bvh.nodeCount == 0)
		{
			return RESTIR_OK;
		}
		const float scale = (m_scene->mesh.radius / 1.75f) * (m_scene->mesh.radius / 1.75f);
		std::string key = std::to_string(m_settings.emissive_lighting) + "/" + std::to_string(m_settings.extra_lights) + "/"
			+ std::to_string(m_settings.extra_intensity) + "/" + std::to_string(m_settings.extra_seed) + "/" + std::to_string(scale);
		if (key == m_scene->lightsKey)
		{
			return RESTIR_OK;
		}
		m_scene->lightsKey = key;
		static const std::vector<Emitter> none;
		m_scene->lights = buildLightList(m_settings.emissive_lighting ? m_scene->bvh.emitters : none, m_settings.extra_lights,
			m_settings.extra_intensity, uint32_t(m_settings.extra_seed), m_scene->mesh.boundsMin, m_scene->mesh.boundsMax, scale);
		cudaStreamSynchronize(m_stream);
		Buffer& b = m_scene->buffers["lights"];
		cudaFree(b.pointer);
		b = Buffer();
		std::vector<float> data = m_scene->lights.data;
		if (data.empty())
		{
			data.assign(16, 0.0f);
		}
		int status = upload(b, data.data(), data.size() * sizeof(float));
		m_state.di_valid = 0; // stored light indices refer to the old list
		releaseGraph();
		return status == 0 ? RESTIR_OK : RESTIR_ERROR_OUT_OF_MEMORY;
	}

	// The extra point lights on their orbits (RestirSettings::extra_light_orbit):
	// light k turns about the vertical axis through the scene's centre by
	// orbit * s_k * t radians, t the frames' accumulated delta_time, s_k a
	// seeded speed in [0.25, 1] with a seeded sign. The moved list is written
	// to one of two pinned host buffers (the other may still be copying) and
	// copied to the device on the frame's stream.
	int orbitLights(float deltaTime)
	{
		const LightListResult& list = m_scene->lights;
		if (!(m_settings.extra_light_orbit > 0.0f) || list.count == list.triangles)
		{
			return RESTIR_OK;
		}
		m_orbitTime += double(deltaTime);
		const size_t floats = size_t(list.count) * 16u;
		const int k = m_orbitSlot;
		m_orbitSlot ^= 1;
		if (m_orbitCapacity[k] < floats)
		{
			cudaEventSynchronize(m_orbitCopied[k]);
			cudaFreeHost(m_orbitHost[k]);
			m_orbitHost[k] = nullptr;
			m_orbitCapacity[k] = 0;
			if (cudaMallocHost(reinterpret_cast<void**>(&m_orbitHost[k]), floats * sizeof(float)) != cudaSuccess)
			{
				return RESTIR_ERROR_OUT_OF_MEMORY;
			}
			m_orbitCapacity[k] = floats;
		}
		// The copy this buffer fed two frames ago has finished before it is rewritten.
		cudaEventSynchronize(m_orbitCopied[k]);
		float* out = m_orbitHost[k];
		std::memcpy(out, list.data.data(), floats * sizeof(float));
		const float cx = m_scene->mesh.center[0], cz = m_scene->mesh.center[2];
		for (uint32_t light = list.triangles; light < list.count; ++light)
		{
			uint32_t h = uint32_t(light - list.triangles) * 2654435761u + uint32_t(m_settings.extra_seed) * 97u + 1u;
			h = h * 747796405u + 2891336453u;
			h = ((h >> ((h >> 28u) + 4u)) ^ h) * 277803737u;
			h = (h >> 22u) ^ h;
			const float speed = (0.25f + 0.75f * float(h >> 8) * (1.0f / 16777216.0f)) * ((h & 1u) ? 1.0f : -1.0f);
			const double angle = double(m_settings.extra_light_orbit) * double(speed) * m_orbitTime;
			const float c = float(std::cos(angle)), sn = float(std::sin(angle));
			float* row = out + size_t(light) * 16u;
			const float dx = row[0] - cx, dz = row[2] - cz;
			row[0] = cx + c * dx + sn * dz;
			row[2] = cz - sn * dx + c * dz;
		}
		if (cudaMemcpyAsync(m_scene->buffers["lights"].pointer, out, floats * sizeof(float), cudaMemcpyHostToDevice,
				m_stream) != cudaSuccess || cudaEventRecord(m_orbitCopied[k], m_stream) != cudaSuccess)
		{
			return RESTIR_ERROR_LAUNCH;
		}
		return RESTIR_OK;
	}

	// createRenderTargets / createShadowMap (renderer.cpp:1240-1453).
	int ensureTargets(const RestirParams& P)
	{
		cudaStreamSynchronize(m_stream);
		releaseGraph();
		releaseTargets();
		m_width = P.width;
		m_height = P.height;
		m_giWidth = P.gi_width;
		m_giHeight = P.gi_height;
		m_faceSize = P.shadow_face_size;
		m_tableSize = P.grid_table_size;
		m_capacity = P.grid_cell_capacity;
		const uint64_t full = uint64_t(P.width) * P.height;
		const uint64_t gi = uint64_t(P.gi_width) * P.gi_height;
		const uint64_t grid = uint64_t(P.grid_table_size) * (2 + P.grid_cell_capacity) * 4;
		struct Spec
		{
			const char* name;
			uint64_t bytes;
		};
		const Spec specs[] = {
			{ "gbuffer.albedo", full * 4 }, { "gbuffer.normal", full * 4 }, { "gbuffer.emissive", full * 8 },
			{ "gbuffer.shading_normal", full * 4 }, { "gbuffer.depth", full * 4 },
			{ "shadow.atlas", 6ull * P.shadow_face_size * P.shadow_face_size * 4 },
			{ "di.sample0", full * 16 }, { "di.receiver0", full * 16 }, { "di.normal0", full * 8 },
			{ "di.sample1", full * 16 }, { "di.receiver1", full * 16 }, { "di.normal1", full * 8 },
			{ "di.diffuse", full * 8 }, { "di.specular", full * 8 }, { "black", full * 8 },
			{ "grid0", grid }, { "grid1", grid },
			{ "gi.sample0", gi * 16 }, { "gi.receiver0", gi * 16 }, { "gi.normal0", gi * 16 },
			{ "gi.sample1", gi * 16 }, { "gi.receiver1", gi * 16 }, { "gi.normal1", gi * 16 },
			{ "gi.color0", gi * 8 }, { "gi.color1", gi * 8 }, { "gi.moments0", gi * 8 }, { "gi.moments1", gi * 8 },
			{ "filtered0", gi * 8 }, { "filtered1", gi * 8 }, { "filter0", gi * 8 }, { "filter1", gi * 8 },
			{ "hdr", full * 8 }, { "reference.mean", full * 24 }, { "reference.alpha", full },
			{ "taa0", full * 8 }, { "taa1", full * 8 }, { "display", full * 4 }, { "exposure", 64 },
			{ "specular0", gi * 8 }, { "specular1", gi * 8 },
			{ "error.scratch", errorScratchBytes() }, { "error.out", 64 },
		};
		for (const Spec& s : specs)
		{
			Buffer b;
			b.bytes = s.bytes;
			if (cudaMalloc(&b.pointer, s.bytes) != cudaSuccess)
			{
				releaseTargets();
				return RESTIR_ERROR_OUT_OF_MEMORY;
			}
			cudaMemsetAsync(b.pointer, 0, s.bytes, m_stream);
			m_targets[s.name] = b;
		}
		m_historyRead = 0;
		m_diRead = 0;
		m_taaRead = 0;
		m_specularRead = 0;
		m_displayTaa = false;
		m_state.history_valid = 0;
		m_state.di_valid = 0;
		m_state.reference_frames = 0;
		m_state.frame_number = 0;
		m_state.taa_valid = 0;
		m_state.exposure_valid = 0;
		std::memset(m_state.previous_view_proj, 0, sizeof(m_state.previous_view_proj));
		for (int i = 0; i < 4; ++i)
		{
			m_state.previous_view_proj[i * 5] = 1.0f;
		}
		cudaStreamSynchronize(m_stream);
		return RESTIR_OK;
	}

	// The wavefront passes' ray queues: GI temporal's, sized by the candidate
	// count (a setting that keeps the history), and the specular pass's;
	// allocated before any capture.
	int ensureWorkspace(const RestirParams& P)
	{
		const int status = ensureBuffer("gi.workspace", m_settings.wavefront ? restir_gi_temporal_workspace_bytes(&P) : 0);
		if (status != RESTIR_OK)
		{
			return status;
		}
		return ensureBuffer("specular.workspace",
			m_settings.wavefront && m_settings.specular_gi ? restir_gi_specular_workspace_bytes(&P) : 0);
	}

	int ensureBuffer(const char* name, uint64_t needed)
	{
		auto found = m_targets.find(name);
		if (needed == 0 || (found != m_targets.end() && found->second.bytes >= needed))
		{
			return RESTIR_OK;
		}
		cudaStreamSynchronize(m_stream);
		releaseGraph();
		if (found != m_targets.end())
		{
			cudaFree(found->second.pointer);
			m_targets.erase(found);
		}
		Buffer b;
		b.bytes = needed;
		if (cudaMalloc(&b.pointer, needed) != cudaSuccess)
		{
			return RESTIR_ERROR_OUT_OF_MEMORY;
		}
		m_targets[name] = b;
		return RESTIR_OK;
	}

	bool targetsMatch(const RestirParams& P) const
	{
		return !m_targets.empty() && P.width == m_width && P.height == m_height && P.gi_width == m_giWidth
			&& P.gi_height == m_giHeight && P.shadow_face_size == m_faceSize && P.grid_table_size == m_tableSize
			&& P.grid_cell_capacity == m_capacity;
	}

public:
	// The per-frame state as a file (a debugging aid, no reference
	// counterpart): the carried state and history indices, then every frame
	// target (name, size, bytes) and the radiance cache's state when there is
	// one. Loading needs targets of the same sizes (a frame rendered first).
	static constexpr char kStateMagic[8] = { 'R', 'S', 'T', 'R', 'S', 'T', '0', '1' };

	struct StateHeader
	{
		char magic[8];
		RestirFrameState state;
		int32_t historyRead, diRead, taaRead, specularRead, displayTaa;
		double orbitTime;
		uint32_t width, height, giWidth, giHeight, faceSize, tableSize, capacity;
		uint32_t buffers;
	};

	std::vector<std::pair<std::string, Buffer>> stateBuffers()
	{
		std::vector<std::pair<std::string, Buffer>> list(m_targets.begin(), m_targets.end());
		auto cache = m_scene->buffers.find("cache.state");
		if (cache != m_scene->buffers.end() && cache->second.pointer != nullptr)
		{
			list.emplace_back("cache.state", cache->second);
		}
		return list;
	}

	void synchronizeAll()
	{
		cudaStreamSynchronize(m_stream);
		cudaStreamSynchronize(m_side);
		cudaStreamSynchronize(m_aside);
	}

	int saveState(const char* path)
	{
		if (path == nullptr || m_targets.empty())
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		synchronizeAll();
		FILE* file = std::fopen(path, "wb");
		if (file == nullptr)
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		const auto list = stateBuffers();
		StateHeader h = {};
		std::memcpy(h.magic, kStateMagic, sizeof(h.magic));
		h.state = m_state;
		h.historyRead = m_historyRead;
		h.diRead = m_diRead;
		h.taaRead = m_taaRead;
		h.specularRead = m_specularRead;
		h.displayTaa = m_displayTaa ? 1 : 0;
		h.orbitTime = m_orbitTime;
		h.width = m_width;
		h.height = m_height;
		h.giWidth = m_giWidth;
		h.giHeight = m_giHeight;
		h.faceSize = m_faceSize;
		h.tableSize = m_tableSize;
		h.capacity = m_capacity;
		h.buffers = uint32_t(list.size());
		bool ok = std::fwrite(&h, sizeof(h), 1, file) == 1;
		std::vector<char> host;
		for (const auto& entry : list)
		{
			const uint32_t length = uint32_t(entry.first.size());
			const uint64_t bytes = entry.second.bytes;
			host.resize(bytes);
			ok = ok && cudaMemcpy(host.data(), entry.second.pointer, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
			ok = ok && std::fwrite(&length, sizeof(length), 1, file) == 1
				&& std::fwrite(entry.first.data(), 1, length, file) == length
				&& std::fwrite(&bytes, sizeof(bytes), 1, file) == 1
				&& std::fwrite(host.data(), 1, bytes, file) == bytes;
		}
		ok = std::fclose(file) == 0 && ok;
		return ok ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
	}

	int loadState(const char* path)
	{
		if (path == nullptr || m_targets.empty())
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		synchronizeAll();
		FILE* file = std::fopen(path, "rb");
		if (file == nullptr)
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		StateHeader h = {};
		const auto list = stateBuffers();
		bool ok = std::fread(&h, sizeof(h), 1, file) == 1 && std::memcmp(h.magic, kStateMagic, sizeof(h.magic)) == 0
			&& h.width == m_width && h.height == m_height && h.giWidth == m_giWidth && h.giHeight == m_giHeight
			&& h.faceSize == m_faceSize && h.tableSize == m_tableSize && h.capacity == m_capacity
			&& h.buffers == uint32_t(list.size());
		std::vector<char> host;
		for (uint32_t k = 0; ok && k < h.buffers; ++k)
		{
			uint32_t length = 0;
			uint64_t bytes = 0;
			std::string name;
			ok = std::fread(&length, sizeof(length), 1, file) == 1 && length < 256u;
			if (ok)
			{
				name.resize(length);
				ok = std::fread(&name[0], 1, length, file) == length && std::fread(&bytes, sizeof(bytes), 1, file) == 1;
			}
			ok = ok && name == list[k].first && bytes == list[k].second.bytes;
			if (ok)
			{
				host.resize(bytes);
				ok = std::fread(host.data(), 1, bytes, file) == bytes
					&& cudaMemcpy(list[k].second.pointer, host.data(), bytes, cudaMemcpyHostToDevice) == cudaSuccess;
			}
		}
		std::fclose(file);
		if (!ok)
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		m_state = h.state;
		m_historyRead = h.historyRead;
		m_diRead = h.diRead;
		m_taaRead = h.taaRead;
		m_specularRead = h.specularRead;
		m_displayTaa = h.displayTaa != 0;
		m_orbitTime = h.orbitTime;
		releaseGraph(); // the captured frame reads the history it was recorded with
		return RESTIR_OK;
	}

private:
	// A pass's edges: its CUDA events (timed frames) and an NVTX range around
	// its launches on the host (the pass groups of the reference's profiler,
	// renderer.h:45-60), which a timeline profiler shows; without one attached
	// NVTX does nothing.
	static const char* passName(int pass)
	{
		static const char* const kNames[RESTIR_PASS_COUNT] = { "shadow", "gbuffer", "di_temporal", "di_spatial", "grid",
			"gi_temporal", "gi_spatial", "denoise", "composite", "reference", "cache", "display", "specular" };
		return pass >= 0 && pass < RESTIR_PASS_COUNT ? kNames[pass] : "pass";
	}

	void mark(int pass, int edge, bool events)
	{
		if (edge == 0)
		{
			nvtxRangePushA(passName(pass));
		}
		if (events)
		{
			cudaEventRecord(m_events[m_slot][pass][edge], m_stream);
		}
		if (edge == 1)
		{
			nvtxRangePop();
		}
	}

	// The passes of one frame, in the reference's order (renderer.cpp:527-1077).
	// part: the whole frame, or (for a batch of views sharing one ray queue)
	// the passes up to the GI candidates, or the GI shading and the rest.
	static constexpr int kWholeFrame = 0, kBeforeTrace = 1, kAfterTrace = 2;
	int enqueue(bool events, int part = kWholeFrame)
	{
		const bool before = part != kAfterTrace;
		const bool after = part != kBeforeTrace;
		const RestirParams& P = m_params;
		const RestirFramePlan& plan = m_plan;
		const int hw = 1 - m_historyRead, hr = m_historyRead, dw = 1 - m_diRead, dr = m_diRead;
		const std::string H = std::to_string(hw), R = std::to_string(hr);
		RestirScene scene = {};
		scene.bvh = static_cast<const float*>(m_scene->buffers["bvh"].pointer);
		scene.node_count = m_scene->bvh.nodeCount;
		scene.triangle_offset = m_scene->bvh.triangleOffset;
		scene.triangle_count = m_scene->bvh.triangleCount;
		scene.lights = static_cast<const float*>(m_scene->buffers["lights"].pointer);
		scene.light_count = m_scene->lights.count;
		scene.triangle_normals = static_cast<const float*>(m_scene->buffers["normals"].pointer);
		scene.materials = static_cast<const float*>(m_scene->buffers["materials"].pointer);
		scene.material_count = uint32_t(m_scene->mesh.materials.size());
		RestirGBuffer gb = { p<uint8_t>("gbuffer.albedo"), p<uint8_t>("gbuffer.normal"), p<uint16_t>("gbuffer.emissive"),
			p<uint8_t>("gbuffer.shading_normal"), p<float>("gbuffer.depth") };
		void* s = m_stream;
		int status = RESTIR_OK;
		for (bool& ran : m_passRan[m_slot])
		{
			ran = false;
		}
		auto run = [&](int pass, auto&& body)
		{
			mark(pass, 0, events);
			status |= body();
			m_passRan[m_slot][pass] = true;
			mark(pass, 1, events);
			if (m_profile != nullptr)
			{
				// restir_counters waits for the device: this pass's work only.
				uint64_t counts[8];
				restir_counters(1, counts);
				for (int k = 0; k < 8; ++k)
				{
					m_profile[pass * 8 + k] += counts[k];
				}
			}
		};
		// Two passes run on a second stream beside the main chain: the shadow
		// atlas (first read by the GI passes) beside the G-buffer and the DI
		// passes, and the specular pass (it reads last frame's GI history and
		// this frame's DI output, nothing the GI passes or the denoiser write)
		// beside the GI passes and the denoiser. Not in a profiling frame (its
		// counters wait pass by pass) nor in a batch's parts.
		const bool overlap = part == kWholeFrame && m_profile == nullptr;
		auto runAside = [&](int pass, cudaEvent_t join, auto&& body)
		{
			cudaEventRecord(m_asideFork, m_stream);
			cudaStreamWaitEvent(m_aside, m_asideFork, 0);
			if (events)
			{
				cudaEventRecord(m_events[m_slot][pass][0], m_aside);
			}
			nvtxRangePushA(passName(pass));
			status |= body(static_cast<void*>(m_aside));
			nvtxRangePop();
			m_passRan[m_slot][pass] = true;
			if (events)
			{
				cudaEventRecord(m_events[m_slot][pass][1], m_aside);
			}
			cudaEventRecord(join, m_aside);
		};
		bool shadowPending = false;
		bool specularPending = false;
		auto needAtlas = [&]()
		{
			if (shadowPending)
			{
				cudaStreamWaitEvent(m_stream, m_shadowJoin, 0);
				shadowPending = false;
			}
		};
		// A batch draws the shadow atlas once for all its views (it depends on the light and scene only).
		float* atlas = m_sharedAtlas != nullptr ? m_sharedAtlas : p<float>("shadow.atlas");
		if (before && m_sharedAtlas == nullptr)
		{
			if (overlap)
			{
				runAside(RESTIR_PASS_SHADOW, m_shadowJoin, [&](void* st) { return restir_shadow_atlas(&P, &scene, atlas, st); });
				shadowPending = true;
			}
			else
			{
				run(RESTIR_PASS_SHADOW, [&] { return restir_shadow_atlas(&P, &scene, atlas, s); });
			}
		}
		if (before)
		{
			run(RESTIR_PASS_GBUFFER, [&] { return restir_gbuffer_primary(&P, &scene, &gb, s); });
		}
		const bool cached = P.radiance_cache > 0.5f;
		void* cacheState = m_scene->buffers["cache.state"].pointer;
		// The cache's training only reads the G-buffer, the shadow atlas and the
		// cache: it runs on a side stream, forked once the frame's queries are
		// enqueued (so they all see the same weights) and joined before the
		// frame ends, overlapping the passes in between. A profiling frame keeps
		// it on the main stream (its counters wait pass by pass).
		bool joinSide = false;
		auto train = [&]()
		{
			needAtlas();
			const Buffer& w = m_targets["gi.workspace"];
			if (m_profile != nullptr)
			{
				run(RESTIR_PASS_CACHE, [&] {
					return restir_cache_train_frame(&P, &scene, &gb, atlas, &m_scene->cacheConfig, cacheState, w.pointer,
						w.bytes, s);
				});
				return;
			}
			cudaEventRecord(m_fork, m_stream);
			cudaStreamWaitEvent(m_side, m_fork, 0);
			if (events)
			{
				cudaEventRecord(m_events[m_slot][RESTIR_PASS_CACHE][0], m_side);
			}
			status |= restir_cache_train_frame(&P, &scene, &gb, atlas, &m_scene->cacheConfig, cacheState, w.pointer, w.bytes,
				m_side);
			m_passRan[m_slot][RESTIR_PASS_CACHE] = true;
			if (events)
			{
				cudaEventRecord(m_events[m_slot][RESTIR_PASS_CACHE][1], m_side);
			}
			cudaEventRecord(m_join, m_side);
			joinSide = true;
		};
		if (plan.gi_from_cache && part == kWholeFrame)
		{
			// The cache-only form's GI needs only the G-buffer: its queries first,
			// then the training overlaps the DI passes.
			RestirGiReservoirs current = { p<float>("gi.sample" + H), p<float>("gi.receiver" + H), p<float>("gi.normal" + H) };
			needAtlas();
			run(RESTIR_PASS_GI_TEMPORAL, [&] {
				const Buffer& w = m_targets["gi.workspace"];
				return restir_gi_from_cache(&P, &scene, &gb, &m_scene->cacheConfig, cacheState, w.pointer, w.bytes, &current,
					p<uint16_t>("gi.color" + H), p<uint16_t>("gi.moments" + H), s);
			});
			train();
		}
		const std::string DW = std::to_string(dw), DR = std::to_string(dr);
		RestirDiReservoirs diPrevious = { p<float>("di.sample" + DR), p<float>("di.receiver" + DR), p<uint16_t>("di.normal" + DR) };
		RestirDiReservoirs diCurrent = { p<float>("di.sample" + DW), p<float>("di.receiver" + DW), p<uint16_t>("di.normal" + DW) };
		if (before && plan.di_active)
		{
			run(RESTIR_PASS_DI_TEMPORAL, [&] { return restir_di_temporal(&P, &scene, &gb, &diPrevious, &diCurrent, s); });
			run(RESTIR_PASS_DI_SPATIAL, [&] {
				return restir_di_spatial(&P, &scene, &gb, &diCurrent, p<uint16_t>("di.diffuse"), p<uint16_t>("di.specular"), s);
			});
		}
		const uint16_t* surface = plan.surface_light_is_di ? (plan.di_active ? p<uint16_t>("di.diffuse") : p<uint16_t>("black"))
			: p<uint16_t>("gbuffer.emissive");
		uint32_t* gridWrite = p<uint32_t>("grid" + H);
		RestirGiHistory history = { p<float>("gi.sample" + R), p<float>("gi.receiver" + R), p<float>("gi.normal" + R),
			plan.denoiser ? p<uint16_t>("filtered" + R) : p<uint16_t>("gi.color" + R), p<uint16_t>("gi.moments" + R) };
		const std::string specularRead = "specular" + std::to_string(m_specularRead);
		const std::string specularWrite = "specular" + std::to_string(1 - m_specularRead);
		auto specular = [&](void* st)
		{
			if (m_settings.wavefront)
			{
				const Buffer& w = m_targets["specular.workspace"];
				return restir_gi_specular_wavefront(&P, &scene, &gb, &history, atlas, surface, p<uint16_t>("hdr"),
					p<uint16_t>(specularRead), p<uint16_t>(specularWrite), w.pointer, w.bytes, st);
			}
			return restir_gi_specular(&P, &scene, &gb, &history, atlas, surface, p<uint16_t>("hdr"),
				p<uint16_t>(specularRead), p<uint16_t>(specularWrite), st);
		};
		if (plan.specular && overlap)
		{
			// Indirect specular (renderer.cpp:835-855): last frame's composite and specular history.
			runAside(RESTIR_PASS_SPECULAR, m_specularJoin, specular);
			specularPending = true;
		}
		if (before && !plan.gi_from_cache)
		{
			run(RESTIR_PASS_GRID, [&] {
				return restir_grid_clear(&P, gridWrite, s) | restir_grid_insert(&P, &gb, gridWrite, s);
			});
		}
		RestirGiReservoirs current = { p<float>("gi.sample" + H), p<float>("gi.receiver" + H), p<float>("gi.normal" + H) };
		needAtlas();
		if (part != kWholeFrame)
		{
			// The batch's shared ray queue: candidates before its one tracer launch, shading after.
			const Buffer& r = m_targets["gi.records"];
			run(RESTIR_PASS_GI_TEMPORAL, [&] {
				return part == kBeforeTrace
					? restir_gi_temporal_candidates(&P, &scene, &gb, &history, p<uint32_t>("grid" + R), atlas, surface, r.pointer,
						r.bytes, m_batchQueue, m_batchQueueCapacity, s)
					: restir_gi_temporal_shade(&P, &scene, &gb, &history, p<uint32_t>("grid" + R), atlas, surface, &current,
						r.pointer, r.bytes, m_batchQueue, m_batchQueueCapacity, s);
			});
		}
		else if (!plan.gi_from_cache) run(RESTIR_PASS_GI_TEMPORAL, [&] {
			const Buffer& w = m_targets["gi.workspace"];
			if (cached)
			{
				return restir_gi_temporal_cached(&P, &scene, &gb, &history, p<uint32_t>("grid" + R), atlas,
					surface, &current, &m_scene->cacheConfig, cacheState, w.pointer, w.bytes, s);
			}
			if (m_settings.wavefront)
			{
				return restir_gi_temporal_wavefront(&P, &scene, &gb, &history, p<uint32_t>("grid" + R), atlas,
					surface, &current, w.pointer, w.bytes, s);
			}
			return restir_gi_temporal(&P, &scene, &gb, &history, p<uint32_t>("grid" + R), atlas, surface,
				&current, s);
		});
		if (!after)
		{
			return status == RESTIR_OK ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
		}
		if (!plan.gi_from_cache) run(RESTIR_PASS_GI_SPATIAL, [&] {
			if (cached)
			{
				const Buffer& w = m_targets["gi.workspace"];
				return restir_gi_spatial_cached(&P, &scene, &gb, &current, gridWrite, &history, atlas, surface,
					p<uint16_t>("gi.color" + H), p<uint16_t>("gi.moments" + H), &m_scene->cacheConfig, cacheState, w.pointer, w.bytes, s);
			}
			return restir_gi_spatial(&P, &scene, &gb, &current, gridWrite, &history, atlas, surface,
				p<uint16_t>("gi.color" + H), p<uint16_t>("gi.moments" + H), s);
		});
		if (plan.specular && !overlap)
		{
			run(RESTIR_PASS_SPECULAR, [&] { return specular(s); });
		}
		if (cached && !plan.gi_from_cache)
		{
			// Training after the frame's queries: every query of a frame sees the same weights.
			train();
		}
		std::string denoised = "gi.color" + H;
		if (plan.denoiser)
		{
			run(RESTIR_PASS_DENOISE, [&] {
				int st = restir_svgf_variance(&P, p<uint16_t>("gi.color" + H), p<uint16_t>("gi.moments" + H),
					p<float>("gi.receiver" + H), p<float>("gi.normal" + H), p<uint16_t>("filter0"), s);
				for (int it = 0; it < plan.atrous_iterations; ++it)
				{
					const std::string src = it == 0 ? "filter0" : (it == 1 ? "filtered" + H : "filter" + std::to_string((it - 1) & 1));
					const std::string dst = it == 0 ? "filtered" + H : "filter" + std::to_string(it & 1);
					st |= restir_svgf_atrous(&P, 1 << it, p<uint16_t>(src), p<float>("gi.receiver" + H), p<float>("gi.normal" + H),
						p<uint16_t>(dst), s);
					denoised = dst;
				}
				return st;
			});
		}
		const uint16_t* diDiffuse = plan.di_active ? p<uint16_t>("di.diffuse") : p<uint16_t>("black");
		const uint16_t* diSpecular = plan.di_active ? p<uint16_t>("di.specular") : p<uint16_t>("black");
		if (specularPending)
		{
			cudaStreamWaitEvent(m_stream, m_specularJoin, 0);
		}
		run(RESTIR_PASS_COMPOSITE, [&] {
			return restir_composite_specular(&P, &gb, atlas, p<uint16_t>(denoised), diDiffuse, diSpecular,
				plan.specular ? p<uint16_t>(specularWrite) : nullptr, p<uint16_t>("hdr"), s);
		});
		if (plan.reference_accumulate)
		{
			run(RESTIR_PASS_REFERENCE, [&] {
				return restir_reference_accumulate(&P, p<uint16_t>("hdr"), p<double>("reference.mean"),
					p<uint8_t>("reference.alpha"), plan.reference_weight_frames, s);
			});
		}
		if (plan.display)
		{
			// Auto exposure, TAA and tone mapping (renderer.cpp:987-1117).
			RestirDisplayParams D;
			status |= restir_display_params(P.inv_view_proj, m_state.previous_unjittered_view_proj, P.width, P.height,
				plan.taa, m_state.taa_valid, plan.exposure, m_state.exposure_valid, m_settings.adaptation_speed,
				m_deltaTime, m_settings.exposure_ev, m_settings.tonemapper, 0, 0, &D);
			const std::string taaRead = "taa" + std::to_string(m_taaRead), taaWrite = "taa" + std::to_string(1 - m_taaRead);
			run(RESTIR_PASS_DISPLAY, [&] {
				return restir_display(&D, p<uint16_t>("hdr"), p<float>("gbuffer.depth"), p<uint16_t>(taaRead),
					p<uint16_t>(taaWrite), p<uint32_t>("exposure"), nullptr, nullptr, p<uint8_t>("display"), s);
			});
		}
		if (joinSide)
		{
			cudaStreamWaitEvent(m_stream, m_join, 0);
		}
		return status == RESTIR_OK ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
	}

	int renderGraph()
	{
		cudaGraph_t graph = nullptr;
		if (cudaStreamBeginCapture(m_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
		{
			return RESTIR_ERROR_LAUNCH;
		}
		int status = enqueue(false);
		if (cudaStreamEndCapture(m_stream, &graph) != cudaSuccess || status != RESTIR_OK)
		{
			if (graph)
			{
				cudaGraphDestroy(graph);
			}
			return RESTIR_ERROR_LAUNCH;
		}
		bool updated = false;
		if (m_graphExec != nullptr)
		{
			cudaGraphExecUpdateResultInfo info;
			updated = cudaGraphExecUpdate(m_graphExec, graph, &info) == cudaSuccess;
			if (!updated)
			{
				cudaGetLastError();
				cudaGraphExecDestroy(m_graphExec);
				m_graphExec = nullptr;
			}
		}
		// Each kernel node keeps the priority of the stream it was captured on (the main
		// chain high, the side passes low), as the stream-launched frame runs them.
		if (!updated && cudaGraphInstantiate(&m_graphExec, graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess)
		{
			cudaGraphDestroy(graph);
			m_graphExec = nullptr;
			return RESTIR_ERROR_LAUNCH;
		}
		cudaGraphDestroy(graph);
		return cudaGraphLaunch(m_graphExec, m_stream) == cudaSuccess ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
	}

	void releaseGraph()
	{
		if (m_graphExec != nullptr)
		{
			cudaGraphExecDestroy(m_graphExec);
			m_graphExec = nullptr;
		}
	}

	void releaseTargets()
	{
		for (auto& kv : m_targets)
		{
			cudaFree(kv.second.pointer);
		}
		m_targets.clear();
	}

	// A fresh, empty scene; the previous one is freed when no renderer holds it.
	void releaseScene()
	{
		m_scene = std::make_shared<SceneState>();
	}

	RestirSettings m_settings;
	RestirFrameState m_state;
	RestirParams m_params = {};
	RestirFramePlan m_plan = {};
	RestirFrameInput m_referenceInput = {};
	// Orbiting extra lights: accumulated time, two pinned host copies of the moved list.
	double m_orbitTime = 0.0;
	float* m_orbitHost[2] = { nullptr, nullptr };
	size_t m_orbitCapacity[2] = { 0, 0 };
	cudaEvent_t m_orbitCopied[2] = {};
	int m_orbitSlot = 0;
	std::shared_ptr<SceneState> m_scene = std::make_shared<SceneState>();
	// Set by a batch: the shared shadow atlas and ray queue.
	float* m_sharedAtlas = nullptr;
	void* m_batchQueue = nullptr;
	uint32_t m_batchQueueCapacity = 0;
	std::map<std::string, Buffer> m_targets;
	uint32_t m_width = 0, m_height = 0, m_giWidth = 0, m_giHeight = 0, m_faceSize = 0, m_tableSize = 0, m_capacity = 0;
	int m_historyRead = 0;
	int m_diRead = 0;
	float m_deltaTime = 0.0f; // the frame input's delta_time (auto exposure)
	int m_taaRead = 0;        // the TAA target holding last frame's output
	int m_specularRead = 0;   // the specular target holding last frame's output
	bool m_displayTaa = false; // the last frame's displayed HDR is its TAA output
	bool m_timed = false;
	// Per-pass events of the last kEventRing stream-launched frames.
	static constexpr uint32_t kEventRing = 128;
	bool m_passRan[kEventRing][RESTIR_PASS_COUNT] = {};
	cudaEvent_t m_events[kEventRing][RESTIR_PASS_COUNT][2] = {};  // start, end of each pass
	uint32_t m_slot = 0;
	uint32_t m_lastSlot = 0;
	uint32_t m_timedFrames = 0;
	cudaStream_t m_stream = nullptr;
	cudaStream_t m_side = nullptr;   // the cache's training, overlapping the rest of the frame
	cudaEvent_t m_fork = nullptr, m_join = nullptr;
	cudaStream_t m_aside = nullptr;  // the shadow atlas and the specular pass, beside the main chain
	cudaEvent_t m_asideFork = nullptr, m_shadowJoin = nullptr, m_specularJoin = nullptr;
	cudaGraphExec_t m_graphExec = nullptr;
	double* m_errorHost = nullptr;
	uint64_t* m_profile = nullptr;
};

// Several views of one scene rendered as one frame (no reference
// counterpart): the views share the scene's buffers, one shadow atlas (it
// depends on the light and the scene only) and one GI ray queue that a single
// persistent tracer launch drains; the frame is captured as one CUDA graph in
// which each view's passes run on its own stream, so that small views fill
// the GPU together. Every view's output equals what a Renderer of that view
// alone produces.
class Batch
{
public:
	Batch(const RestirSettings& settings, uint32_t views)
	{
		RestirSettings s = settings;
		s.radiance_cache = 0;  // the batch path runs the plain GI passes
		s.wavefront = 1;
		for (uint32_t v = 0; v < views; ++v)
		{
			m_views.push_back(new (std::nothrow) Renderer(s));
		}
		cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking);
		cudaEventCreateWithFlags(&m_fork, cudaEventDisableTiming);
		cudaEventCreateWithFlags(&m_traced, cudaEventDisableTiming);
		m_joins.resize(2 * views);
		for (cudaEvent_t& e : m_joins)
		{
			cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
		}
		m_tuning.tracer_threads = 128;
		m_tuning.tracer_blocks_per_sm = 0;
		m_tuning.ms_per_frame = 0.0f;
	}

	~Batch()
	{
		synchronize();
		if (m_graphExec != nullptr)
		{
			cudaGraphExecDestroy(m_graphExec);
		}
		for (Renderer* r : m_views)
		{
			delete r;
		}
		cudaFree(m_queue);
		cudaFree(m_atlas);
		for (cudaEvent_t e : m_joins)
		{
			cudaEventDestroy(e);
		}
		cudaEventDestroy(m_fork);
		cudaEventDestroy(m_traced);
		cudaStreamDestroy(m_stream);
	}

	bool valid() const
	{
		for (Renderer* r : m_views)
		{
			if (r == nullptr)
			{
				return false;
			}
		}
		return !m_views.empty() && m_stream != nullptr;
	}

	uint32_t views() const { return uint32_t(m_views.size()); }
	Renderer& view(uint32_t v) { return *m_views[v]; }
	cudaStream_t stream() const { return m_stream; }
	const RestirBatchTuning& tuning() const { return m_tuning; }

	int setTuning(const RestirBatchTuning& t)
	{
		if (t.tracer_threads != 64 && t.tracer_threads != 128 && t.tracer_threads != 256)
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		m_tuning.tracer_threads = t.tracer_threads;
		m_tuning.tracer_blocks_per_sm = t.tracer_blocks_per_sm;
		return RESTIR_OK;
	}

	int setScene(const Mesh& mesh, bool useSceneDefaults)
	{
		synchronize();
		int status = m_views[0]->setScene(mesh, useSceneDefaults);
		for (uint32_t v = 1; v < views() && status == RESTIR_OK; ++v)
		{
			status = m_views[v]->setSettings(m_views[0]->settings());
			m_views[v]->shareScene(*m_views[0]);
		}
		return status;
	}

	int setSettings(const RestirSettings& settings)
	{
		RestirSettings s = settings;
		s.radiance_cache = 0;
		s.wavefront = 1;
		int status = RESTIR_OK;
		for (Renderer* r : m_views)
		{
			status |= r->setSettings(s);
		}
		return status == RESTIR_OK ? RESTIR_OK : RESTIR_ERROR_INVALID_ARGUMENT;
	}

	int render(const RestirFrameInput* inputs)
	{
		uint32_t rays = 0;
		for (uint32_t v = 0; v < views(); ++v)
		{
			int status = m_views[v]->prepare(inputs[v]);
			if (status == RESTIR_OK)
			{
				status = m_views[v]->ensureRecords();
			}
			if (status != RESTIR_OK)
			{
				return status;
			}
			rays += m_views[v]->candidateRays();
		}
		const RestirParams& first = m_views[0]->params();
		int status = ensureShared(rays, 6ull * first.shadow_face_size * first.shadow_face_size * 4);
		if (status != RESTIR_OK)
		{
			return status;
		}
		for (Renderer* r : m_views)
		{
			r->setBatch(m_atlas, m_queue, m_queueCapacity);
		}
		status = launchFrame();
		if (status != RESTIR_OK)
		{
			return status;
		}
		for (uint32_t v = 0; v < views(); ++v)
		{
			m_views[v]->advance(inputs[v]);
		}
		return RESTIR_OK;
	}

	// Tries tracer shapes (threads per block x resident blocks per SM) on
	// `frames` frames each and keeps the fastest (device time of the whole
	// batch frame, CUDA events on the batch stream).
	int autotune(const RestirFrameInput* inputs, uint32_t frames, RestirBatchTuning* best)
	{
		static const uint32_t shapes[][2] = { { 128, 0 }, { 64, 0 }, { 256, 0 }, { 128, 4 }, { 128, 2 }, { 256, 2 } };
		cudaEvent_t start, stop;
		cudaEventCreate(&start);
		cudaEventCreate(&stop);
		RestirBatchTuning winner = m_tuning;
		winner.ms_per_frame = 0.0f;
		int status = RESTIR_OK;
		for (const auto& shape : shapes)
		{
			m_tuning.tracer_threads = shape[0];
			m_tuning.tracer_blocks_per_sm = shape[1];
			status = render(inputs);  // warm: capture, instantiate
			cudaEventRecord(start, m_stream);
			for (uint32_t f = 0; f < frames && status == RESTIR_OK; ++f)
			{
				status = render(inputs);
			}
			cudaEventRecord(stop, m_stream);
			if (status != RESTIR_OK || cudaEventSynchronize(stop) != cudaSuccess)
			{
				status = status != RESTIR_OK ? status : RESTIR_ERROR_LAUNCH;
				break;
			}
			float ms = 0.0f;
			cudaEventElapsedTime(&ms, start, stop);
			ms /= float(frames > 0 ? frames : 1);
			if (winner.ms_per_frame == 0.0f || ms < winner.ms_per_frame)
			{
				winner.tracer_threads = shape[0];
				winner.tracer_blocks_per_sm = shape[1];
				winner.ms_per_frame = ms;
			}
		}
		cudaEventDestroy(start);
		cudaEventDestroy(stop);
		m_tuning = winner;
		if (best != nullptr)
		{
			*best = winner;
		}
		return status;
	}

	int synchronize()
	{
		int status = cudaStreamSynchronize(m_stream) == cudaSuccess ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
		for (Renderer* r : m_views)
		{
			if (r != nullptr && cudaStreamSynchronize(r->stream()) != cudaSuccess)
			{
				status = RESTIR_ERROR_LAUNCH;
			}
		}
		return status;
	}

private:
	int ensureShared(uint32_t rays, uint64_t atlasBytes)
	{
		if (rays > m_queueCapacity || m_queue == nullptr)
		{
			synchronize();
			releaseGraph();
			cudaFree(m_queue);
			m_queue = nullptr;
			if (cudaMalloc(&m_queue, restir_ray_queue_bytes(rays)) != cudaSuccess)
			{
				m_queueCapacity = 0;
				m_queue = nullptr;
				return RESTIR_ERROR_OUT_OF_MEMORY;
			}
			m_queueCapacity = rays;
		}
		if (atlasBytes > m_atlasBytes || m_atlas == nullptr)
		{
			synchronize();
			releaseGraph();
			cudaFree(m_atlas);
			m_atlas = nullptr;
			if (cudaMalloc(reinterpret_cast<void**>(&m_atlas), atlasBytes) != cudaSuccess)
			{
				m_atlasBytes = 0;
				return RESTIR_ERROR_OUT_OF_MEMORY;
			}
			m_atlasBytes = atlasBytes;
		}
		return RESTIR_OK;
	}

	// The frame as one graph: queue reset and the shared atlas, then every
	// view's passes up to its GI candidates on its own stream, the one tracer
	// launch, every view's GI shading and later passes.
	int launchFrame()
	{
		RestirScene scene = m_views[0]->deviceScene();
		const RestirParams& first = m_views[0]->params();
		cudaGraph_t graph = nullptr;
		if (cudaStreamBeginCapture(m_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
		{
			return RESTIR_ERROR_LAUNCH;
		}
		int status = restir_ray_queue_reset(m_queue, m_stream);
		status |= restir_shadow_atlas(&first, &scene, m_atlas, m_stream);
		cudaEventRecord(m_fork, m_stream);
		for (uint32_t v = 0; v < views(); ++v)
		{
			cudaStream_t s = m_views[v]->stream();
			cudaStreamWaitEvent(s, m_fork, 0);
			status |= m_views[v]->enqueue(false, Renderer::kBeforeTrace);
			cudaEventRecord(m_joins[2 * v], s);
			cudaStreamWaitEvent(m_stream, m_joins[2 * v], 0);
		}
		status |= restir_trace_queue(&scene, m_queue, m_queueCapacity, m_tuning.tracer_threads, m_tuning.tracer_blocks_per_sm,
			m_stream);
		cudaEventRecord(m_traced, m_stream);
		for (uint32_t v = 0; v < views(); ++v)
		{
			cudaStream_t s = m_views[v]->stream();
			cudaStreamWaitEvent(s, m_traced, 0);
			status |= m_views[v]->enqueue(false, Renderer::kAfterTrace);
			cudaEventRecord(m_joins[2 * v + 1], s);
			cudaStreamWaitEvent(m_stream, m_joins[2 * v + 1], 0);
		}
		if (cudaStreamEndCapture(m_stream, &graph) != cudaSuccess || status != RESTIR_OK)
		{
			if (graph != nullptr)
			{
				cudaGraphDestroy(graph);
			}
			cudaGetLastError();
			return RESTIR_ERROR_LAUNCH;
		}
		bool updated = false;
		if (m_graphExec != nullptr)
		{
			cudaGraphExecUpdateResultInfo info;
			updated = cudaGraphExecUpdate(m_graphExec, graph, &info) == cudaSuccess;
			if (!updated)
			{
				cudaGetLastError();
				cudaGraphExecDestroy(m_graphExec);
				m_graphExec = nullptr;
			}
		}
		// Each kernel node keeps the priority of the stream it was captured on (the main
		// chain high, the side passes low), as the stream-launched frame runs them.
		if (!updated && cudaGraphInstantiate(&m_graphExec, graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess)
		{
			cudaGraphDestroy(graph);
			m_graphExec = nullptr;
			return RESTIR_ERROR_LAUNCH;
		}
		cudaGraphDestroy(graph);
		return cudaGraphLaunch(m_graphExec, m_stream) == cudaSuccess ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
	}

	void releaseGraph()
	{
		if (m_graphExec != nullptr)
		{
			cudaGraphExecDestroy(m_graphExec);
			m_graphExec = nullptr;
		}
	}

	std::vector<Renderer*> m_views;
	cudaStream_t m_stream = nullptr;
	cudaEvent_t m_fork = nullptr;
	cudaEvent_t m_traced = nullptr;
	std::vector<cudaEvent_t> m_joins;
	cudaGraphExec_t m_graphExec = nullptr;
	void* m_queue = nullptr;
	uint32_t m_queueCapacity = 0;
	float* m_atlas = nullptr;
	uint64_t m_atlasBytes = 0;
	RestirBatchTuning m_tuning = {};
};

} // namespace
} // namespace restir

using restir::Batch;
using restir::Renderer;

extern "C" void* restir_renderer_create(const RestirSettings* settings)
{
	RestirSettings s;
	if (settings != nullptr)
	{
		s = *settings;
	}
	else
	{
		restir_settings_default(&s);
	}
	return new (std::nothrow) Renderer(s);
}

extern "C" void restir_renderer_destroy(void* renderer)
{
	delete static_cast<Renderer*>(renderer);
}

extern "C" int restir_renderer_set_scene(void* renderer, void* mesh, int use_scene_defaults)
{
	if (renderer == nullptr || mesh == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->setScene(*static_cast<restir::Mesh*>(mesh), use_scene_defaults != 0);
}

extern "C" int restir_renderer_set_settings(void* renderer, const RestirSettings* settings)
{
	if (renderer == nullptr || settings == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->setSettings(*settings);
}

extern "C" int restir_renderer_get_settings(void* renderer, RestirSettings* settings)
{
	if (renderer == nullptr || settings == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	*settings = static_cast<Renderer*>(renderer)->settings();
	return RESTIR_OK;
}

extern "C" int restir_renderer_render(void* renderer, const RestirFrameInput* input)
{
	if (renderer == nullptr || input == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->render(*input, false);
}

extern "C" int restir_renderer_render_graph(void* renderer, const RestirFrameInput* input)
{
	if (renderer == nullptr || input == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->render(*input, true);
}

extern "C" int restir_renderer_measure(void* renderer, RestirMetrics* metrics)
{
	if (renderer == nullptr || metrics == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->measure(metrics);
}

extern "C" int restir_renderer_pass_history(void* renderer, uint32_t frames, float* ms)
{
	if (renderer == nullptr || ms == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->passHistory(frames, ms);
}

extern "C" int restir_renderer_profile_frame(void* renderer, const RestirFrameInput* input, uint64_t* counts)
{
	if (renderer == nullptr || input == nullptr || counts == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->profile(*input, counts);
}

extern "C" void restir_renderer_set_reference_accumulation(void* renderer, int accumulate)
{
	if (renderer != nullptr)
	{
		static_cast<Renderer*>(renderer)->setReferenceAccumulation(accumulate != 0);
	}
}

extern "C" void restir_renderer_invalidate_history(void* renderer)
{
	if (renderer != nullptr)
	{
		static_cast<Renderer*>(renderer)->invalidateHistory();
	}
}

extern "C" int restir_renderer_synchronize(void* renderer)
{
	if (renderer == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return cudaStreamSynchronize(static_cast<Renderer*>(renderer)->stream()) == cudaSuccess ? RESTIR_OK : RESTIR_ERROR_LAUNCH;
}

extern "C" void* restir_renderer_stream(void* renderer)
{
	return renderer != nullptr ? static_cast<void*>(static_cast<Renderer*>(renderer)->stream()) : nullptr;
}

extern "C" int restir_renderer_last_frame(void* renderer, RestirParams* params, RestirFramePlan* plan, RestirFrameState* state)
{
	if (renderer == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	static_cast<Renderer*>(renderer)->lastFrame(params, plan, state);
	return RESTIR_OK;
}

extern "C" int restir_renderer_save_state(void* renderer, const char* path)
{
	return renderer == nullptr ? RESTIR_ERROR_INVALID_ARGUMENT : static_cast<Renderer*>(renderer)->saveState(path);
}

extern "C" int restir_renderer_load_state(void* renderer, const char* path)
{
	return renderer == nullptr ? RESTIR_ERROR_INVALID_ARGUMENT : static_cast<Renderer*>(renderer)->loadState(path);
}

extern "C" int restir_renderer_buffer(void* renderer, const char* name, void** pointer, uint64_t* bytes)
{
	if (renderer == nullptr || name == nullptr || pointer == nullptr || bytes == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->buffer(name, pointer, bytes);
}

// --- batches --------------------------------------------------------------------

extern "C" void* restir_batch_create(const RestirSettings* settings, uint32_t views)
{
	if (views == 0u || views > 64u)
	{
		return nullptr;
	}
	RestirSettings s;
	if (settings != nullptr)
	{
		s = *settings;
	}
	else
	{
		restir_settings_default(&s);
	}
	Batch* batch = new (std::nothrow) Batch(s, views);
	if (batch != nullptr && !batch->valid())
	{
		delete batch;
		return nullptr;
	}
	return batch;
}

extern "C" void restir_batch_destroy(void* batch)
{
	delete static_cast<Batch*>(batch);
}

extern "C" int restir_batch_set_scene(void* batch, void* mesh, int use_scene_defaults)
{
	if (batch == nullptr || mesh == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Batch*>(batch)->setScene(*static_cast<restir::Mesh*>(mesh), use_scene_defaults != 0);
}

extern "C" int restir_batch_set_settings(void* batch, const RestirSettings* settings)
{
	if (batch == nullptr || settings == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Batch*>(batch)->setSettings(*settings);
}

extern "C" int restir_batch_render(void* batch, const RestirFrameInput* inputs)
{
	if (batch == nullptr || inputs == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Batch*>(batch)->render(inputs);
}

extern "C" int restir_batch_autotune(void* batch, const RestirFrameInput* inputs, uint32_t frames, RestirBatchTuning* best)
{
	if (batch == nullptr || inputs == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Batch*>(batch)->autotune(inputs, frames, best);
}

extern "C" int restir_batch_set_tuning(void* batch, const RestirBatchTuning* tuning)
{
	if (batch == nullptr || tuning == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Batch*>(batch)->setTuning(*tuning);
}

extern "C" int restir_batch_get_tuning(void* batch, RestirBatchTuning* tuning)
{
	if (batch == nullptr || tuning == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	*tuning = static_cast<Batch*>(batch)->tuning();
	return RESTIR_OK;
}

extern "C" int restir_batch_synchronize(void* batch)
{
	return batch != nullptr ? static_cast<Batch*>(batch)->synchronize() : RESTIR_ERROR_INVALID_ARGUMENT;
}

extern "C" void* restir_batch_stream(void* batch)
{
	return batch != nullptr ? static_cast<void*>(static_cast<Batch*>(batch)->stream()) : nullptr;
}

extern "C" int restir_batch_view_buffer(void* batch, uint32_t view, const char* name, void** pointer, uint64_t* bytes)
{
	if (batch == nullptr || view >= static_cast<Batch*>(batch)->views() || name == nullptr || pointer == nullptr
		|| bytes == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Batch*>(batch)->view(view).buffer(name, pointer, bytes);
}

extern "C" int restir_batch_view_last_frame(void* batch, uint32_t view, RestirParams* params, RestirFramePlan* plan,
	RestirFrameState* state)
{
	if (batch == nullptr || view >= static_cast<Batch*>(batch)->views())
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	static_cast<Batch*>(batch)->view(view).lastFrame(params, plan, state);
	return RESTIR_OK;
}
