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
#include "../../include/restir_frame.h"
#include "bvh_build.h"

#include <cuda_runtime.h>

#include <cstring>
#include <map>
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

class Renderer
{
public:
	explicit Renderer(const RestirSettings& settings) : m_settings(settings)
	{
		std::memset(&m_state, 0, sizeof(m_state));
		for (int i = 0; i < 4; ++i)
		{
			m_state.previous_view_proj[i * 5] = 1.0f;
		}
		cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking);
		for (auto& frame : m_events)
		{
			for (auto& pass : frame)
			{
				cudaEventCreate(&pass[0]);
				cudaEventCreate(&pass[1]);
			}
		}
		cudaMallocHost(&m_errorHost, 4 * sizeof(double));
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
		cudaStreamDestroy(m_stream);
	}

	int setScene(const Mesh& mesh, bool useSceneDefaults)
	{
		cudaStreamSynchronize(m_stream);
		releaseGraph();
		releaseScene();
		m_mesh = mesh;
		if (useSceneDefaults)
		{
			std::memcpy(m_settings.light_position, mesh.lightPosition, sizeof(m_settings.light_position));
			m_settings.sky_enabled = mesh.sky ? 1 : 0;
		}
		m_bvh = buildBvh(mesh, 8);
		int status = upload(m_sceneBuffers["bvh"], m_bvh.data.data(), m_bvh.data.size() * sizeof(float));
		status |= upload(m_sceneBuffers["normals"], m_bvh.triangleNormals.data(), m_bvh.triangleNormals.size() * sizeof(float));
		status |= upload(m_sceneBuffers["materials"], mesh.materialData.data(), mesh.materialData.size() * sizeof(float));
		m_lightsKey.clear();
		status |= updateLights();
		status |= initCache(mesh);
		m_state.history_valid = 0;
		m_state.di_valid = 0;
		m_state.reference_frames = 0;
		m_hasScene = status == 0;
		return status == 0 ? RESTIR_OK : RESTIR_ERROR_OUT_OF_MEMORY;
	}

	// The radiance cache over the scene's box (1% of the radius wider), fresh
	// for every scene.
	int initCache(const Mesh& mesh)
	{
		restir_cache_config_default(&m_cacheConfig);
		for (int i = 0; i < 3; ++i)
		{
			m_cacheConfig.bounds_min[i] = mesh.boundsMin[i] - 0.01f * mesh.radius;
			m_cacheConfig.bounds_max[i] = mesh.boundsMax[i] + 0.01f * mesh.radius;
		}
		const uint64_t bytes = restir_cache_state_bytes(&m_cacheConfig);
		Buffer& b = m_sceneBuffers["cache.state"];
		b.bytes = bytes;
		if (bytes == 0 || cudaMalloc(&b.pointer, bytes) != cudaSuccess)
		{
			b.pointer = nullptr;
			return 1;
		}
		return restir_cache_init(&m_cacheConfig, b.pointer, m_stream) == RESTIR_OK ? 0 : 1;
	}

	int setSettings(const RestirSettings& settings)
	{
		m_settings = settings;
		return updateLights();
	}

	const RestirSettings& settings() const { return m_settings; }

	int render(const RestirFrameInput& input, bool graph)
	{
		if (!m_hasScene)
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		int status = updateLights();
		if (status != RESTIR_OK)
		{
			return status;
		}
		RestirMeshDesc desc = describe();
		RestirBvhDesc bvhDesc = {};
		bvhDesc.node_count = m_bvh.nodeCount;
		bvhDesc.triangle_offset = m_bvh.triangleOffset;
		bvhDesc.triangle_count = m_bvh.triangleCount;
		// Reference mode: a moved camera starts the reference again (renderer.cpp:1050-1060).
		if (m_state.reference_accumulating && m_state.reference_frames > 0
			&& (std::memcmp(&m_referenceInput, &input, sizeof(input)) != 0))
		{
			m_state.reference_frames = 0;
		}
		m_referenceInput = input;
		status = restir_frame_params(&m_settings, &desc, m_lights.count, &bvhDesc, &input, &m_state, &m_params, &m_plan);
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
				status = restir_frame_params(&m_settings, &desc, m_lights.count, &bvhDesc, &input, &m_state, &m_params, &m_plan);
			}
			if (status != RESTIR_OK)
			{
				return status;
			}
		}
		status = ensureWorkspace(m_params);
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
		restir_frame_advance(&m_params, &m_plan, &input, &m_state);
		m_historyRead = 1 - m_historyRead;
		if (m_plan.di_active)
		{
			m_diRead = 1 - m_diRead;
		}
		m_timed = !graph;
		return RESTIR_OK;
	}

	int measure(RestirMetrics* metrics)
	{
		std::memset(metrics, 0, sizeof(*metrics));
		if (m_targets.empty())
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
		int status = launchError(&m_params, p<uint16_t>("hdr"), p<double>("reference.mean"), p<uint8_t>("reference.alpha"),
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
		m_state.history_valid = 0;
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

	int buffer(const std::string& name, void** pointer, uint64_t* bytes)
	{
		auto it = m_targets.find(name);
		if (it == m_targets.end())
		{
			it = m_sceneBuffers.find(name);
			if (it == m_sceneBuffers.end())
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
		d.triangle_count = m_mesh.triangleCount();
		d.material_count = uint32_t(m_mesh.materials.size());
		std::memcpy(d.bounds_min, m_mesh.boundsMin, sizeof(d.bounds_min));
		std::memcpy(d.bounds_max, m_mesh.boundsMax, sizeof(d.bounds_max));
		std::memcpy(d.center, m_mesh.center, sizeof(d.center));
		d.radius = m_mesh.radius;
		return d;
	}

	// Renderer::updateLightList (renderer.cpp:1170-1207): rebuilt when its inputs change.
	int updateLights()
	{
		if (!m_hasScene && m_bvh.nodeCount == 0)
		{
			return RESTIR_OK;
		}
		const float scale = (m_mesh.radius / 1.75f) * (m_mesh.radius / 1.75f);
		std::string key = std::to_string(m_settings.emissive_lighting) + "/" + std::to_string(m_settings.extra_lights) + "/"
			+ std::to_string(m_settings.extra_intensity) + "/" + std::to_string(m_settings.extra_seed) + "/" + std::to_string(scale);
		if (key == m_lightsKey)
		{
			return RESTIR_OK;
		}
		m_lightsKey = key;
		static const std::vector<Emitter> none;
		m_lights = buildLightList(m_settings.emissive_lighting ? m_bvh.emitters : none, m_settings.extra_lights,
			m_settings.extra_intensity, uint32_t(m_settings.extra_seed), m_mesh.boundsMin, m_mesh.boundsMax, scale);
		cudaStreamSynchronize(m_stream);
		Buffer& b = m_sceneBuffers["lights"];
		cudaFree(b.pointer);
		b = Buffer();
		std::vector<float> data = m_lights.data;
		if (data.empty())
		{
			data.assign(16, 0.0f);
		}
		int status = upload(b, data.data(), data.size() * sizeof(float));
		m_state.di_valid = 0; // stored light indices refer to the old list
		releaseGraph();
		return status == 0 ? RESTIR_OK : RESTIR_ERROR_OUT_OF_MEMORY;
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
		m_state.history_valid = 0;
		m_state.di_valid = 0;
		m_state.reference_frames = 0;
		m_state.frame_number = 0;
		std::memset(m_state.previous_view_proj, 0, sizeof(m_state.previous_view_proj));
		for (int i = 0; i < 4; ++i)
		{
			m_state.previous_view_proj[i * 5] = 1.0f;
		}
		cudaStreamSynchronize(m_stream);
		return RESTIR_OK;
	}

	// The wavefront GI temporal pass's ray queue, sized by the candidate count
	// (a setting that keeps the history); allocated before any capture.
	int ensureWorkspace(const RestirParams& P)
	{
		const uint64_t needed = m_settings.wavefront ? restir_gi_temporal_workspace_bytes(&P) : 0;
		auto found = m_targets.find("gi.workspace");
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
		m_targets["gi.workspace"] = b;
		return RESTIR_OK;
	}

	bool targetsMatch(const RestirParams& P) const
	{
		return !m_targets.empty() && P.width == m_width && P.height == m_height && P.gi_width == m_giWidth
			&& P.gi_height == m_giHeight && P.shadow_face_size == m_faceSize && P.grid_table_size == m_tableSize
			&& P.grid_cell_capacity == m_capacity;
	}

	void mark(int pass, int edge, bool events)
	{
		if (events)
		{
			cudaEventRecord(m_events[m_slot][pass][edge], m_stream);
		}
	}

	// The passes of one frame, in the reference's order (renderer.cpp:527-1077).
	int enqueue(bool events)
	{
		const RestirParams& P = m_params;
		const RestirFramePlan& plan = m_plan;
		const int hw = 1 - m_historyRead, hr = m_historyRead, dw = 1 - m_diRead, dr = m_diRead;
		const std::string H = std::to_string(hw), R = std::to_string(hr);
		RestirScene scene = {};
		scene.bvh = static_cast<const float*>(m_sceneBuffers["bvh"].pointer);
		scene.node_count = m_bvh.nodeCount;
		scene.triangle_offset = m_bvh.triangleOffset;
		scene.triangle_count = m_bvh.triangleCount;
		scene.lights = static_cast<const float*>(m_sceneBuffers["lights"].pointer);
		scene.light_count = m_lights.count;
		scene.triangle_normals = static_cast<const float*>(m_sceneBuffers["normals"].pointer);
		scene.materials = static_cast<const float*>(m_sceneBuffers["materials"].pointer);
		scene.material_count = uint32_t(m_mesh.materials.size());
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
		run(RESTIR_PASS_SHADOW, [&] { return restir_shadow_atlas(&P, &scene, p<float>("shadow.atlas"), s); });
		run(RESTIR_PASS_GBUFFER, [&] { return restir_gbuffer_primary(&P, &scene, &gb, s); });
		const std::string DW = std::to_string(dw), DR = std::to_string(dr);
		RestirDiReservoirs diPrevious = { p<float>("di.sample" + DR), p<float>("di.receiver" + DR), p<uint16_t>("di.normal" + DR) };
		RestirDiReservoirs diCurrent = { p<float>("di.sample" + DW), p<float>("di.receiver" + DW), p<uint16_t>("di.normal" + DW) };
		if (plan.di_active)
		{
			run(RESTIR_PASS_DI_TEMPORAL, [&] { return restir_di_temporal(&P, &scene, &gb, &diPrevious, &diCurrent, s); });
			run(RESTIR_PASS_DI_SPATIAL, [&] {
				return restir_di_spatial(&P, &scene, &gb, &diCurrent, p<uint16_t>("di.diffuse"), p<uint16_t>("di.specular"), s);
			});
		}
		const uint16_t* surface = plan.surface_light_is_di ? (plan.di_active ? p<uint16_t>("di.diffuse") : p<uint16_t>("black"))
			: p<uint16_t>("gbuffer.emissive");
		uint32_t* gridWrite = p<uint32_t>("grid" + H);
		run(RESTIR_PASS_GRID, [&] {
			return restir_grid_clear(&P, gridWrite, s) | restir_grid_insert(&P, &gb, gridWrite, s);
		});
		RestirGiHistory history = { p<float>("gi.sample" + R), p<float>("gi.receiver" + R), p<float>("gi.normal" + R),
			plan.denoiser ? p<uint16_t>("filtered" + R) : p<uint16_t>("gi.color" + R), p<uint16_t>("gi.moments" + R) };
		RestirGiReservoirs current = { p<float>("gi.sample" + H), p<float>("gi.receiver" + H), p<float>("gi.normal" + H) };
		const bool cached = P.radiance_cache > 0.5f;
		void* cacheState = m_sceneBuffers["cache.state"].pointer;
		run(RESTIR_PASS_GI_TEMPORAL, [&] {
			const Buffer& w = m_targets["gi.workspace"];
			if (cached)
			{
				return restir_gi_temporal_cached(&P, &scene, &gb, &history, p<uint32_t>("grid" + R), p<float>("shadow.atlas"),
					surface, &current, &m_cacheConfig, cacheState, w.pointer, w.bytes, s);
			}
			if (m_settings.wavefront)
			{
				return restir_gi_temporal_wavefront(&P, &scene, &gb, &history, p<uint32_t>("grid" + R), p<float>("shadow.atlas"),
					surface, &current, w.pointer, w.bytes, s);
			}
			return restir_gi_temporal(&P, &scene, &gb, &history, p<uint32_t>("grid" + R), p<float>("shadow.atlas"), surface,
				&current, s);
		});
		run(RESTIR_PASS_GI_SPATIAL, [&] {
			if (cached)
			{
				const Buffer& w = m_targets["gi.workspace"];
				return restir_gi_spatial_cached(&P, &scene, &gb, &current, gridWrite, &history, p<float>("shadow.atlas"), surface,
					p<uint16_t>("gi.color" + H), p<uint16_t>("gi.moments" + H), &m_cacheConfig, cacheState, w.pointer, w.bytes, s);
			}
			return restir_gi_spatial(&P, &scene, &gb, &current, gridWrite, &history, p<float>("shadow.atlas"), surface,
				p<uint16_t>("gi.color" + H), p<uint16_t>("gi.moments" + H), s);
		});
		if (cached)
		{
			// Training after the frame's queries: every query of a frame sees the same weights.
			run(RESTIR_PASS_CACHE, [&] {
				const Buffer& w = m_targets["gi.workspace"];
				return restir_cache_train_frame(&P, &scene, &gb, p<float>("shadow.atlas"), &m_cacheConfig, cacheState, w.pointer,
					w.bytes, s);
			});
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
		run(RESTIR_PASS_COMPOSITE, [&] {
			return restir_composite(&P, &gb, p<float>("shadow.atlas"), p<uint16_t>(denoised), diDiffuse, diSpecular,
				p<uint16_t>("hdr"), s);
		});
		if (plan.reference_accumulate)
		{
			run(RESTIR_PASS_REFERENCE, [&] {
				return restir_reference_accumulate(&P, p<uint16_t>("hdr"), p<double>("reference.mean"),
					p<uint8_t>("reference.alpha"), plan.reference_weight_frames, s);
			});
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
		if (!updated && cudaGraphInstantiate(&m_graphExec, graph, 0) != cudaSuccess)
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

	void releaseScene()
	{
		for (auto& kv : m_sceneBuffers)
		{
			cudaFree(kv.second.pointer);
		}
		m_sceneBuffers.clear();
		m_hasScene = false;
	}

	RestirSettings m_settings;
	RestirFrameState m_state;
	RestirParams m_params = {};
	RestirFramePlan m_plan = {};
	RestirFrameInput m_referenceInput = {};
	Mesh m_mesh;
	BvhResult m_bvh;
	LightListResult m_lights;
	std::string m_lightsKey;
	std::map<std::string, Buffer> m_sceneBuffers;
	std::map<std::string, Buffer> m_targets;
	uint32_t m_width = 0, m_height = 0, m_giWidth = 0, m_giHeight = 0, m_faceSize = 0, m_tableSize = 0, m_capacity = 0;
	int m_historyRead = 0;
	int m_diRead = 0;
	bool m_hasScene = false;
	bool m_timed = false;
	// Per-pass events of the last kEventRing stream-launched frames.
	static constexpr uint32_t kEventRing = 128;
	bool m_passRan[kEventRing][RESTIR_PASS_COUNT] = {};
	cudaEvent_t m_events[kEventRing][RESTIR_PASS_COUNT][2] = {};  // start, end of each pass
	RestirCacheConfig m_cacheConfig = {};
	uint32_t m_slot = 0;
	uint32_t m_lastSlot = 0;
	uint32_t m_timedFrames = 0;
	cudaStream_t m_stream = nullptr;
	cudaGraphExec_t m_graphExec = nullptr;
	double* m_errorHost = nullptr;
	uint64_t* m_profile = nullptr;
};

} // namespace
} // namespace restir

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

extern "C" int restir_renderer_buffer(void* renderer, const char* name, void** pointer, uint64_t* bytes)
{
	if (renderer == nullptr || name == nullptr || pointer == nullptr || bytes == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	return static_cast<Renderer*>(renderer)->buffer(name, pointer, bytes);
}
