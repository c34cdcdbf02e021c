/*
 * restir-b200: the frame driver, a C++ replacement of the reference's
 * Renderer (src/renderer.h:73-125, src/renderer.cpp:435-1166) over the pass
 * ABI of restir_gpu.h. It owns every device buffer of a frame and its
 * history, derives each pass's uniforms exactly as Renderer::render does,
 * and runs the passes in the reference's order on one CUDA stream
 * (optionally replayed from a CUDA graph).
 *
 * Scope: the passes named in restir_gpu.h (specular GI included) and the
 * display chain of restir_display.h (auto exposure, TAA, tone mapping into a
 * BGRA8 image). The debug views are not part of this driver.
 */
#ifndef RESTIR_FRAME_H
#define RESTIR_FRAME_H

#include "restir_gpu.h"
#include "restir_host.h"

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The renderer's settings (src/settings.h:153-227), defaults from
 * restir_settings_default. Enumerations as in settings.h: ray_mode 0 depth
 * buffer, 1 hybrid, 2 BVH; direct_lighting 0 ReSTIR DI, 1 through GI only. */
typedef struct RestirSettings
{
	float light_position[3];
	float light_color[3];
	float light_intensity;
	int extra_lights;
	float extra_intensity;
	int extra_seed;
	int sky_enabled;
	float sky_zenith[3];
	float sky_horizon[3];
	float sky_ground[3];
	float sky_intensity;
	int multiple_bounces;
	int shadows;
	int denoiser;
	int world_space_reuse;
	int emissive_lighting;
	int ray_mode;
	int direct_lighting;
	int clamp_jacobian;
	int clamp_outliers;
	int boiling_filter;
	int gi_divisor;          /* 1, 2 or 4 (kGiResolutions) */
	int shadow_face_size;    /* texels (kShadowFaceSizes: 256, 512, 1024, 2048) */
	int atrous_iterations;   /* 0-5 */
	int initial_candidates;
	int temporal_taps;
	int spatial_taps;
	int trace_steps;
	int di_candidates;
	int di_spatial_taps;
	uint32_t grid_table_size;
	uint32_t grid_cell_capacity;
	uint32_t grid_mode;      /* RESTIR_GRID_* */
	uint32_t wavefront;      /* no reference counterpart: 1 runs the GI temporal pass as
	                            restir_gi_temporal_wavefront (same output), 0 as restir_gi_temporal */
	uint32_t radiance_cache; /* no reference counterpart: 1 takes the indirect light at GI
	                            sample points from the radiance cache (restir_cache.h),
	                            trained every frame; needs wavefront */
	uint32_t cache_training_samples;  /* path suffixes per frame (default 65,536) */
	uint32_t wave_visibility;         /* 1: visibility rays in warp lock step (traceBvhWave,
	                                     bvh.sh:177-212, the reference's Vulkan path) */
	int taa;                 /* temporal anti-aliasing: jittered frames blended in the TAA
	                            pass (settings.h:194) */
	int auto_exposure;       /* settings.h:214 */
	int tonemapper;          /* RESTIR_TONEMAP_* (settings.h:212) */
	float exposure_ev;       /* settings.h:213 */
	float adaptation_speed;  /* settings.h:215, per second */
	int display;             /* no reference counterpart (the reference always draws to its
	                            window): 0 skips exposure, TAA and tone mapping */
	int bvh_on_device;       /* no reference counterpart: 1 builds the scene's BVH on the GPU
	                            (restir_bvh_build_gpu, the same buffer), 0 on the host */
	int specular_gi;         /* indirect specular (glossy reflections, settings.h:195) */
	int cache_only_gi;       /* no reference counterpart: with radiance_cache, the GI is the
	                            cache at each GI pixel's surface (restir_gi_from_cache): no GI
	                            rays, no reuse, no denoiser */
	float cache_learning_rate; /* no reference counterpart: the cache's Adam step size
	                              (0: restir_cache_config_default's) */
	float extra_light_orbit;   /* no reference counterpart (the reference orbits only its
	                              main light, main.cpp:505-518): > 0 moves every extra point
	                              light on a horizontal circle about the scene's vertical
	                              axis, light i at extra_light_orbit * s_i radians per
	                              second of RestirFrameInput::delta_time, s_i a seeded speed
	                              in [-1, -0.25] or [0.25, 1]; the list is uploaded per frame */
} RestirSettings;

/* FrameInput (renderer.h) with the fly camera's pose. */
typedef struct RestirFrameInput
{
	uint32_t width, height;
	float eye[3];
	float yaw, pitch;
	float delta_time;        /* FrameInput::m_deltaTime, seconds (auto exposure's adaptation) */
} RestirFrameInput;

/* What Renderer carries from frame to frame. */
typedef struct RestirFrameState
{
	uint32_t frame_number;
	int history_valid;
	int di_valid;
	float previous_view_proj[16];
	float previous_eye[3];
	int reference_accumulating;
	uint32_t reference_frames;
	float previous_unjittered_view_proj[16]; /* m_previousUnjitteredViewProj (TAA) */
	int taa_valid;                           /* m_taaValid */
	int exposure_valid;                      /* m_exposureValid */
} RestirFrameState;

/* Which passes the frame runs. */
typedef struct RestirFramePlan
{
	int di_active;                /* ReSTIR DI on, lights and a BVH present */
	int denoiser;                 /* variance + a-trous iterations */
	int atrous_iterations;
	int reference_accumulate;     /* the reference accumulates this frame */
	uint32_t reference_weight_frames; /* frames in the mean before this one */
	int surface_light_is_di;      /* GI reads the DI diffuse (else the G-buffer emission) */
	int display;                  /* the display chain runs (settings.display) */
	int taa;                      /* TAA runs: settings.taa, not while the reference accumulates */
	int exposure;                 /* auto exposure runs */
	int specular;                 /* restir_gi_specular runs and the composite adds it */
	int gi_from_cache;            /* the cache-only GI replaces the GI temporal and spatial passes */
	float unjittered_view_proj[16]; /* this frame's, for the next frame's TAA */
} RestirFramePlan;

void restir_settings_default(RestirSettings* settings);

/* The uniforms and the plan of one frame, from the settings, the scene's
 * description, its light count and the carried state (renderer.cpp:435-731).
 * Pure host arithmetic: no device work. */
int restir_frame_params(const RestirSettings* settings, const RestirMeshDesc* scene, uint32_t light_count,
	const RestirBvhDesc* bvh, const RestirFrameInput* input, const RestirFrameState* state,
	RestirParams* params, RestirFramePlan* plan);

/* Advances the carried state after a frame (renderer.cpp:1119-1124). */
void restir_frame_advance(const RestirParams* params, const RestirFramePlan* plan, const RestirFrameInput* input,
	RestirFrameState* state);

/* --- the renderer ---------------------------------------------------------- */

/* Per-pass device times of the last frame, in milliseconds (cudaEvent pairs
 * on the renderer's stream; the reference's per-view GPU times, ui.cpp:20-66). */
#define RESTIR_PASS_SHADOW 0
#define RESTIR_PASS_GBUFFER 1
#define RESTIR_PASS_DI_TEMPORAL 2
#define RESTIR_PASS_DI_SPATIAL 3
#define RESTIR_PASS_GRID 4
#define RESTIR_PASS_GI_TEMPORAL 5
#define RESTIR_PASS_GI_SPATIAL 6
#define RESTIR_PASS_DENOISE 7
#define RESTIR_PASS_COMPOSITE 8
#define RESTIR_PASS_REFERENCE 9
#define RESTIR_PASS_CACHE 10      /* radiance-cache training (no reference counterpart) */
#define RESTIR_PASS_DISPLAY 11    /* auto exposure, TAA and tone mapping */
#define RESTIR_PASS_SPECULAR 12   /* indirect specular (fs_specular.sc) */
#define RESTIR_PASS_COUNT 13

typedef struct RestirMetrics
{
	int valid;
	double relative_mse;          /* ReferenceMetrics::m_relativeMse */
	double bias;                  /* mean image / mean reference - 1 */
	double error[4];              /* the error pass's record */
	float pass_ms[RESTIR_PASS_COUNT];
	uint32_t reference_frames;
} RestirMetrics;

/* Creates a renderer on the current CUDA device, with its own stream. */
void* restir_renderer_create(const RestirSettings* settings);
void restir_renderer_destroy(void* renderer);
/* Builds the BVH and light list on the host and uploads them
 * (Renderer::setScene, renderer.cpp:365-419). Takes the light position and
 * sky from the scene when use_scene_defaults is set (main.cpp:539-565). */
int restir_renderer_set_scene(void* renderer, void* mesh, int use_scene_defaults);
int restir_renderer_set_settings(void* renderer, const RestirSettings* settings);
int restir_renderer_get_settings(void* renderer, RestirSettings* settings);
/* Renders one frame (Renderer::render). The work is enqueued on the
 * renderer's stream; the call returns without waiting for it. */
int restir_renderer_render(void* renderer, const RestirFrameInput* input);
/* Records one frame into a CUDA graph on first use and replays it after:
 * the same as restir_renderer_render for inputs of the same size. */
int restir_renderer_render_graph(void* renderer, const RestirFrameInput* input);
/* Runs the error pass against the reference on the last frame and reads its
 * record back (waits for the stream), as Renderer::frameSubmitted does. */
int restir_renderer_measure(void* renderer, RestirMetrics* metrics);
/* Per-pass device times (cudaEvent pairs on the renderer's stream) of the
 * last `frames` frames rendered without a graph, oldest first, as
 * ms[frame * RESTIR_PASS_COUNT + pass]; up to 128 frames are kept. Waits for
 * the stream; returns the number of frames written. */
int restir_renderer_pass_history(void* renderer, uint32_t frames, float* ms);

/* Renders one frame with the work counters of restir_counters on, and adds
 * each pass's counts to counts[pass * 8 + k] (RESTIR_PASS_COUNT x 8). The
 * device is synchronised after every pass: a profiling frame, not a timed
 * one. No counterpart in the reference. */
int restir_renderer_profile_frame(void* renderer, const RestirFrameInput* input, uint64_t* counts);
void restir_renderer_set_reference_accumulation(void* renderer, int accumulate);
void restir_renderer_invalidate_history(void* renderer);
/* Waits for the renderer's stream. */
int restir_renderer_synchronize(void* renderer);
/* The renderer's stream (a cudaStream_t). */
void* restir_renderer_stream(void* renderer);
/* The last frame's uniforms, plan and carried state. */
int restir_renderer_last_frame(void* renderer, RestirParams* params, RestirFramePlan* plan, RestirFrameState* state);

/* Device buffers of the renderer, by name ("hdr", "gbuffer.depth",
 * "gi.sample", "grid", "reference.mean", ...): pointer and byte size. */
int restir_renderer_buffer(void* renderer, const char* name, void** pointer, uint64_t* bytes);

/* The per-frame state as a file, so that any frame can be replayed for
 * debugging (no reference counterpart; the reference's history is per
 * frame and never saved, renderer.h:87-88): save writes the carried state
 * (RestirFrameState, the ping-pong indices, the orbit time) and every frame
 * target (reservoirs, grids, histories, G-buffer, reference mean, TAA and
 * specular histories) plus the radiance cache's state; load reads such a
 * file back into a renderer whose targets have the same sizes (render one
 * frame of that size first) and the same scene and settings. Both wait for
 * the renderer's streams. RESTIR_ERROR_INVALID_ARGUMENT for a file that does
 * not match. */
int restir_renderer_save_state(void* renderer, const char* path);
int restir_renderer_load_state(void* renderer, const char* path);

/* --- Batches of views (no reference counterpart) ------------------------ */

/* Several views of one scene (each with its own camera and resolution)
 * rendered as one frame: the scene is uploaded once, the shadow atlas drawn
 * once, the GI candidate rays of every view go to one ray queue that a single
 * persistent tracer launch drains (restir_trace_queue), and the whole frame
 * is one CUDA graph whose per-view branches run on their own streams. Each
 * view's output equals a renderer's for that view alone. The radiance cache
 * is not available in a batch (settings.radiance_cache is ignored). */
typedef struct RestirBatchTuning
{
	uint32_t tracer_threads;       /* 64, 128 or 256 threads per block */
	uint32_t tracer_blocks_per_sm; /* resident blocks per SM, 0: as many as fit */
	float ms_per_frame;            /* autotune: the winner's device time per batch frame */
} RestirBatchTuning;

void* restir_batch_create(const RestirSettings* settings, uint32_t views);
void restir_batch_destroy(void* batch);
int restir_batch_set_scene(void* batch, void* mesh, int use_scene_defaults);
int restir_batch_set_settings(void* batch, const RestirSettings* settings);
/* inputs: one per view (width, height and camera of each). */
int restir_batch_render(void* batch, const RestirFrameInput* inputs);
/* Renders `frames` frames with each of a fixed list of tracer shapes and
 * keeps the fastest (the frames advance the views' histories). */
int restir_batch_autotune(void* batch, const RestirFrameInput* inputs, uint32_t frames, RestirBatchTuning* best);
int restir_batch_set_tuning(void* batch, const RestirBatchTuning* tuning);
int restir_batch_get_tuning(void* batch, RestirBatchTuning* tuning);
int restir_batch_synchronize(void* batch);
/* The stream the batch frame's graph is launched on. */
void* restir_batch_stream(void* batch);
/* A view's buffers and last frame, as restir_renderer_buffer / _last_frame. */
int restir_batch_view_buffer(void* batch, uint32_t view, const char* name, void** pointer, uint64_t* bytes);
int restir_batch_view_last_frame(void* batch, uint32_t view, RestirParams* params, RestirFramePlan* plan,
	RestirFrameState* state);

#ifdef __cplusplus
}
#endif

#endif /* RESTIR_FRAME_H */
