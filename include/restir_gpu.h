/*
 * restir-b200: C ABI of the per-frame light-transport passes.
 *
 * Each entry point replaces one pass of the reference renderer
 * (pkonecki/restir, src/renderer.cpp, Renderer::render, lines 435-1125),
 * which binds textures and buffers at fixed stages, sets vec4 uniforms and
 * calls bgfx::dispatch or bgfx::submit. Here the bound resources are plain
 * device pointers, the uniforms are one POD struct (RestirParams), and every
 * call is enqueued on the caller's CUDA stream (passed as void*, a
 * cudaStream_t) and returns a status code. Calls never allocate, never
 * synchronise the device and never throw.
 *
 * Layouts are the reference's (see each struct):
 *   - BVH: one array of float4, nodes then triangles (src/bvh.h:7-22);
 *   - light list: 4 float4 per light (src/lights.h:5-17);
 *   - hash grid: uint32 [checksums T][counts T][entries T*C]
 *     (shaders/hashgrid.sh:25-33, 53-59);
 *   - images: row-major arrays indexed y * width + x, row 0 at the top
 *     (texture coordinate v = 0), 4 channels per pixel: float4 for RGBA32F,
 *     IEEE half x4 for RGBA16F, 4 bytes in B, G, R, A order for BGRA8,
 *     one float for D32F / R32F.
 * Numeric conventions (rounding, half and unorm8 encodings, sin/cos/exp)
 * are those of restir_numeric.h.
 *
 * Point sampling: a pass at one resolution that reads a target of another
 * resolution reads texel floor(uv * size), clamped to the image (the
 * reference's point samplers with clamp, renderer.cpp:1324-1328).
 */
#ifndef RESTIR_GPU_H
#define RESTIR_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define RESTIR_OK 0
#define RESTIR_ERROR_INVALID_ARGUMENT (-1)
#define RESTIR_ERROR_LAUNCH (-2)
#define RESTIR_ERROR_STEP_CAP (-3)   /* a traversal hit kBvhMaxSteps (set in the status word) */
#define RESTIR_ERROR_UNSUPPORTED (-4)
#define RESTIR_ERROR_TIMEOUT (-5)
#define RESTIR_ERROR_OUT_OF_MEMORY (-6)
#define RESTIR_ERROR_TOO_LARGE (-7)  /* input beyond a fixed-size variant's limit */

/* Ray modes (shaders/bvh.sh:16-19, settings.h:59-65). */
#define RESTIR_RAY_MODE_SCREEN 0
#define RESTIR_RAY_MODE_HYBRID 1
#define RESTIR_RAY_MODE_BVH 2

/* Hash grid insertion modes. ATOMIC keeps the first C arrivals of a cell in
 * arrival order (shaders/hashgrid.sh:182-200). DETERMINISTIC keeps the C
 * lowest GI pixel indices of a cell in increasing order, which is what a
 * sequential insertion in pixel order produces; it needs the entries cleared
 * as well (restir_grid_clear does that in this mode). */
#define RESTIR_GRID_ATOMIC 0
#define RESTIR_GRID_DETERMINISTIC 1

/* Ray kinds of restir_trace. */
#define RESTIR_TRACE_CLOSEST 0           /* nearest-first, short stack (bvh.sh:216-295) */
#define RESTIR_TRACE_ANY 1               /* stackless, first hit (bvh.sh:140-174) */
#define RESTIR_TRACE_CLOSEST_STACKLESS 2 /* stackless, nearest hit (bvh.sh:140-174) */
#define RESTIR_TRACE_CLOSEST_WATERTIGHT 3 /* full stack, watertight triangle test */
#define RESTIR_TRACE_CLOSEST_QUEUE 4     /* RESTIR_TRACE_CLOSEST through the persistent
                                            queue tracer (same results; no reference
                                            counterpart) */
#define RESTIR_TRACE_ANY_WAVE 5          /* any hit in warp lock step (bvh.sh:177-212); rays
                                            32i..32i+31 form one warp */

/*
 * Everything the reference passes read from vec4 uniforms, by name. Values
 * are those renderer.cpp sets (lines 490-731). Matrices are row-major and
 * map a column vector: clip = M * (x, y, z, 1).
 */
typedef struct RestirParams
{
	/* u_sceneViewProj, u_sceneInvViewProj (jittered when TAA or the
	 * reference is on), u_previousViewProj */
	float view_proj[16];
	float inv_view_proj[16];
	float prev_view_proj[16];
	/* u_shadowViewProj[6], and their inverses for the atlas ray cast */
	float shadow_view_proj[6][16];
	float shadow_inv_view_proj[6][16];

	float light_position[4];     /* u_lightPosition */
	float light_color[4];        /* u_lightColor, scaled by intensity * sceneScale^2 */
	float camera_position[4];    /* u_cameraPosition; also u_gridCamera of this frame's grid */
	float prev_camera_position[4]; /* u_diPrevious; u_gridCamera of last frame's grid */

	float frame_index;           /* u_frameInfo.x: frame number & 0xffffff */
	float history_valid;         /* u_frameInfo.y */
	float origin_bottom_left;    /* u_frameInfo.z (0: texture row 0 at the top) */
	float multiple_bounces;      /* u_frameInfo.w */

	uint32_t width, height;      /* full resolution (u_screenSize.xy) */
	uint32_t gi_width, gi_height;/* GI resolution (u_screenInfo.xy) */

	float scene_scale;           /* u_sceneInfo.x */
	float boiling_filter;        /* u_sceneInfo.y: 0 off, else 4 */
	float jacobian_clamp;        /* u_sceneInfo.z: 0 off, else 10 */
	float outlier_clamp;         /* u_sceneInfo.w: 0 off, else 8 */

	float surface_light_scale;   /* u_lightingInfo.x */
	float emission_scale;        /* u_lightingInfo.y */

	int32_t initial_candidates;  /* u_restirOptions.x */
	int32_t temporal_taps;       /* u_restirOptions.y */
	int32_t spatial_taps;        /* u_restirOptions.z */
	int32_t trace_steps;         /* u_restirOptions.w */

	float grid_min_cell;         /* u_gridInfo.x */
	float grid_pixel_size;       /* u_gridInfo.y: world size of a GI pixel at unit distance */
	float grid_cell_pixels;      /* u_gridInfo.z */
	float world_space_reuse;     /* u_gridInfo.w */
	uint32_t grid_table_size;    /* T, a power of two (kGridTableSize) */
	uint32_t grid_cell_capacity; /* C (kGridCellCapacity) */
	uint32_t grid_mode;          /* RESTIR_GRID_* */

	int32_t ray_mode;            /* u_bvhInfo.w: RESTIR_RAY_MODE_* */

	int32_t di_light_count;      /* u_diInfo.x */
	int32_t di_candidates;       /* u_diInfo.y */
	int32_t di_spatial_taps;     /* u_diInfo.z */
	float di_history_valid;      /* u_diInfo.w */

	float shadow_far;            /* u_shadowInfo.x */
	float shadow_tan_half_fov;   /* u_shadowInfo.y */
	float shadow_inv_face_size;  /* u_shadowInfo.z */
	float shadows_enabled;       /* u_shadowOptions.x */
	uint32_t shadow_face_size;   /* texels per face side; the atlas is 3x2 faces */

	float sky_zenith[4];         /* u_skyZenith: rgb premultiplied, w 1 when on */
	float sky_horizon[4];        /* u_skyHorizon */
	float sky_ground[4];         /* u_skyGround */

	float composite_options[4];  /* u_compositeOptions */
	/* No reference counterpart: > 0.5 when the GI passes take the indirect
	 * light leaving a sample point from the radiance cache
	 * (restir_gi_temporal_cached, restir_gi_spatial_cached) instead of
	 * previousIndirect (restir.sh:265-298). */
	float radiance_cache;
	uint32_t cache_training_samples;  /* path suffixes traced per frame to train it */
	/* > 0.5: visibility rays walk the BVH in warp lock step (traceBvhWave,
	 * bvh.sh:177-212, the reference's Vulkan build) instead of per lane
	 * (traceBvhStackless); the hits are the same. */
	float wave_visibility;
	/* u_compositeSpecular.x (renderer.cpp:955-961): the weight of the indirect
	 * specular in restir_composite_specular (1 with specular GI on). */
	float composite_specular;
} RestirParams;

/* Scene buffers, uploaded once per scene (renderer.cpp:365-419, 1170-1207). */
typedef struct RestirScene
{
	const float* bvh;            /* float4s: node_count nodes (2 each), then triangles (4 each) */
	uint32_t node_count;
	uint32_t triangle_offset;    /* first triangle, in float4s (2 * node_count) */
	uint32_t triangle_count;
	const float* lights;         /* float4s, 4 per light (lights.h) */
	uint32_t light_count;
	/* Primary-ray inputs, standing in for the raster pass's vertex
	 * attributes and material uniforms (fs_gbuffer.sc): per triangle in BVH
	 * order one float4 (shading normal xyz, w: 1 if two-sided), and per
	 * material two float4 (base colour rgb, roughness), (emission rgb,
	 * metallic). */
	const float* triangle_normals;
	const float* materials;
	uint32_t material_count;
} RestirScene;

/* The G-buffer (renderer.cpp:1363-1376), full resolution. */
typedef struct RestirGBuffer
{
	uint8_t* albedo;         /* BGRA8: rgb base colour, a roughness */
	uint8_t* normal;         /* BGRA8: rgb surface normal * 0.5 + 0.5, a metallic */
	uint16_t* emissive;      /* RGBA16F: rgb emission, a occlusion */
	uint8_t* shading_normal; /* BGRA8: rgb shading normal * 0.5 + 0.5 */
	float* depth;            /* D32F: NDC depth in [0, 1], 1 where nothing was hit */
} RestirGBuffer;

/* ReSTIR GI reservoir targets at GI resolution, float4 each (restir.sh:11-15):
 * sample (position, M), receiver (position, W), normal (normal, sample id). */
typedef struct RestirGiReservoirs
{
	float* sample;
	float* receiver;
	float* normal;
} RestirGiReservoirs;

/* Last frame's GI targets the GI passes read (renderer.cpp:772-815). */
typedef struct RestirGiHistory
{
	const float* sample;      /* s_historySample (temporal pass) */
	const float* receiver;    /* s_historyReceiver */
	const float* normal;      /* s_historyNormal */
	const uint16_t* color;    /* s_historyColor: half4, the filtered history with the denoiser */
	const uint16_t* moments;  /* s_historyMoments: half4 (spatial pass) */
} RestirGiHistory;

/* ReSTIR DI reservoirs, full resolution (di.sh:12-16): sample float4
 * (point, light), receiver float4 (position, W), normal half4 (normal, M). */
typedef struct RestirDiReservoirs
{
	float* sample;
	float* receiver;
	uint16_t* normal;
} RestirDiReservoirs;

/* --- Scene-side passes ------------------------------------------------ */

/* Traces n rays. rays: 8 floats each, (origin xyz, tmax), (direction xyz,
 * unused). Writes the triangle index (BVH order, -1 for none) and the
 * distance (tmax when nothing was hit). kind: RESTIR_TRACE_*. Replaces the
 * traversal of shaders/bvh.sh:298-319 for a fixed ray set. */
int restir_trace(const RestirParams* params, const RestirScene* scene, const float* rays,
	int32_t* hit_triangle, float* hit_distance, uint32_t n, int kind, void* stream);

/* The point light's distance atlas, 3 x 2 faces of shadow_face_size texels:
 * distance to the nearest surface / shadow_far, 1 where nothing is hit.
 * Replaces the six shadow views (renderer.cpp:527-593, fs_shadow.sc). */
int restir_shadow_atlas(const RestirParams* params, const RestirScene* scene, float* atlas, void* stream);

/* The G-buffer by primary rays through pixel centres, nearest front-facing
 * triangle. Replaces the geometry view (renderer.cpp:595-612, fs_gbuffer.sc). */
int restir_gbuffer_primary(const RestirParams* params, const RestirScene* scene,
	const RestirGBuffer* gbuffer, void* stream);

/* --- Hash grid (cs_grid_clear.sc, cs_grid_insert.sc) ------------------- */

/* Zeroes the checksums and counts (and, in the deterministic mode, sets the
 * entries to 0xffffffff). grid: T * (2 + C) uint32. */
int restir_grid_clear(const RestirParams* params, uint32_t* grid, void* stream);

/* Lists every GI pixel in the cell of its receiver, at a jittered position. */
int restir_grid_insert(const RestirParams* params, const RestirGBuffer* gbuffer, uint32_t* grid, void* stream);

/* --- ReSTIR DI (cs_di_temporal.sc, cs_di_spatial.sc) ------------------- */

int restir_di_temporal(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirDiReservoirs* previous, const RestirDiReservoirs* output, void* stream);

/* diffuse, specular: half4 full resolution. */
int restir_di_spatial(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirDiReservoirs* current, uint16_t* diffuse, uint16_t* specular, void* stream);

/* --- ReSTIR GI (cs_restir_temporal.sc, cs_restir_spatial.sc) ----------- */

/* surface_light: half4 full resolution (the DI diffuse output, or the
 * G-buffer emission). shadow_atlas as written by restir_shadow_atlas. */
int restir_gi_temporal(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, const RestirGiReservoirs* output, void* stream);

/* No reference counterpart: the bytes of device workspace that
 * restir_gi_temporal_wavefront needs for these params (60 bytes per GI
 * pixel and initial candidate, in six regions each rounded up to 256). */
uint64_t restir_gi_temporal_workspace_bytes(const RestirParams* params);

/* restir_gi_temporal as a wavefront, with identical outputs: a candidates
 * pass (directions and depth-buffer marches) appends the rays it cannot
 * answer to a queue in the workspace, a persistent tracer walks the queue
 * (a lane takes the next ray as soon as its own finishes), and a shading
 * pass completes cs_restir_temporal.sc from the recorded hits. workspace:
 * 256-byte aligned device memory of at least
 * restir_gi_temporal_workspace_bytes; it must not be shared with a call
 * whose kernels may overlap this one's. */
int restir_gi_temporal_wavefront(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, const RestirGiReservoirs* output, void* workspace, uint64_t workspace_bytes,
	void* stream);

/* No reference counterpart: the wavefront's three steps with a ray queue the
 * caller owns, so that several views can fill one queue and have it traced
 * by a single persistent launch (restir_batch_* does this):
 *   restir_ray_queue_reset(queue)                         counters to zero
 *   restir_gi_temporal_candidates(view ..., records, queue)   per view
 *   restir_trace_queue(scene, queue, ...)                 once
 *   restir_gi_temporal_shade(view ..., records, queue)        per view
 * The outputs equal restir_gi_temporal's. queue: 256-byte aligned,
 * restir_ray_queue_bytes(capacity) bytes, capacity >= the sum of the views'
 * GI pixels x initial_candidates (rays past it are not traced: status bit
 * 2). records: 256-byte aligned, restir_gi_candidate_records_bytes(params)
 * per view. restir_trace_queue's threads (64, 128 or 256 per block) and
 * blocks_per_sm (0: as many as fit) shape the resident grid. */
uint64_t restir_ray_queue_bytes(uint32_t capacity);
int restir_ray_queue_reset(void* queue, void* stream);
uint64_t restir_gi_candidate_records_bytes(const RestirParams* params);
int restir_gi_temporal_candidates(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, void* records, uint64_t records_bytes, void* queue, uint32_t queue_capacity,
	void* stream);
int restir_trace_queue(const RestirScene* scene, void* queue, uint32_t queue_capacity, uint32_t threads,
	uint32_t blocks_per_sm, void* stream);
int restir_gi_temporal_shade(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, const RestirGiReservoirs* output, const void* records, uint64_t records_bytes,
	const void* queue, uint32_t queue_capacity, void* stream);

/* color, moments: half4 at GI resolution. */
int restir_gi_spatial(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiReservoirs* current, const uint32_t* current_grid, const RestirGiHistory* history,
	const float* shadow_atlas, const uint16_t* surface_light, uint16_t* color, uint16_t* moments, void* stream);

/* --- Denoiser (fs_svgf_variance.sc, fs_svgf_atrous.sc) ----------------- */

/* out: half4 (demodulated GI, variance) at GI resolution. receiver and
 * normal are this frame's GI reservoir targets. */
int restir_svgf_variance(const RestirParams* params, const uint16_t* color, const uint16_t* moments,
	const float* receiver, const float* normal, uint16_t* output, void* stream);

/* One a-trous iteration with taps step texels apart (1, 2, 4, 8, 16). */
int restir_svgf_atrous(const RestirParams* params, int step, const uint16_t* input,
	const float* receiver, const float* normal, uint16_t* output, void* stream);

/* --- Composite, reference and error ------------------------------------ */

/* hdr: half4 full resolution. gi: the denoised (or raw) demodulated GI at
 * GI resolution. di_diffuse, di_specular may be null (black). */
int restir_composite(const RestirParams* params, const RestirGBuffer* gbuffer, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, uint16_t* hdr, void* stream);

/* The composite with indirect specular (fs_composite.sc:48-143 whole):
 * restir_composite plus the GI-resolution specular target of
 * restir_gi_specular, upsampled with the same weights as the diffuse GI and
 * multiplied back by the split-sum specular albedo, the occlusion and
 * params->composite_specular. specular may be null (then equal to
 * restir_composite). */
int restir_composite_specular(const RestirParams* params, const RestirGBuffer* gbuffer, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, const uint16_t* specular, uint16_t* hdr,
	void* stream);

/* Indirect specular (fs_specular.sc, renderer.cpp:835-855), at GI
 * resolution: one GGX visible-normal ray per pixel, traced through the depth
 * buffer then the BVH (the stackless walk of a fragment shader) then the sky;
 * the radiance at a visible hit from last frame's HDR image (previous_hdr),
 * else from the hit's direct, bounce and emitted light; demodulated by the
 * specular albedo, clamped, and blended into the reprojected history
 * (specular_history, same surface only) over 4 to 32 frames by roughness.
 * Output RGBA16F: rgb demodulated radiance, a history length. The history is
 * last frame's GI targets (receiver, normal, colour). specular must not
 * alias specular_history. */
int restir_gi_specular(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const float* shadow_atlas, const uint16_t* surface_light, const uint16_t* previous_hdr,
	const uint16_t* specular_history, uint16_t* specular, void* stream);

/* No reference counterpart: the bytes of device workspace that
 * restir_gi_specular_wavefront needs for these params (56 bytes per GI
 * pixel, in five regions each rounded up to 256). */
uint64_t restir_gi_specular_workspace_bytes(const RestirParams* params);

/* restir_gi_specular as a wavefront, with identical outputs: a rays pass
 * (reflection directions and depth-buffer marches) appends the rays the
 * march does not answer to a queue in the workspace, a persistent tracer
 * runs the stackless walk over the queue (a lane takes the next ray as soon
 * as its own ends), and a shading pass completes fs_specular.sc from the
 * recorded hits. workspace: 256-byte aligned device memory of at least
 * restir_gi_specular_workspace_bytes; it must not be shared with a call
 * whose kernels may overlap this one's. */
int restir_gi_specular_wavefront(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const float* shadow_atlas, const uint16_t* surface_light, const uint16_t* previous_hdr,
	const uint16_t* specular_history, uint16_t* specular, void* workspace, uint64_t workspace_bytes, void* stream);

/* The running mean of the composite in FP64 (fs_reference.sc):
 * mean = mean * (1 - w) + color * w with w = 1 / (frames + 1), NaN colours
 * keep the mean. mean: 3 planes of width * height doubles (r, g, b);
 * alpha: one byte per pixel, the composite's alpha of the last frame.
 * Images of more than 2^32 - 1 pixels return RESTIR_ERROR_TOO_LARGE. */
int restir_reference_accumulate(const RestirParams* params, const uint16_t* hdr, double* mean,
	uint8_t* alpha, uint32_t frames, void* stream);

/* Bytes of scratch memory restir_error needs for an image of the given size. */
uint64_t restir_error_scratch_bytes(uint32_t width, uint32_t height);

/* The error of an image against the reference (cs_error.sc), reduced in
 * FP64 in a fixed order: out[0] relative MSE, out[1] mean luminance of the
 * image, out[2] mean luminance of the reference, out[3] pixels compared.
 * scratch: restir_error_scratch_bytes bytes of device memory. Images of more
 * than 2^32 - 1 pixels return RESTIR_ERROR_TOO_LARGE. */
int restir_error(const RestirParams* params, const uint16_t* display, const double* mean,
	const uint8_t* alpha, double* out, void* scratch, void* stream);

/* restir_error for callers that cannot allocate device memory: hosts such as
 * game engines whose own memory manager owns the whole device budget and
 * hands out no more, and real-time loops that must never enter the driver's
 * allocator (cudaMalloc and cudaFree can synchronise the device and stall the
 * frame). No counterpart in the reference. The caller passes only inputs and
 * the 4-double output; the reduction's partial records live in a 64 KB array
 * inside the library, which every device that loads the library keeps until
 * the process exits. Limit: width * height <= 8,388,608 pixels (3840x2160
 * fits); larger images return RESTIR_ERROR_TOO_LARGE. The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current, so make it before any stream capture; the address is
 * kept until the process exits, so do not call this entry point again after
 * resetting the device (cudaDeviceReset) in the same process. All calls share
 * the one array: calls whose kernels overlap on the GPU (on two streams, say)
 * race on it and must be ordered by the caller. Nothing in the array needs
 * to start at zero; each call overwrites the records it reads. */
int restir_error_noalloc(const RestirParams* params, const uint16_t* display, const double* mean,
	const uint8_t* alpha, double* out, void* stream);

/* The byte size of a public struct of this ABI by its name ("RestirParams",
 * "RestirSettings", ...; every struct of the include/ headers), 0 for an
 * unknown name: a binding in another language checks its copies of the
 * layouts against it. Host only. */
uint64_t restir_struct_size(const char* name);

/* Reads and clears the device status word: bit 0 a traversal reached its
 * step cap, bit 1 a hash grid probe sequence was exhausted, bit 2 a ray
 * queue was full (rays past its capacity are not traced), bit 3 a
 * tensor-core step of the radiance cache failed (a bounded wait gave up or a
 * shared-memory tile was misaligned; that launch's results are invalid), bit
 * 4 an index out of range (bounds-checked builds, RESTIR_CHECKS=1, only). */
int restir_status(uint32_t* flags);

/* Work counters: waits for the device, returns the counts gathered since the
 * last call (8 values: nearest-hit ray casts, short-stack closest-hit rays,
 * stackless any-hit rays, depth-buffer marches, BVH node fetches, triangle
 * tests, depth-buffer steps, rays cut short by the step cap or a full
 * traversal stack), clears them, and turns counting on or
 * off for the launches that follow. Off by default; a counted frame does
 * extra atomics. No counterpart in the reference (its profiler counts
 * time only, ui.cpp:20-66). */
int restir_counters(int enable, uint64_t* counters);

/* Evaluates one numeric convention of restir_numeric.h on the device, for
 * tests: fn 0 sin, 1 cos, 2 exp, 3 half round trip (hardware), 4 half round
 * trip (restir_numeric.h), 5 unorm8 store, 6 floor(log2), 7 x^64. No
 * counterpart in the reference (a test hook). */
int restir_numeric_eval(int fn, const float* input, float* output, uint32_t n, void* stream);

/* A bandwidth probe with the traversal kernels' fetch pattern (a measurement
 * hook, no counterpart in the reference): blocks x 256 threads each gather
 * `gathers` rows of 32 bytes (two 16-byte read-only loads, the size of a BVH
 * node) at seeded random indices of rows (row_count rows, 16-byte aligned)
 * and write one float each to out (blocks x 256 floats). Fetched bytes =
 * blocks x 256 x gathers x 32; with a buffer that fits the L2 the rate is
 * the L2's for node-sized gathers. */
int restir_gather_probe(const float* rows, uint32_t row_count, uint32_t blocks, uint32_t gathers, uint32_t seed,
	float* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RESTIR_GPU_H */
