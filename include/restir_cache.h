/*
 * restir-b200: the radiance cache, C ABI.
 *
 * No reference counterpart: the reference renderer has no learned cache.
 * The cache stands in for previousIndirect (shaders/restir.sh:265-298, called
 * at restir.sh:519 and 525), the indirect light that leaves a GI sample point:
 * instead of last frame's denoised irradiance at the point's screen position
 * (zero off screen), a small network predicts it from the point's position,
 * direction, normal, roughness and albedo, trained online on the radiance
 * of path suffixes the renderer traces itself (Mueller, Rousselle, Novak,
 * Keller, "Real-time Neural Radiance Caching for Path Tracing", 2021).
 *
 * Network (fixed shape):
 *   - input encoding: a multiresolution hash grid of position (Mueller,
 *     Evans, Schied, Keller, "Instant Neural Graphics Primitives with a
 *     Multiresolution Hash Encoding", 2022): RESTIR_CACHE_LEVELS levels of
 *     RESTIR_CACHE_FEATURES half-precision features, trilinear, level l at
 *     resolution floor(n_min * b^l), b = (n_max / n_min)^(1 / (levels - 1)),
 *     corners stored in 2x2x2 bricks of 8 consecutive entries (one 32-byte
 *     sector: a cell's corners touch 3.4 sectors on average, not up to 8),
 *     brick (x / 2, y / 2, z / 2) numbered densely where the level's bricks
 *     fit the table (8 * ceil((res + 1) / 2)^3 <= entries), else hashed as
 *     (bx * 1 ^ by * 2654435761 ^ bz * 805459861) mod (entries / 8);
 *   - 64 inputs: the 32 encoded features, direction (3), normal (3),
 *     roughness, albedo (3), a constant 1, zeros; rounded to bfloat16;
 *   - 4 hidden layers of 64 (ReLU), 3 outputs (linear) padded to 16, no
 *     biases; bfloat16 weights on the tensor cores with FP32 accumulation,
 *     FP32 master weights;
 *   - loss: relative L2, sum over RGB of (y - t)^2 / (y^2 + 0.01) with y held
 *     constant in the denominator, mean over samples and channels; the
 *     backward pass is scaled by a dynamic loss scale (halved and the step
 *     skipped on a non-finite gradient, doubled after 1000 clean steps);
 *   - Adam (beta1, beta2, epsilon from the config) on the weights and the
 *     hash-grid features.
 * The cache's value for a point is max(output, 0): demodulated irradiance,
 * like the history color it replaces (multiply by the point's albedo).
 *
 * Memory: one caller-owned device block of restir_cache_state_bytes, 256-byte
 * aligned; restir_cache_layout gives the byte offset of every region in it.
 * Queries: 16 floats each, (position xyz, roughness), (normal xyz, valid),
 * (direction xyz, 0), (albedo rgb, 0); valid is 1 for a query and 0 for a
 * padding row, whose value comes back with alpha 0. Targets: 4 floats,
 * (rgb, weight); a sample's loss and gradient are scaled by its weight (0
 * drops it).
 */
#ifndef RESTIR_CACHE_H
#define RESTIR_CACHE_H

#include <stdint.h>

#include "restir_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RESTIR_CACHE_LEVELS 16
#define RESTIR_CACHE_FEATURES 2
#define RESTIR_CACHE_INPUTS 64
#define RESTIR_CACHE_HIDDEN 64
#define RESTIR_CACHE_HIDDEN_LAYERS 4
#define RESTIR_CACHE_OUTPUTS 16      /* 3 used */
/* Weights: 4 matrices of 64 x 64 then 16 x 64, each [out][in] row-major. */
#define RESTIR_CACHE_WEIGHTS (4 * 64 * 64 + 16 * 64)
#define RESTIR_CACHE_QUERY_FLOATS 16
#define RESTIR_CACHE_MAX_BATCH (1u << 20)
/* A row of weight_partials: the weight gradients, then the block's loss sum. */
#define RESTIR_CACHE_PARTIAL_STRIDE (RESTIR_CACHE_WEIGHTS + 64)

typedef struct RestirCacheConfig
{
	float bounds_min[3];      /* scene box the encoding covers */
	float bounds_max[3];
	uint32_t table_log2;      /* hash table entries per level, log2 (12-22) */
	float n_min;              /* coarsest resolution (cells across the box) */
	float n_max;              /* finest resolution */
	float learning_rate;
	float beta1;
	float beta2;
	float epsilon;
	float initial_loss_scale;
	uint32_t seed;            /* weight initialisation */
} RestirCacheConfig;

/* Byte offsets in the state block. */
typedef struct RestirCacheLayout
{
	uint64_t weights;         /* float[RESTIR_CACHE_WEIGHTS], master */
	uint64_t weights_bf16;    /* uint16[RESTIR_CACHE_WEIGHTS], the tensor-core copy */
	uint64_t weight_m;        /* float[RESTIR_CACHE_WEIGHTS], Adam first moment */
	uint64_t weight_v;        /* second moment */
	uint64_t weight_grad;     /* float[RESTIR_CACHE_WEIGHTS], last gradient (unscaled) */
	uint64_t weight_partials; /* float[partial blocks][RESTIR_CACHE_PARTIAL_STRIDE], scaled */
	uint64_t table;           /* float[levels][entries][features], master */
	uint64_t table_half;      /* uint16 copy the queries read */
	uint64_t table_m;
	uint64_t table_v;
	uint64_t table_grad;      /* float, the last gradient (unscaled) */
	uint64_t table_grad_fixed; /* int64, the loss-scaled gradient summed in units of 2^-32
	                              (fixed point: the sum does not depend on the order of the
	                              samples' scattered contributions) */
	uint64_t scalars;         /* RestirCacheScalars */
	uint64_t bytes;           /* total */
	uint32_t entries;         /* per level */
	uint32_t partial_blocks;  /* rows of weight_partials */
	float level_scale[RESTIR_CACHE_LEVELS]; /* resolution of each level */
	uint32_t level_dense[RESTIR_CACHE_LEVELS]; /* 1: indexed densely */
} RestirCacheLayout;

typedef struct RestirCacheScalars
{
	float loss_scale;
	uint32_t step;            /* Adam steps taken */
	uint32_t clean_steps;     /* since the loss scale last changed */
	uint32_t skipped_steps;   /* non-finite gradients */
	float loss;               /* last training batch's mean loss */
	uint32_t nonfinite;       /* the last gradients were not finite */
	uint32_t samples;         /* last batch size */
	uint32_t blocks;          /* partial rows the last gradients wrote */
	float beta1_power;        /* beta1^step, beta2^step (running products) */
	float beta2_power;
	uint32_t pad[6];
} RestirCacheScalars;

/* Fills cfg with the defaults: box [0,1]^3, 2^18 entries per level,
 * n_min 16, n_max 2048, learning rate 1e-2, beta1 0.9, beta2 0.99,
 * epsilon 1e-15, loss scale 128, seed 1337. */
void restir_cache_config_default(RestirCacheConfig* cfg);

/* The layout of the state block for cfg (host only). Returns
 * RESTIR_ERROR_INVALID_ARGUMENT for a bad config. */
int restir_cache_layout(const RestirCacheConfig* cfg, RestirCacheLayout* layout);

uint64_t restir_cache_state_bytes(const RestirCacheConfig* cfg);

/* Seeded initialisation: weights uniform in +-sqrt(6 / (fan_in + fan_out)),
 * features uniform in +-1e-4, moments and gradients zero. */
int restir_cache_init(const RestirCacheConfig* cfg, void* state, void* stream);

/* The cache's value (max(output, 0) in rgb, the query's valid flag in
 * alpha) for n queries, as half4. */
int restir_cache_query(const RestirCacheConfig* cfg, const void* state, const float* queries, uint32_t n,
	uint16_t* output, void* stream);

/* The network's 64 bfloat16 inputs for n queries (for tests). */
int restir_cache_features(const RestirCacheConfig* cfg, const void* state, const float* queries, uint32_t n,
	uint16_t* features, void* stream);

/* The raw network outputs (16 floats per query, for tests). */
int restir_cache_forward(const RestirCacheConfig* cfg, const void* state, const float* queries, uint32_t n,
	float* outputs, void* stream);

/* Gradients of the loss over a batch of n <= RESTIR_CACHE_MAX_BATCH samples:
 * weight_grad and table_grad (both unscaled when this returns), the loss and
 * the non-finite flag in the scalars. */
int restir_cache_gradients(const RestirCacheConfig* cfg, void* state, const float* queries, const float* targets,
	uint32_t n, void* stream);

/* One Adam step from the gradients of the last restir_cache_gradients (or
 * none, with the loss scale halved, when they were not finite). */
int restir_cache_adam(const RestirCacheConfig* cfg, void* state, void* stream);

/* restir_cache_gradients then restir_cache_adam. */
int restir_cache_train(const RestirCacheConfig* cfg, void* state, const float* queries, const float* targets,
	uint32_t n, void* stream);

/* --- the cache in the GI passes (params->radiance_cache > 0.5) ---------- */

/* restir_gi_temporal_wavefront with the cache standing in for
 * previousIndirect at every sample point the pass shades: the candidates'
 * hits and last frame's reservoirs' samples each get a query row (the
 * point's surface as evaluateSample finds it, the direction toward its
 * receiver), answered in one restir_cache_query before the shading.
 * workspace: restir_gi_temporal_workspace_bytes(params) (which includes the
 * cache's rows and the training batch when params->radiance_cache is set).
 * The rows: candidate (pixel * initial_candidates + k) first, then last
 * frame's reservoir i at GI pixels x initial_candidates + i; the values
 * (half4) follow the same order. */
int restir_gi_temporal_cached(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, const RestirGiReservoirs* output, const RestirCacheConfig* cache_config,
	const void* cache_state, void* workspace, uint64_t workspace_bytes, void* stream);

/* restir_gi_spatial with the cache's values for this frame's reservoirs
 * (rows 0 .. GI pixels - 1 of the same workspace). */
int restir_gi_spatial_cached(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiReservoirs* current, const uint32_t* current_grid, const RestirGiHistory* history,
	const float* shadow_atlas, const uint16_t* surface_light, uint16_t* color, uint16_t* moments,
	const RestirCacheConfig* cache_config, const void* cache_state, void* workspace, uint64_t workspace_bytes,
	void* stream);

/* The cache-only form of the GI (no reference counterpart): the cache
 * queried at every GI pixel's own surface, exactly as the training points
 * query it (position, normal, view direction, roughness, diffuse albedo), in
 * place of the GI temporal and spatial passes; no GI ray is traced. Writes
 * the GI targets the later passes read: color (demodulated irradiance,
 * clamped as the spatial pass clamps), moments, and the receiver and normal
 * rows (sample rows zeroed). workspace: restir_gi_temporal_workspace_bytes
 * with params->radiance_cache set. */
int restir_gi_from_cache(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirCacheConfig* cache_config, const void* cache_state, void* workspace, uint64_t workspace_bytes,
	const RestirGiReservoirs* output, uint16_t* color, uint16_t* moments, void* stream);

/* One training step on params->cache_training_samples path suffixes. Half of
 * them start at seeded GI pixels' G-buffer surfaces; the other half start at
 * the first hits of the previous frame's call's suffixes (where the GI
 * passes query the cache), which the workspace keeps between calls: pass the
 * same workspace every frame. Rows the previous call did not write (the first
 * call, another frame index than the previous one + 1) are padding. Each takes
 * a cosine-distributed direction and its first hit through the BVH; the
 * target is the light leaving that hit toward the start (point light with the
 * shadow atlas, the triangle's emission, the sky on a miss) plus the hit's
 * albedo times the cache's own value there. */
int restir_cache_train_frame(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const float* shadow_atlas, const RestirCacheConfig* cache_config, void* cache_state, void* workspace,
	uint64_t workspace_bytes, void* stream);

/* A check of the bounded wait that guards every tensor-core step (no
 * reference counterpart): one block waits, exactly as the cache's kernels
 * wait for their MMAs, on an mbarrier that no one arrives at, for at most
 * `polls` polls (1 to 4,194,304), and no MMA is issued. The wait gives up,
 * raises status bit 3 (value 8, read and cleared by restir_status) and the
 * kernel returns; *result (device memory) is 0 then. Lets a test show that
 * a failed tensor-core step ends with an error status instead of a hang. */
int restir_cache_wait_check(uint32_t polls, uint32_t* result, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RESTIR_CACHE_H */
