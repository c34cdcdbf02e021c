/*
 * ORACLE (test infrastructure): the C interface of the CPU restatement.
 *
 * One function per pass of include/restir_gpu.h, with the same arguments
 * but host pointers, no stream, and (for oracle_error) no scratch. Tests,
 * __graft_entry__.smoke() and bench.py's CPU baseline load liboracle.so
 * through ctypes; nothing in the product links it.
 */
#ifndef ORACLE_H
#define ORACLE_H

#include "../include/restir_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

int oracle_trace(const RestirParams* params, const RestirScene* scene, const float* rays,
	int32_t* hit_triangle, float* hit_distance, uint32_t n, int kind);
int oracle_shadow_atlas(const RestirParams* params, const RestirScene* scene, float* atlas);
int oracle_gbuffer_primary(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer);
int oracle_grid_clear(const RestirParams* params, uint32_t* grid);
int oracle_grid_insert(const RestirParams* params, const RestirGBuffer* gbuffer, uint32_t* grid);
int oracle_di_temporal(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirDiReservoirs* previous, const RestirDiReservoirs* output);
int oracle_di_spatial(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirDiReservoirs* current, uint16_t* diffuse, uint16_t* specular);
int oracle_gi_temporal(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, const RestirGiReservoirs* output);
int oracle_gi_spatial(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	const RestirGiReservoirs* current, const uint32_t* current_grid, const RestirGiHistory* history,
	const float* shadow_atlas, const uint16_t* surface_light, uint16_t* color, uint16_t* moments);
int oracle_svgf_variance(const RestirParams* params, const uint16_t* color, const uint16_t* moments,
	const float* receiver, const float* normal, uint16_t* output);
int oracle_svgf_atrous(const RestirParams* params, int step, const uint16_t* input,
	const float* receiver, const float* normal, uint16_t* output);
int oracle_composite(const RestirParams* params, const RestirGBuffer* gbuffer, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, uint16_t* hdr);
int oracle_reference_accumulate(const RestirParams* params, const uint16_t* hdr, double* mean,
	uint8_t* alpha, uint32_t frames);
int oracle_error(const RestirParams* params, const uint16_t* display, const double* mean,
	const uint8_t* alpha, double* out);

/* Rays counted by the last oracle call of a GI or DI pass (BVH rays and
 * screen-space marches), and the node visits and triangle tests of its BVH
 * rays: the algorithmic work the roofline figures are computed from. */
void oracle_last_counts(uint64_t* counts /* [5]: bvh rays, screen rays, node visits, triangle tests, pixels */);

/* gridCellSize, gridJitter and gridKey (hashgrid.sh:82-127) for n
 * positions, normals and random pairs: cell size bits, first slot, checksum.
 * constants: min cell, pixel size, cell pixels. */
void oracle_grid_keys(const float* camera, const float* constants, uint32_t table_size, const float* positions,
	const float* normals, const float* randoms, uint32_t n, uint32_t* cell_bits, uint32_t* slots, uint32_t* checksums);

/* The host evaluation of restir_numeric_eval's functions (same fn codes). */
void oracle_numeric_eval(int fn, const float* input, float* output, uint32_t n);

/* The host side of a frame (oracle_frame.cpp): the renderer's defaults, the
 * uniforms of a frame and the state carried on (renderer.cpp:435-731,
 * 1119-1124), the display passes' uniforms, and the seeded procedural
 * workload scenes. Same arguments as the product's restir_settings_default,
 * restir_frame_params, restir_frame_advance, restir_display_params and
 * restir_mesh_procedural / _describe / _destroy. */
struct RestirSettings;
struct RestirMeshDesc;
struct RestirBvhDesc;
struct RestirFrameInput;
struct RestirFrameState;
struct RestirFramePlan;
struct RestirDisplayParams;
void oracle_settings_default(struct RestirSettings* settings);
int oracle_frame_params(const struct RestirSettings* settings, const struct RestirMeshDesc* scene, uint32_t light_count,
	const struct RestirBvhDesc* bvh, const struct RestirFrameInput* input, const struct RestirFrameState* state,
	RestirParams* params, struct RestirFramePlan* plan);
void oracle_frame_advance(const RestirParams* params, const struct RestirFramePlan* plan,
	const struct RestirFrameInput* input, struct RestirFrameState* state);
int oracle_display_params(const float* inv_view_proj, const float* previous_unjittered_view_proj, uint32_t width,
	uint32_t height, int taa, int taa_history_valid, int auto_exposure, int exposure_valid, float adaptation_speed,
	float delta_time, float exposure_ev, int tonemapper, int pass_through, int reference_view,
	struct RestirDisplayParams* out);
void* oracle_mesh_procedural(int kind, uint32_t seed, uint32_t target_triangles);
int oracle_mesh_describe(void* mesh, struct RestirMeshDesc* out);
void oracle_mesh_destroy(void* mesh);

/* Threads the oracle uses; 0: all hardware threads. */
void oracle_set_threads(int threads);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif /* ORACLE_H */
