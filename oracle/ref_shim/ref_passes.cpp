/*
 * ORACLE (test infrastructure): a C interface over the reference's own
 * shader code (pkonecki/restir, the shaders directory), compiled as C++ by oracle/Makefile
 * into oracle/_ref/libref_shaders.so after oracle/ref_shim/glsl_to_cpp.py
 * has made the shader files C++ (see shader_shim.h). Tests hand the same
 * inputs to these functions and to the oracle restatement (oracle.cpp and its headers) and
 * require equal outputs: that pins the restatement, and through it the CUDA
 * kernels, to the reference's shader source.
 *
 * This file is compiled once per shader file (REF_PASS selects which): the
 * shaders declare their uniforms and resources as globals of the same
 * names and guard their headers, so each needs a translation unit of its
 * own; inside it the shader's code sits in a namespace.
 * Dispatch is sequential: compute invocations run one after another in
 * row-major pixel order, a legal schedule of the shader (for the grid
 * insert's atomics it is the order in which the first 32 arrivals are the
 * lowest pixel indices, the oracle's deterministic mode).
 *
 *   ref_trace          bvh.sh:32-319 (traceBvh with BVH_SHARED_STACK for
 *                      closest hits, traceBvhStackless for any hits and
 *                      stackless closest hits)
 *   ref_grid_keys      hashgrid.sh:82-127 (gridCellSize, gridJitter, gridKey)
 *   ref_grid_insert    cs_grid_insert.sc:40-73 with hashgrid.sh:132-200
 *   ref_gi_temporal    cs_restir_temporal.sc:57-297 (its 4x8 groups run as 32
 *                      lane threads meeting at the shader's barriers)
 *   ref_gi_spatial     cs_restir_spatial.sc:95-246
 *   ref_di_temporal    cs_di_temporal.sc:32-180
 *   ref_di_spatial     cs_di_spatial.sc:30-169
 *   ref_svgf_variance  fs_svgf_variance.sc:29-76
 *   ref_svgf_atrous    fs_svgf_atrous.sc:29-95
 *   ref_composite      fs_composite.sc:48-143
 *   ref_gi_specular    fs_specular.sc:127-226
 * with restir.sh, di.sh, brdf.sh, shadow.sh, sky.sh, svgf.sh, compute.sh and
 * bvh.sh underneath. Fragment passes run at texel centres (v_texcoord0 =
 * (pixel + 0.5) / size) and store gl_FragColor in the target's format.
 * The arguments are those of the oracle's function of the same pass.
 */
#include "ref_common.h"

using namespace refsh;

// The resources and uniforms of restir.sh (with shadow.sh, bvh.sh, sky.sh and
// hashgrid.sh) as Renderer::render binds them for the GI passes
// (renderer.cpp:693-802); the values come from RestirParams, whose fields
// are the uniforms by name. GRID_CAMERA: the camera the bound grid's cell
// sizes were chosen from.
#define BIND_RESTIR_SH(NS, P, SCENE, GB, HISTORY, ATLAS, SURFACE_LIGHT, GRID, GRID_CAMERA) \
	do \
	{ \
		const uint32_t W_ = (P)->width, H_ = (P)->height, w_ = (P)->gi_width, h_ = (P)->gi_height; \
		g_originBottomLeft = (P)->origin_bottom_left > 0.5f; \
		NS::s_albedo = image((GB)->albedo, W_, H_, kFormatBGRA8); \
		NS::s_normal = image((GB)->normal, W_, H_, kFormatBGRA8); \
		NS::s_depth = image((GB)->depth, W_, H_, kFormatR32F); \
		NS::s_historyColor = image((HISTORY)->color, w_, h_, kFormatRGBA16F); \
		NS::s_historyNormal = image((HISTORY)->normal, w_, h_, kFormatRGBA32F); \
		NS::s_historyReceiver = image((HISTORY)->receiver, w_, h_, kFormatRGBA32F); \
		NS::s_surfaceLight = image((SURFACE_LIGHT), W_, H_, kFormatRGBA16F); \
		bindShadow##NS(P, ATLAS); \
		NS::u_sceneInvViewProj = matrix((P)->inv_view_proj); \
		NS::u_sceneViewProj = matrix((P)->view_proj); \
		NS::u_previousViewProj = matrix((P)->prev_view_proj); \
		NS::u_lightPosition = vec4At((P)->light_position); \
		NS::u_lightColor = vec4At((P)->light_color); \
		NS::u_frameInfo = vec4((P)->frame_index, (P)->history_valid, (P)->origin_bottom_left, (P)->multiple_bounces); \
		NS::u_screenInfo = vec4(float(w_), float(h_), 1.0f / float(w_), 1.0f / float(h_)); \
		NS::u_sceneInfo = vec4((P)->scene_scale, (P)->boiling_filter, (P)->jacobian_clamp, (P)->outlier_clamp); \
		NS::u_lightingInfo = vec4((P)->surface_light_scale, (P)->emission_scale, 0.0f, 0.0f); \
		NS::u_restirOptions = vec4(float((P)->initial_candidates), float((P)->temporal_taps), \
			float((P)->spatial_taps), float((P)->trace_steps)); \
		NS::u_gridInfo = vec4((P)->grid_min_cell, (P)->grid_pixel_size, (P)->grid_cell_pixels, (P)->world_space_reuse); \
		NS::u_gridCamera = vec4((GRID_CAMERA)[0], (GRID_CAMERA)[1], (GRID_CAMERA)[2], 1.0f); \
		NS::b_grid.data = const_cast<uint32_t*>(GRID); \
		NS::b_grid.count = (GRID) != nullptr ? size_t(65536u) * (2u + 32u) : 0u; \
		NS::u_skyZenith = vec4At((P)->sky_zenith); \
		NS::u_skyHorizon = vec4At((P)->sky_horizon); \
		NS::u_skyGround = vec4At((P)->sky_ground); \
		NS::b_scene.data = reinterpret_cast<vec4*>(const_cast<float*>((SCENE)->bvh)); \
		NS::b_scene.count = (SCENE)->triangle_offset + 4u * (SCENE)->triangle_count; \
		NS::u_bvhInfo = vec4(float((SCENE)->triangle_offset), 0.0f, float((SCENE)->node_count), float((P)->ray_mode)); \
	} while (false)

// shadow.sh's resources (renderer.cpp:527-593, 1282-1318).
#define DEFINE_BIND_SHADOW(NS) \
	void bindShadow##NS(const RestirParams* P, const float* atlas) \
	{ \
		const uint32_t F = P->shadow_face_size; \
		NS::s_shadowMap = image(atlas, 3u * F, 2u * F, kFormatR32F); \
		for (int f = 0; f < 6; ++f) \
		{ \
			NS::u_shadowViewProj[f] = matrix(P->shadow_view_proj[f]); \
		} \
		NS::u_shadowInfo = vec4(P->shadow_far, P->shadow_tan_half_fov, P->shadow_inv_face_size, P->origin_bottom_left); \
		NS::u_shadowOptions = vec4(P->shadows_enabled, 0.0f, 0.0f, 0.0f); \
	}

// di.sh's resources and uniforms (renderer.cpp:627-685).
#define BIND_DI_SH(NS, P, SCENE, GB) \
	do \
	{ \
		const uint32_t W_ = (P)->width, H_ = (P)->height; \
		g_originBottomLeft = (P)->origin_bottom_left > 0.5f; \
		NS::s_albedo = image((GB)->albedo, W_, H_, kFormatBGRA8); \
		NS::s_normal = image((GB)->normal, W_, H_, kFormatBGRA8); \
		NS::s_depth = image((GB)->depth, W_, H_, kFormatR32F); \
		NS::s_shadingNormal = image((GB)->shading_normal, W_, H_, kFormatBGRA8); \
		NS::b_lights.data = reinterpret_cast<vec4*>(const_cast<float*>((SCENE)->lights)); \
		NS::b_lights.count = 4u * (SCENE)->light_count; \
		NS::u_sceneInvViewProj = matrix((P)->inv_view_proj); \
		NS::u_cameraPosition = vec4At((P)->camera_position); \
		NS::u_sceneInfo = vec4((P)->scene_scale, (P)->boiling_filter, (P)->jacobian_clamp, (P)->outlier_clamp); \
		NS::u_frameInfo = vec4((P)->frame_index, (P)->history_valid, (P)->origin_bottom_left, (P)->multiple_bounces); \
		NS::u_diInfo = vec4(float((P)->di_light_count), float((P)->di_candidates), float((P)->di_spatial_taps), \
			(P)->di_history_valid); \
		NS::u_screenSize = vec4(float(W_), float(H_), 1.0f / float(W_), 1.0f / float(H_)); \
		NS::b_scene.data = reinterpret_cast<vec4*>(const_cast<float*>((SCENE)->bvh)); \
		NS::b_scene.count = (SCENE)->triangle_offset + 4u * (SCENE)->triangle_count; \
		NS::u_bvhInfo = vec4(float((SCENE)->triangle_offset), 0.0f, float((SCENE)->node_count), float((P)->ray_mode)); \
	} while (false)


#if REF_PASS == 1 // bvh.sh and cs_grid_insert.sc: ref_trace, ref_grid_keys, ref_grid_insert

// --- bvh.sh --------------------------------------------------------------------------------------

namespace shader_bvh
{
#define BVH_STAGE 0
#define BVH_SHARED_STACK 1
#include "bvh.sh"
#undef BVH_SHARED_STACK
#undef BVH_STAGE
} // namespace shader_bvh


// --- hashgrid.sh and cs_grid_insert.sc -----------------------------------------------------------

namespace shader_grid_insert
{
#include "cs_grid_insert.sc"
} // namespace shader_grid_insert


namespace
{

void bindBvh(const RestirScene* scene)
{
	const uint32_t vec4Count = scene->triangle_offset + 4u * scene->triangle_count;
	shader_bvh::b_scene.data = reinterpret_cast<vec4*>(const_cast<float*>(scene->bvh));
	shader_bvh::b_scene.count = vec4Count;
	shader_bvh::u_bvhInfo = vec4(float(scene->triangle_offset), 0.0f, float(scene->node_count), 2.0f);
}

} // namespace

extern "C"
{

/* The reference's traversal of n rays (8 floats each: origin, tmax,
 * direction, unused), as restir_trace / oracle_trace take them: triangle id
 * (BVH order) or -1, and the distance (tmax when nothing was hit).
 * kind: RESTIR_TRACE_CLOSEST (nearest-first shared short stack),
 * RESTIR_TRACE_ANY, RESTIR_TRACE_CLOSEST_STACKLESS. */
int ref_trace(const RestirScene* scene, const float* rays, int32_t* hit_triangle, float* hit_distance, uint32_t n,
	int kind)
{
	if (scene == nullptr || rays == nullptr || hit_triangle == nullptr || hit_distance == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	if (kind != RESTIR_TRACE_CLOSEST && kind != RESTIR_TRACE_ANY && kind != RESTIR_TRACE_CLOSEST_STACKLESS)
	{
		return RESTIR_ERROR_UNSUPPORTED;
	}
	bindBvh(scene);
	shader_bvh::g_bvhThread = 0;
	for (uint32_t i = 0; i < n; ++i)
	{
		const float* r = rays + 8 * size_t(i);
		vec3 origin(r[0], r[1], r[2]);
		vec3 direction(r[4], r[5], r[6]);
		float distance = r[3];
		int hit;
		if (kind == RESTIR_TRACE_CLOSEST_STACKLESS)
		{
			hit = shader_bvh::bvhAvailable() ? shader_bvh::traceBvhStackless(origin, direction, false, distance) : -1;
		}
		else
		{
			hit = shader_bvh::traceBvh(origin, direction, r[3], kind == RESTIR_TRACE_ANY, distance);
		}
		hit_triangle[i] = hit;
		hit_distance[i] = distance;
	}
	return RESTIR_OK;
}

/* gridCellSize, gridJitter and gridKey for n positions, normals (3 floats
 * each) and random pairs, with the same arguments as oracle_grid_keys
 * (constants: min cell, pixel size, cell pixels). The reference's table has
 * 65,536 slots (hashgrid.sh:53-55); other sizes are refused. */
int ref_grid_keys(const float* camera, const float* constants, uint32_t table_size, const float* positions,
	const float* normals, const float* randoms, uint32_t n, uint32_t* cell_bits, uint32_t* slots, uint32_t* checksums)
{
	if (table_size != 65536u)
	{
		return RESTIR_ERROR_UNSUPPORTED;
	}
	using namespace shader_grid_insert;
	u_gridInfo = vec4(constants[0], constants[1], constants[2], 1.0f);
	u_gridCamera = vec4(camera[0], camera[1], camera[2], 1.0f);
	for (uint32_t i = 0; i < n; ++i)
	{
		vec3 position(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
		vec3 normal(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]);
		float cellSize = gridCellSize(position);
		vec3 jittered = gridJitter(position, normal, cellSize, randoms[2 * i], randoms[2 * i + 1]);
		uint slot = 0u, checksum = 0u;
		gridKey(jittered, normal, cellSize, slot, checksum);
		cell_bits[i] = floatBitsToUint(cellSize);
		slots[i] = slot;
		checksums[i] = checksum;
	}
	return RESTIR_OK;
}

/* cs_grid_insert.sc over the GI image, invocations in row-major pixel order,
 * into a cleared grid of the reference's size (T = 65,536, C = 32). Same
 * arguments as oracle_grid_insert. */
int ref_grid_insert(const RestirParams* P, const RestirGBuffer* gbuffer, uint32_t* grid)
{
	if (P == nullptr || gbuffer == nullptr || grid == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	if (P->grid_table_size != 65536u || P->grid_cell_capacity != 32u)
	{
		return RESTIR_ERROR_UNSUPPORTED;
	}
	using namespace shader_grid_insert;
	g_originBottomLeft = P->origin_bottom_left > 0.5f;
	b_grid.data = grid;
	b_grid.count = size_t(65536u) * (2u + 32u);
	s_normal.data = gbuffer->normal;
	s_normal.width = int(P->width);
	s_normal.height = int(P->height);
	s_normal.format = kFormatBGRA8;
	s_depth.data = gbuffer->depth;
	s_depth.width = int(P->width);
	s_depth.height = int(P->height);
	s_depth.format = kFormatR32F;
	u_sceneInvViewProj = matrix(P->inv_view_proj);
	u_frameInfo = vec4(P->frame_index, P->history_valid, P->origin_bottom_left, P->multiple_bounces);
	u_screenInfo = vec4(float(P->gi_width), float(P->gi_height), 1.0f / float(P->gi_width),
		1.0f / float(P->gi_height));
	u_gridInfo = vec4(P->grid_min_cell, P->grid_pixel_size, P->grid_cell_pixels, P->world_space_reuse);
	u_gridCamera = vec4(P->camera_position[0], P->camera_position[1], P->camera_position[2], 1.0f);
	for (uint32_t y = 0; y < P->gi_height; ++y)
	{
		for (uint32_t x = 0; x < P->gi_width; ++x)
		{
			gl_GlobalInvocationID = uvec3(x, y, 0u);
			main();
		}
	}
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 1

#if REF_PASS == 2 // cs_restir_temporal.sc: ref_gi_temporal

namespace shader_gi_temporal
{
#include "cs_restir_temporal.sc"
} // namespace shader_gi_temporal

namespace
{
DEFINE_BIND_SHADOW(shader_gi_temporal)
} // namespace

extern "C"
{

int ref_gi_temporal(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiHistory* history, const uint32_t* previous_grid, const float* shadow_atlas,
	const uint16_t* surface_light, const RestirGiReservoirs* output)
{
	if (P->grid_table_size != 65536u || P->grid_cell_capacity != 32u)
	{
		return RESTIR_ERROR_UNSUPPORTED;
	}
	namespace NS = shader_gi_temporal;
	BIND_RESTIR_SH(shader_gi_temporal, P, scene, gb, history, shadow_atlas, surface_light, previous_grid,
		P->prev_camera_position);
	const uint32_t w = P->gi_width, h = P->gi_height;
	NS::s_historySample = image(history->sample, w, h, kFormatRGBA32F);
	NS::o_sample = image(nullptr, w, h, kFormatRGBA32F, output->sample);
	NS::o_receiver = image(nullptr, w, h, kFormatRGBA32F, output->receiver);
	NS::o_normal = image(nullptr, w, h, kFormatRGBA32F, output->normal);
	dispatchGroups(w, h, 4u, 8u, [] { NS::main(); });
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 2

#if REF_PASS == 3 // cs_restir_spatial.sc: ref_gi_spatial

namespace shader_gi_spatial
{
#include "cs_restir_spatial.sc"
} // namespace shader_gi_spatial

namespace
{
DEFINE_BIND_SHADOW(shader_gi_spatial)
} // namespace

extern "C"
{

int ref_gi_spatial(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiReservoirs* current, const uint32_t* current_grid, const RestirGiHistory* history,
	const float* shadow_atlas, const uint16_t* surface_light, uint16_t* color, uint16_t* moments)
{
	if (P->grid_table_size != 65536u || P->grid_cell_capacity != 32u)
	{
		return RESTIR_ERROR_UNSUPPORTED;
	}
	namespace NS = shader_gi_spatial;
	BIND_RESTIR_SH(shader_gi_spatial, P, scene, gb, history, shadow_atlas, surface_light, current_grid,
		P->camera_position);
	const uint32_t w = P->gi_width, h = P->gi_height;
	NS::s_reservoirSample = image(current->sample, w, h, kFormatRGBA32F);
	NS::s_reservoirReceiver = image(current->receiver, w, h, kFormatRGBA32F);
	NS::s_reservoirNormal = image(current->normal, w, h, kFormatRGBA32F);
	NS::s_historyMoments = image(history->moments, w, h, kFormatRGBA16F);
	NS::o_colorImage = image(nullptr, w, h, kFormatRGBA16F, color);
	NS::o_momentsImage = image(nullptr, w, h, kFormatRGBA16F, moments);
	dispatchSequential(w, h, [] { NS::main(); });
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 3

#if REF_PASS == 4 // cs_di_temporal.sc: ref_di_temporal

namespace shader_di_temporal
{
#include "cs_di_temporal.sc"
} // namespace shader_di_temporal

extern "C"
{

int ref_di_temporal(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirDiReservoirs* previous, const RestirDiReservoirs* output)
{
	namespace NS = shader_di_temporal;
	BIND_DI_SH(shader_di_temporal, P, scene, gb);
	const uint32_t W = P->width, H = P->height;
	NS::s_previousSample = image(previous->sample, W, H, kFormatRGBA32F);
	NS::s_previousReceiver = image(previous->receiver, W, H, kFormatRGBA32F);
	NS::s_previousNormal = image(previous->normal, W, H, kFormatRGBA16F);
	NS::u_previousViewProj = matrix(P->prev_view_proj);
	NS::u_diPrevious = vec4At(P->prev_camera_position);
	NS::o_sampleImage = image(nullptr, W, H, kFormatRGBA32F, output->sample);
	NS::o_receiverImage = image(nullptr, W, H, kFormatRGBA32F, output->receiver);
	NS::o_normalImage = image(nullptr, W, H, kFormatRGBA16F, output->normal);
	dispatchSequential(W, H, [] { NS::main(); });
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 4

#if REF_PASS == 5 // cs_di_spatial.sc: ref_di_spatial

namespace shader_di_spatial
{
#include "cs_di_spatial.sc"
} // namespace shader_di_spatial

extern "C"
{

int ref_di_spatial(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirDiReservoirs* current, uint16_t* diffuse, uint16_t* specular)
{
	namespace NS = shader_di_spatial;
	BIND_DI_SH(shader_di_spatial, P, scene, gb);
	const uint32_t W = P->width, H = P->height;
	NS::s_reservoirSample = image(current->sample, W, H, kFormatRGBA32F);
	NS::s_reservoirReceiver = image(current->receiver, W, H, kFormatRGBA32F);
	NS::s_reservoirNormal = image(current->normal, W, H, kFormatRGBA16F);
	NS::o_diffuseImage = image(nullptr, W, H, kFormatRGBA16F, diffuse);
	NS::o_specularImage = image(nullptr, W, H, kFormatRGBA16F, specular);
	dispatchSequential(W, H, [] { NS::main(); });
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 5

#if REF_PASS == 6 // fs_svgf_variance.sc: ref_svgf_variance

namespace shader_svgf_variance
{
#include "fs_svgf_variance.sc"
} // namespace shader_svgf_variance

extern "C"
{

int ref_svgf_variance(const RestirParams* P, const uint16_t* color, const uint16_t* moments, const float* receiver,
	const float* normal, uint16_t* output)
{
	namespace NS = shader_svgf_variance;
	const uint32_t w = P->gi_width, h = P->gi_height;
	NS::s_giColor = image(color, w, h, kFormatRGBA16F);
	NS::s_giMoments = image(moments, w, h, kFormatRGBA16F);
	NS::s_giReceiver = image(receiver, w, h, kFormatRGBA32F);
	NS::s_giNormal = image(normal, w, h, kFormatRGBA32F);
	NS::u_screenInfo = vec4(float(w), float(h), 1.0f / float(w), 1.0f / float(h));
	NS::u_sceneInfo = vec4(P->scene_scale, P->boiling_filter, P->jacobian_clamp, P->outlier_clamp);
	dispatchFragments(w, h, [] { NS::main(); }, image(nullptr, w, h, kFormatRGBA16F, output));
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 6

#if REF_PASS == 7 // fs_svgf_atrous.sc: ref_svgf_atrous

namespace shader_svgf_atrous
{
#include "fs_svgf_atrous.sc"
} // namespace shader_svgf_atrous

extern "C"
{

int ref_svgf_atrous(const RestirParams* P, int step, const uint16_t* input, const float* receiver, const float* normal,
	uint16_t* output)
{
	namespace NS = shader_svgf_atrous;
	const uint32_t w = P->gi_width, h = P->gi_height;
	NS::s_filterInput = image(input, w, h, kFormatRGBA16F);
	NS::s_giReceiver = image(receiver, w, h, kFormatRGBA32F);
	NS::s_giNormal = image(normal, w, h, kFormatRGBA32F);
	NS::u_screenInfo = vec4(float(w), float(h), 1.0f / float(w), 1.0f / float(h));
	NS::u_sceneInfo = vec4(P->scene_scale, P->boiling_filter, P->jacobian_clamp, P->outlier_clamp);
	NS::u_atrousInfo = vec4(float(step), 0.0f, 0.0f, 0.0f);
	dispatchFragments(w, h, [] { NS::main(); }, image(nullptr, w, h, kFormatRGBA16F, output));
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 7

#if REF_PASS == 8 // fs_composite.sc: ref_composite_specular

namespace shader_composite
{
#include "fs_composite.sc"
} // namespace shader_composite

namespace
{
DEFINE_BIND_SHADOW(shader_composite)
} // namespace

extern "C"
{

/* fs_composite.sc; specular_target may be null (u_compositeSpecular.x = 0). */
int ref_composite_specular(const RestirParams* P, const RestirGBuffer* gb, const float* shadow_atlas,
	const uint16_t* gi, const uint16_t* di_diffuse, const uint16_t* di_specular, const uint16_t* specular_target,
	uint16_t* hdr)
{
	namespace NS = shader_composite;
	const uint32_t W = P->width, H = P->height, w = P->gi_width, h = P->gi_height;
	g_originBottomLeft = P->origin_bottom_left > 0.5f;
	NS::s_albedo = image(gb->albedo, W, H, kFormatBGRA8);
	NS::s_normal = image(gb->normal, W, H, kFormatBGRA8);
	NS::s_depth = image(gb->depth, W, H, kFormatR32F);
	NS::s_gi = image(gi, w, h, kFormatRGBA16F);
	NS::s_emissive = image(gb->emissive, W, H, kFormatRGBA16F);
	NS::s_shadingNormal = image(gb->shading_normal, W, H, kFormatBGRA8);
	NS::s_diDiffuse = image(di_diffuse, W, H, kFormatRGBA16F);
	NS::s_diSpecular = image(di_specular, W, H, kFormatRGBA16F);
	NS::s_specular = image(specular_target, w, h, kFormatRGBA16F);
	bindShadowshader_composite(P, shadow_atlas);
	NS::u_sceneInvViewProj = matrix(P->inv_view_proj);
	NS::u_lightPosition = vec4At(P->light_position);
	NS::u_lightColor = vec4At(P->light_color);
	NS::u_cameraPosition = vec4At(P->camera_position);
	NS::u_screenInfo = vec4(float(w), float(h), 1.0f / float(w), 1.0f / float(h));
	NS::u_sceneInfo = vec4(P->scene_scale, P->boiling_filter, P->jacobian_clamp, P->outlier_clamp);
	NS::u_compositeOptions = vec4At(P->composite_options);
	NS::u_compositeSpecular = vec4(specular_target != nullptr ? P->composite_specular : 0.0f, 0.0f, 0.0f, 0.0f);
	NS::u_skyZenith = vec4At(P->sky_zenith);
	NS::u_skyHorizon = vec4At(P->sky_horizon);
	NS::u_skyGround = vec4At(P->sky_ground);
	dispatchFragments(W, H, [] { NS::main(); }, image(nullptr, W, H, kFormatRGBA16F, hdr));
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 8

#if REF_PASS == 9 // fs_specular.sc: ref_gi_specular

namespace shader_specular
{
#include "fs_specular.sc"
} // namespace shader_specular

namespace
{
DEFINE_BIND_SHADOW(shader_specular)
} // namespace

extern "C"
{

int ref_gi_specular(const RestirParams* P, const RestirScene* scene, const RestirGBuffer* gb,
	const RestirGiHistory* history, const float* shadow_atlas, const uint16_t* surface_light, const uint16_t* previous_hdr,
	const uint16_t* specular_history, uint16_t* specular)
{
	namespace NS = shader_specular;
	BIND_RESTIR_SH(shader_specular, P, scene, gb, history, shadow_atlas, surface_light, static_cast<const uint32_t*>(nullptr),
		P->camera_position);
	const uint32_t W = P->width, H = P->height, w = P->gi_width, h = P->gi_height;
	NS::s_previousHdr = image(previous_hdr, W, H, kFormatRGBA16F);
	NS::s_specularHistory = image(specular_history, w, h, kFormatRGBA16F);
	NS::u_cameraPosition = vec4At(P->camera_position);
	dispatchFragments(w, h, [] { NS::main(); }, image(nullptr, w, h, kFormatRGBA16F, specular));
	return RESTIR_OK;
}

} // extern "C"

#endif // REF_PASS == 9
