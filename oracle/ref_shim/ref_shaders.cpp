/*
 * ORACLE (test infrastructure): a C interface over the reference's own
 * shader code (pkonecki/restir, the shaders directory), compiled as C++ by oracle/Makefile
 * into oracle/_ref/libref_shaders.so after oracle/ref_shim/glsl_to_cpp.py
 * has made the shader files C++ (see shader_shim.h). Tests hand the same
 * inputs to these functions and to the oracle restatement (oracle.cpp and its headers) and
 * require equal outputs: that pins the restatement, and through it the CUDA
 * kernels, to the reference's shader source.
 *
 * Each shader file is compiled inside a namespace of its own (the shaders
 * declare their uniforms and resources as globals of the same names).
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
 */
#include "shader_shim.h"

#include "../../include/restir_gpu.h"

#include <mutex>

namespace refsh
{
thread_local uvec3 gl_GlobalInvocationID;
thread_local uvec3 gl_LocalInvocationID;
thread_local uvec3 gl_WorkGroupID;
thread_local uint gl_LocalInvocationIndex;
thread_local vec4 gl_FragCoord;
thread_local vec4 gl_FragColor;
thread_local vec4 gl_FragData[4];
bool g_originBottomLeft = false;

namespace
{
std::recursive_mutex g_atomics;
}

void atomicLock() { g_atomics.lock(); }
void atomicUnlock() { g_atomics.unlock(); }
// Sequential dispatch: every barrier is already met.
void barrier() {}

inline vec4 vec4At(const float* p) { return vec4(p[0], p[1], p[2], p[3]); }

inline mat4 matrix(const float* p)
{
	mat4 m;
	std::memcpy(m.m, p, sizeof(m.m));
	return m;
}
} // namespace refsh

using namespace refsh;

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
