/*
 * restir-b200: C ABI of the host-side scene preparation.
 *
 * The reference builds its acceleration structure and light list in C++
 * when a scene loads (src/bvh.cpp buildBvh, src/lights.cpp buildLightList,
 * called from Renderer::setScene and Renderer::updateLightList,
 * renderer.cpp:365-419, 1170-1207). These are this library's own
 * implementations, emitting the same buffer layouts (src/bvh.h:7-22,
 * src/lights.h:5-17), plus the seeded procedural scenes the benchmarks use
 * in place of glTF files.
 *
 * Handles own their arrays; pointers returned by the describe calls stay
 * valid until the handle is destroyed. Nothing here touches the GPU.
 */
#ifndef RESTIR_HOST_H
#define RESTIR_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Procedural scenes. */
#define RESTIR_SCENE_CORNELL 0   /* open-front Cornell box, 36 triangles */
#define RESTIR_SCENE_COURTYARD 1 /* seeded boxes and arches, ~target triangles */
#define RESTIR_SCENE_CITY 2      /* seeded boxes, 512-triangle spheres, thin planes */
#define RESTIR_SCENE_CITY_LIT 3  /* the city with 2,048 emissive panels (4,096 emissive triangles)
                                    instead of 128: the stress configuration's scene */

/* A triangle soup with one material per triangle. Materials: 8 floats each,
 * (base colour rgb, roughness), (emission rgb, metallic). */
typedef struct RestirMeshDesc
{
	uint32_t triangle_count;
	const float* positions;          /* 9 floats per triangle */
	const float* normals;            /* 3 floats per triangle: the shading normal */
	const uint32_t* triangle_material;
	uint32_t material_count;
	const float* materials;
	float bounds_min[3];
	float bounds_max[3];
	/* describeScene (scene.cpp:810-834): centre, radius and the point light's
	 * default position; the camera pose the scene is framed from. */
	float center[3];
	float radius;
	float light_position[3];
	float camera_eye[3];
	float camera_yaw;
	float camera_pitch;
	int sky;                         /* whether the sky starts on */
	const uint8_t* two_sided;        /* per triangle, 1 for double-sided materials; may be null */
} RestirMeshDesc;

void* restir_mesh_procedural(int kind, uint32_t seed, uint32_t target_triangles);
/* A mesh from caller arrays (copied). */
void* restir_mesh_create(const RestirMeshDesc* desc);
/* A mesh from a glTF 2.0 file (.gltf with external or data-URI buffers, or
 * .glb), as the reference's loadScene flattens a model (scene.cpp:105-381,
 * 722-808): the default scene's nodes with their transforms, triangle-list
 * primitives, triangles grouped by material in material order, material
 * factors (base colour, metallic, roughness, emission times
 * KHR_materials_emissive_strength, double-sided), the light placed by
 * describeScene (scene.cpp:810-834) and the first view of main.cpp:58-83.
 * Textures, vertex colours and sparse accessors are not read. Null on
 * failure, with a message in error (may be null). */
void* restir_mesh_load_gltf(const char* path, char* error, uint32_t error_capacity);
int restir_mesh_describe(void* mesh, RestirMeshDesc* out);
void restir_mesh_destroy(void* mesh);

/* The BVH: binned SAH with 12 bins, leaves of up to 4 triangles (always
 * split above 16), depth at most 40 (bvh.cpp:58-60, bvh.h:49), emitted in
 * depth-first order with skip links. Also the shading normal of each
 * triangle in BVH order (float4: normal, 1 if two-sided) and the emissive
 * triangles (EmissiveTriangle, bvh.h:28-36: 10 floats each, triangle index
 * as float, 9 vertex floats... see restir_bvh_emitters). */
typedef struct RestirBvhDesc
{
	const float* data;               /* float4s: nodes then triangles */
	uint64_t float_count;
	uint32_t node_count;
	uint32_t triangle_offset;        /* in float4s */
	uint32_t triangle_count;
	uint32_t depth;                  /* deepest leaf, root = 1 */
	const float* triangle_normals;   /* float4 per triangle, BVH order */
	const uint32_t* order;           /* BVH slot -> input triangle */
	uint32_t emitter_count;
	const float* emitters;           /* 13 floats each: BVH index, v0, v1, v2, emission */
	double build_ms;
} RestirBvhDesc;

void* restir_bvh_build(const RestirMeshDesc* mesh, int threads);
/* The same BVH built on the current CUDA device (binned SAH breadth first,
 * std::partition's permutation reproduced in parallel): the buffer, order,
 * normals and emitters equal restir_bvh_build's bit for bit. stream: a
 * cudaStream_t (null: the default stream); waits for it. No counterpart in
 * the reference (its builder runs on the host, bvh.cpp:253). */
void* restir_bvh_build_gpu(const RestirMeshDesc* mesh, void* stream);
int restir_bvh_describe(void* bvh, RestirBvhDesc* out);
void restir_bvh_destroy(void* bvh);

/* The light list: emissive triangles then extra point lights, 16 floats
 * per light, selection in proportion to power (lights.cpp:40-119). */
typedef struct RestirLightsDesc
{
	const float* data;
	uint32_t count;
	uint32_t triangles;
} RestirLightsDesc;

void* restir_lights_build(void* bvh, int include_emitters, int extra_count, float extra_intensity,
	uint32_t extra_seed, const float* bounds_min, const float* bounds_max, float intensity_scale);
int restir_lights_describe(void* lights, RestirLightsDesc* out);
void restir_lights_destroy(void* lights);

/* Camera matrices of the reference's fly camera (camera.cpp:107-124):
 * right-handed look-at with +y up, vertical field of view 48 degrees, near
 * 0.05 radius, far max(distance to centre + 2 radius, 2.5 radius), NDC depth
 * in [0, 1]. Row-major, clip = M * v. */
void restir_camera_matrices(const float* eye, float yaw, float pitch, float aspect, const float* center,
	float radius, float* view, float* projection);

#ifdef __cplusplus
}
#endif

#endif /* RESTIR_HOST_H */
