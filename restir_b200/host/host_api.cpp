// C ABI of include/restir_host.h over the host scene code.
#include "../../include/restir_gpu.h"
#include "bvh_build.h"

#include <cmath>
#include <cstring>
#include <new>

using namespace restir;

namespace
{

struct BvhHandle
{
	BvhResult bvh;
};

struct LightsHandle
{
	LightListResult lights;
};

} // namespace

extern "C" void* restir_mesh_procedural(int kind, uint32_t seed, uint32_t target_triangles)
{
	Mesh* mesh = new (std::nothrow) Mesh();
	if (mesh == nullptr)
	{
		return nullptr;
	}
	switch (kind)
	{
	case RESTIR_SCENE_CORNELL:
		*mesh = makeCornell();
		break;
	case RESTIR_SCENE_COURTYARD:
		*mesh = makeCourtyard(seed, target_triangles);
		break;
	case RESTIR_SCENE_CITY:
		*mesh = makeCity(seed, target_triangles);
		break;
	case RESTIR_SCENE_CITY_LIT:
		*mesh = makeCity(seed, target_triangles, 2048);
		break;
	default:
		delete mesh;
		return nullptr;
	}
	return mesh;
}

extern "C" void* restir_mesh_create(const RestirMeshDesc* desc)
{
	if (desc == nullptr || desc->positions == nullptr || desc->triangle_material == nullptr || desc->materials == nullptr)
	{
		return nullptr;
	}
	Mesh* mesh = new (std::nothrow) Mesh();
	if (mesh == nullptr)
	{
		return nullptr;
	}
	const size_t n = desc->triangle_count;
	mesh->positions.assign(desc->positions, desc->positions + n * 9);
	if (desc->normals != nullptr)
	{
		mesh->normals.assign(desc->normals, desc->normals + n * 3);
	}
	else
	{
		mesh->normals.resize(n * 3);
		for (size_t t = 0; t < n; ++t)
		{
			const float* p = desc->positions + t * 9;
			float a[3] = { p[3] - p[0], p[4] - p[1], p[5] - p[2] };
			float b[3] = { p[6] - p[0], p[7] - p[1], p[8] - p[2] };
			float c[3] = { a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0] };
			float l = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
			for (int k = 0; k < 3; ++k)
			{
				mesh->normals[t * 3 + k] = l > 0.0f ? c[k] / l : 0.0f;
			}
		}
	}
	mesh->material.assign(desc->triangle_material, desc->triangle_material + n);
	if (desc->two_sided != nullptr)
	{
		mesh->twoSided.assign(desc->two_sided, desc->two_sided + n);
	}
	else
	{
		mesh->twoSided.assign(n, 0);
	}
	for (uint32_t m = 0; m < desc->material_count; ++m)
	{
		Material q;
		const float* d = desc->materials + m * 8;
		q.base[0] = d[0];
		q.base[1] = d[1];
		q.base[2] = d[2];
		q.roughness = d[3];
		q.emission[0] = d[4];
		q.emission[1] = d[5];
		q.emission[2] = d[6];
		q.metallic = d[7];
		mesh->materials.push_back(q);
	}
	mesh->finalize();
	std::memcpy(mesh->lightPosition, desc->light_position, sizeof(mesh->lightPosition));
	std::memcpy(mesh->cameraEye, desc->camera_eye, sizeof(mesh->cameraEye));
	mesh->cameraYaw = desc->camera_yaw;
	mesh->cameraPitch = desc->camera_pitch;
	mesh->sky = desc->sky != 0;
	return mesh;
}

extern "C" int restir_mesh_describe(void* handle, RestirMeshDesc* out)
{
	const Mesh* mesh = static_cast<const Mesh*>(handle);
	if (mesh == nullptr || out == nullptr)
	{
		return -1;
	}
	out->triangle_count = mesh->triangleCount();
	out->positions = mesh->positions.data();
	out->normals = mesh->normals.data();
	out->triangle_material = mesh->material.data();
	out->material_count = uint32_t(mesh->materials.size());
	out->materials = mesh->materialData.data();
	std::memcpy(out->bounds_min, mesh->boundsMin, sizeof(out->bounds_min));
	std::memcpy(out->bounds_max, mesh->boundsMax, sizeof(out->bounds_max));
	std::memcpy(out->center, mesh->center, sizeof(out->center));
	out->radius = mesh->radius;
	std::memcpy(out->light_position, mesh->lightPosition, sizeof(out->light_position));
	std::memcpy(out->camera_eye, mesh->cameraEye, sizeof(out->camera_eye));
	out->camera_yaw = mesh->cameraYaw;
	out->camera_pitch = mesh->cameraPitch;
	out->sky = mesh->sky ? 1 : 0;
	out->two_sided = mesh->twoSided.empty() ? nullptr : mesh->twoSided.data();
	return 0;
}

extern "C" void restir_mesh_destroy(void* mesh)
{
	delete static_cast<Mesh*>(mesh);
}

extern "C" void* restir_bvh_build(const RestirMeshDesc* desc, int threads)
{
	if (desc == nullptr)
	{
		return nullptr;
	}
	void* meshHandle = restir_mesh_create(desc);
	if (meshHandle == nullptr)
	{
		return nullptr;
	}
	BvhHandle* handle = new (std::nothrow) BvhHandle();
	if (handle != nullptr)
	{
		handle->bvh = buildBvh(*static_cast<Mesh*>(meshHandle), threads);
		for (const Emitter& e : handle->bvh.emitters)
		{
			handle->bvh.emitterFloats.push_back(float(e.triangle));
			handle->bvh.emitterFloats.insert(handle->bvh.emitterFloats.end(), e.vertices, e.vertices + 9);
			handle->bvh.emitterFloats.insert(handle->bvh.emitterFloats.end(), e.emission, e.emission + 3);
		}
	}
	restir_mesh_destroy(meshHandle);
	return handle;
}

extern "C" void* restir_bvh_build_gpu(const RestirMeshDesc* desc, void* stream)
{
	if (desc == nullptr)
	{
		return nullptr;
	}
	void* meshHandle = restir_mesh_create(desc);
	if (meshHandle == nullptr)
	{
		return nullptr;
	}
	BvhHandle* handle = new (std::nothrow) BvhHandle();
	if (handle != nullptr && buildBvhGpu(*static_cast<Mesh*>(meshHandle), stream, handle->bvh) != RESTIR_OK)
	{
		delete handle;
		handle = nullptr;
	}
	if (handle != nullptr)
	{
		for (const Emitter& e : handle->bvh.emitters)
		{
			handle->bvh.emitterFloats.push_back(float(e.triangle));
			handle->bvh.emitterFloats.insert(handle->bvh.emitterFloats.end(), e.vertices, e.vertices + 9);
			handle->bvh.emitterFloats.insert(handle->bvh.emitterFloats.end(), e.emission, e.emission + 3);
		}
	}
	restir_mesh_destroy(meshHandle);
	return handle;
}

extern "C" int restir_bvh_describe(void* h, RestirBvhDesc* out)
{
	const BvhHandle* handle = static_cast<const BvhHandle*>(h);
	if (handle == nullptr || out == nullptr)
	{
		return -1;
	}
	const BvhResult& b = handle->bvh;
	out->data = b.data.data();
	out->float_count = b.data.size();
	out->node_count = b.nodeCount;
	out->triangle_offset = b.triangleOffset;
	out->triangle_count = b.triangleCount;
	out->depth = b.depth;
	out->triangle_normals = b.triangleNormals.data();
	out->order = b.order.data();
	out->emitter_count = uint32_t(b.emitters.size());
	out->emitters = b.emitterFloats.data();
	out->build_ms = b.buildMs;
	return 0;
}

extern "C" void restir_bvh_destroy(void* h)
{
	delete static_cast<BvhHandle*>(h);
}

extern "C" void* restir_lights_build(void* bvh, int include_emitters, int extra_count, float extra_intensity,
	uint32_t extra_seed, const float* bounds_min, const float* bounds_max, float intensity_scale)
{
	const BvhHandle* handle = static_cast<const BvhHandle*>(bvh);
	static const std::vector<Emitter> none;
	LightsHandle* lights = new (std::nothrow) LightsHandle();
	if (lights != nullptr)
	{
		lights->lights = buildLightList(handle != nullptr && include_emitters ? handle->bvh.emitters : none,
			extra_count, extra_intensity, extra_seed, bounds_min, bounds_max, intensity_scale);
	}
	return lights;
}

extern "C" int restir_lights_describe(void* h, RestirLightsDesc* out)
{
	const LightsHandle* handle = static_cast<const LightsHandle*>(h);
	if (handle == nullptr || out == nullptr)
	{
		return -1;
	}
	out->data = handle->lights.data.data();
	out->count = handle->lights.count;
	out->triangles = handle->lights.triangles;
	return 0;
}

extern "C" void restir_lights_destroy(void* h)
{
	delete static_cast<LightsHandle*>(h);
}
