/*
 * ORACLE (test infrastructure): the host side of a frame, restated, so that
 * the CPU arm of the benchmark (and any test) can run frames without the
 * product's library:
 *
 *   oracle_settings_default   settings.h:183-227 (the renderer's defaults)
 *   oracle_frame_params       renderer.cpp:435-731: the uniforms of one
 *                             frame (reference-mode overrides 437-451, Halton
 *                             jitter 472-488, matrices 490-495, scene, light,
 *                             grid, DI and shadow-face uniforms 496-731)
 *   oracle_frame_advance      renderer.cpp:1119-1124 (the state carried on)
 *   oracle_display_params     renderer.cpp:987-1045 (TAA, exposure, tone map)
 *   oracle_mesh_*             the seeded procedural workload (the benchmark's
 *                             input scenes), built by the same generator
 *                             source as the product (restir_b200/host/
 *                             scene.cpp is compiled into this library): it
 *                             defines the input, it is not part of the path
 *
 * The camera and shadow-face matrices are bx's right-handed look-at and
 * perspective (camera.cpp:107-124, renderer.cpp:531-563) with NDC depth in
 * [0, 1], evaluated in double precision and rounded once to float, and a
 * double-precision Gauss-Jordan inverse: the conventions the product fixes
 * for the same uniforms, so the two must agree bit for bit.
 */
#include "oracle.h"

#include "../include/restir_cache.h"
#include "../include/restir_display.h"
#include "../include/restir_frame.h"
#include "../restir_b200/host/mesh.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

namespace
{

// renderer.cpp:51-85 and settings.h:28-34
constexpr float kReferenceSceneRadius = 1.75f;
constexpr int kShadowFaceBorder = 4;
constexpr float kGridMinCellSize = 0.02f;
constexpr float kGridCellPixels = 6.0f;
constexpr uint32_t kReferenceJitterCount = 1024u;
constexpr uint32_t kTaaJitterCount = 8u;
constexpr float kJacobianClamp = 10.0f;
constexpr float kOutlierClamp = 8.0f;
constexpr float kBoilingFilter = 4.0f;
constexpr float kCameraFovYDegrees = 48.0f;
constexpr double kPi = 3.14159265358979323846;

// renderer.cpp:66-79: the radical inverse of index in base.
float radicalInverse(uint32_t index, uint32_t base)
{
	float value = 0.0f;
	float scale = 1.0f;
	while (index > 0u)
	{
		scale /= float(base);
		value += scale * float(index % base);
		index /= base;
	}
	return value;
}

void store(float* out, const double* m)
{
	for (int i = 0; i < 16; ++i)
	{
		out[i] = float(m[i]);
	}
}

// Row-major, clip = M * v; view space looks down -z.
void lookAt(const float* eye, const float* at, const float* up, float* out)
{
	double forward[3], side[3], upward[3];
	for (int k = 0; k < 3; ++k)
	{
		forward[k] = double(at[k]) - eye[k];
	}
	double length = std::sqrt(forward[0] * forward[0] + forward[1] * forward[1] + forward[2] * forward[2]);
	for (double& v : forward)
	{
		v /= length;
	}
	side[0] = forward[1] * up[2] - forward[2] * up[1];
	side[1] = forward[2] * up[0] - forward[0] * up[2];
	side[2] = forward[0] * up[1] - forward[1] * up[0];
	length = std::sqrt(side[0] * side[0] + side[1] * side[1] + side[2] * side[2]);
	for (double& v : side)
	{
		v /= length;
	}
	upward[0] = side[1] * forward[2] - side[2] * forward[1];
	upward[1] = side[2] * forward[0] - side[0] * forward[2];
	upward[2] = side[0] * forward[1] - side[1] * forward[0];
	auto along = [&](const double* axis) { return axis[0] * eye[0] + axis[1] * eye[1] + axis[2] * eye[2]; };
	const double m[16] = {
		side[0], side[1], side[2], -along(side),
		upward[0], upward[1], upward[2], -along(upward),
		-forward[0], -forward[1], -forward[2], along(forward),
		0.0, 0.0, 0.0, 1.0,
	};
	store(out, m);
}

void perspective(float fovY, float aspect, float nearPlane, float farPlane, float* out)
{
	const double yScale = 1.0 / std::tan(0.5 * double(fovY));
	const double xScale = yScale / double(aspect);
	const double depthRange = double(nearPlane) - double(farPlane);
	const double m[16] = {
		xScale, 0.0, 0.0, 0.0,
		0.0, yScale, 0.0, 0.0,
		0.0, 0.0, double(farPlane) / depthRange, double(nearPlane) * double(farPlane) / depthRange,
		0.0, 0.0, -1.0, 0.0,
	};
	store(out, m);
}

// out = a * b, each entry a double-precision dot product rounded once.
void product(const float* a, const float* b, float* out)
{
	double m[16];
	for (int row = 0; row < 4; ++row)
	{
		for (int column = 0; column < 4; ++column)
		{
			double sum = 0.0;
			for (int k = 0; k < 4; ++k)
			{
				sum += double(a[row * 4 + k]) * double(b[k * 4 + column]);
			}
			m[row * 4 + column] = sum;
		}
	}
	store(out, m);
}

// Gauss-Jordan with partial pivoting on [M | I], in double precision.
bool inverse(const float* in, float* out)
{
	double a[4][8];
	for (int row = 0; row < 4; ++row)
	{
		for (int column = 0; column < 4; ++column)
		{
			a[row][column] = in[row * 4 + column];
			a[row][column + 4] = row == column ? 1.0 : 0.0;
		}
	}
	for (int column = 0; column < 4; ++column)
	{
		int pivot = column;
		for (int row = column + 1; row < 4; ++row)
		{
			if (std::fabs(a[row][column]) > std::fabs(a[pivot][column]))
			{
				pivot = row;
			}
		}
		if (a[pivot][column] == 0.0)
		{
			return false;
		}
		if (pivot != column)
		{
			for (int k = 0; k < 8; ++k)
			{
				std::swap(a[column][k], a[pivot][k]);
			}
		}
		const double scale = 1.0 / a[column][column];
		for (int k = 0; k < 8; ++k)
		{
			a[column][k] *= scale;
		}
		for (int row = 0; row < 4; ++row)
		{
			if (row == column || a[row][column] == 0.0)
			{
				continue;
			}
			const double factor = a[row][column];
			for (int k = 0; k < 8; ++k)
			{
				a[row][k] -= factor * a[column][k];
			}
		}
	}
	for (int row = 0; row < 4; ++row)
	{
		for (int column = 0; column < 4; ++column)
		{
			out[row * 4 + column] = float(a[row][column + 4]);
		}
	}
	return true;
}

// FlyCamera::matrices (camera.cpp:107-124): yaw and pitch give the forward
// direction; near 0.05 radii, far past the scene seen from the eye.
void cameraMatrices(const float* eye, float yaw, float pitch, float aspect, const float* center, float radius,
	float* view, float* projection)
{
	const float cp = std::cos(pitch);
	const float forward[3] = { -cp * std::sin(yaw), -std::sin(pitch), -cp * std::cos(yaw) };
	const float at[3] = { eye[0] + forward[0], eye[1] + forward[1], eye[2] + forward[2] };
	const float up[3] = { 0.0f, 1.0f, 0.0f };
	lookAt(eye, at, up, view);
	const float d[3] = { eye[0] - center[0], eye[1] - center[1], eye[2] - center[2] };
	const float farPlane = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + 2.0f * radius;
	perspective(kCameraFovYDegrees * 3.14159265358979f / 180.0f, aspect, 0.05f * radius,
		std::max(farPlane, 2.5f * radius), projection);
}

} // namespace

extern "C"
{

void oracle_settings_default(RestirSettings* s)
{
	std::memset(s, 0, sizeof(*s));
	for (int k = 0; k < 3; ++k)
	{
		s->light_color[k] = 1.0f;
	}
	s->light_intensity = 1.0f;
	s->extra_intensity = 0.3f;
	s->extra_seed = 1;
	s->sky_enabled = 1;
	const float zenith[3] = { 0.30f, 0.50f, 0.95f }, horizon[3] = { 0.85f, 0.88f, 0.92f },
		ground[3] = { 0.32f, 0.29f, 0.26f };
	for (int k = 0; k < 3; ++k)
	{
		s->sky_zenith[k] = zenith[k];
		s->sky_horizon[k] = horizon[k];
		s->sky_ground[k] = ground[k];
	}
	s->sky_intensity = 1.0f;
	s->multiple_bounces = 1;
	s->shadows = 1;
	s->denoiser = 1;
	s->world_space_reuse = 1;
	s->emissive_lighting = 1;
	s->ray_mode = RESTIR_RAY_MODE_HYBRID;
	s->direct_lighting = 0;
	s->clamp_jacobian = 1;
	s->clamp_outliers = 1;
	s->boiling_filter = 1;
	s->gi_divisor = 2;
	s->shadow_face_size = 512;
	s->atrous_iterations = 5;
	s->initial_candidates = 2;
	s->temporal_taps = 2;
	s->spatial_taps = 4;
	s->trace_steps = 32;
	s->di_candidates = 8;
	s->di_spatial_taps = 3;
	s->grid_table_size = 65536u;
	s->grid_cell_capacity = 32u;
	s->grid_mode = RESTIR_GRID_ATOMIC;
	s->wavefront = 1u;
	s->cache_training_samples = 65536u;
	s->taa = 1;
	s->tonemapper = RESTIR_TONEMAP_AGX;
	s->adaptation_speed = 1.5f;
	s->display = 1;
	s->bvh_on_device = 1;
	s->specular_gi = 1;
}

int oracle_frame_params(const RestirSettings* requested, const RestirMeshDesc* scene, uint32_t light_count,
	const RestirBvhDesc* bvh, const RestirFrameInput* input, const RestirFrameState* state, RestirParams* p,
	RestirFramePlan* plan)
{
	if (requested == nullptr || scene == nullptr || input == nullptr || state == nullptr || p == nullptr
		|| input->width == 0u || input->height == 0u || requested->gi_divisor <= 0
		|| requested->shadow_face_size <= 2 * kShadowFaceBorder)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const bool reference = state->reference_accumulating != 0;
	RestirSettings s = *requested;
	bool diHistory = state->di_valid != 0;
	if (reference)
	{
		// Every biased shortcut off (renderer.cpp:437-451); the jitter stays.
		s.temporal_taps = 0;
		s.spatial_taps = 0;
		s.denoiser = 0;
		s.clamp_jacobian = 0;
		s.clamp_outliers = 0;
		s.boiling_filter = 0;
		s.di_spatial_taps = 0;
		diHistory = false;
	}
	std::memset(p, 0, sizeof(*p));
	const uint32_t width = input->width, height = input->height;

	float view[16], projection[16], unjittered[16];
	cameraMatrices(input->eye, input->yaw, input->pitch, float(width) / float(height), scene->center, scene->radius,
		view, projection);
	product(projection, view, unjittered);
	const bool taa = s.taa != 0 && s.display != 0 && !reference;
	if (taa || reference)
	{
		// clip.xy += jitter * clip.w (renderer.cpp:476-488).
		const uint32_t index = state->frame_number % (reference ? kReferenceJitterCount : kTaaJitterCount) + 1u;
		const float jx = (radicalInverse(index, 2u) - 0.5f) * 2.0f / float(width);
		const float jy = (radicalInverse(index, 3u) - 0.5f) * 2.0f / float(height);
		for (int column = 0; column < 4; ++column)
		{
			projection[column] += jx * projection[12 + column];
			projection[4 + column] += jy * projection[12 + column];
		}
	}
	product(projection, view, p->view_proj);
	if (!inverse(p->view_proj, p->inv_view_proj))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	std::memcpy(p->prev_view_proj, state->previous_view_proj, sizeof(p->prev_view_proj));

	const float sceneScale = scene->radius / kReferenceSceneRadius;
	const float lightScale = s.light_intensity * sceneScale * sceneScale;
	for (int k = 0; k < 3; ++k)
	{
		p->light_position[k] = s.light_position[k];
		p->light_color[k] = s.light_color[k] * lightScale;
		p->camera_position[k] = input->eye[k];
		p->prev_camera_position[k] = state->previous_eye[k];
	}
	p->light_position[3] = p->light_color[3] = p->camera_position[3] = p->prev_camera_position[3] = 1.0f;

	p->frame_index = float(state->frame_number & 0xffffffu);
	p->history_valid = state->history_valid ? 1.0f : 0.0f;
	p->origin_bottom_left = 0.0f;
	p->multiple_bounces = s.multiple_bounces ? 1.0f : 0.0f;
	p->width = width;
	p->height = height;
	p->gi_width = std::max(1u, width / uint32_t(s.gi_divisor));
	p->gi_height = std::max(1u, height / uint32_t(s.gi_divisor));
	p->scene_scale = sceneScale;
	p->boiling_filter = s.boiling_filter ? kBoilingFilter : 0.0f;
	p->jacobian_clamp = s.clamp_jacobian ? kJacobianClamp : 0.0f;
	p->outlier_clamp = s.clamp_outliers ? kOutlierClamp : 0.0f;

	// Lighting and DI (renderer.cpp:624-702).
	const bool restirDi = s.direct_lighting == 0;
	const bool diActive = restirDi && light_count > 0u && bvh != nullptr && bvh->node_count > 0u;
	const bool emitters = s.emissive_lighting != 0;
	p->surface_light_scale = restirDi || emitters ? 1.0f : 0.0f;
	p->emission_scale = !restirDi && emitters ? 1.0f : 0.0f;
	p->di_light_count = int32_t(light_count);
	p->di_candidates = s.di_candidates;
	p->di_spatial_taps = s.di_spatial_taps;
	p->di_history_valid = diHistory ? 1.0f : 0.0f;

	p->initial_candidates = s.initial_candidates;
	p->temporal_taps = s.temporal_taps;
	p->spatial_taps = s.spatial_taps;
	p->trace_steps = s.trace_steps;

	// The hash grid (renderer.cpp:704-720): a GI pixel's world size at unit distance.
	p->grid_min_cell = kGridMinCellSize * sceneScale;
	p->grid_pixel_size = float(2.0 * std::tan(0.5 * double(kCameraFovYDegrees) * kPi / 180.0)) / float(p->gi_height);
	p->grid_cell_pixels = kGridCellPixels;
	p->world_space_reuse = s.world_space_reuse ? 1.0f : 0.0f;
	p->grid_table_size = s.grid_table_size;
	p->grid_cell_capacity = s.grid_cell_capacity;
	p->grid_mode = s.grid_mode;
	p->ray_mode = s.ray_mode;
	p->radiance_cache = s.radiance_cache && s.wavefront && !reference ? 1.0f : 0.0f;
	p->cache_training_samples = std::min<uint32_t>(s.cache_training_samples, RESTIR_CACHE_MAX_BATCH);
	p->wave_visibility = s.wave_visibility ? 1.0f : 0.0f;
	p->composite_specular = s.specular_gi ? 1.0f : 0.0f;

	// Shadow faces (renderer.cpp:527-593): a little wider than 90 degrees, so a
	// border of kShadowFaceBorder texels overlaps the neighbouring faces.
	const uint32_t face = uint32_t(s.shadow_face_size);
	const float tanHalf = float(face) / float(face - 2u * uint32_t(kShadowFaceBorder));
	const float shadowFar = 2.5f * scene->radius;
	p->shadow_far = shadowFar;
	p->shadow_tan_half_fov = tanHalf;
	p->shadow_inv_face_size = 1.0f / float(face);
	p->shadows_enabled = s.shadows ? 1.0f : 0.0f;
	p->shadow_face_size = face;
	float shadowProjection[16];
	perspective(float(2.0 * std::atan(double(tanHalf))), 1.0f, 0.01f * scene->radius, shadowFar, shadowProjection);
	static const float kFaceDirections[6][3] = { { 1, 0, 0 }, { -1, 0, 0 }, { 0, 1, 0 }, { 0, -1, 0 }, { 0, 0, 1 },
		{ 0, 0, -1 } };
	for (int f = 0; f < 6; ++f)
	{
		const bool vertical = f == 2 || f == 3;
		const float up[3] = { 0.0f, vertical ? 0.0f : 1.0f, vertical ? 1.0f : 0.0f };
		const float at[3] = { s.light_position[0] + kFaceDirections[f][0], s.light_position[1] + kFaceDirections[f][1],
			s.light_position[2] + kFaceDirections[f][2] };
		float faceView[16];
		lookAt(s.light_position, at, up, faceView);
		product(shadowProjection, faceView, p->shadow_view_proj[f]);
		inverse(p->shadow_view_proj[f], p->shadow_inv_view_proj[f]);
	}

	for (int k = 0; k < 3; ++k)
	{
		p->sky_zenith[k] = s.sky_zenith[k] * s.sky_intensity;
		p->sky_horizon[k] = s.sky_horizon[k] * s.sky_intensity;
		p->sky_ground[k] = s.sky_ground[k] * s.sky_intensity;
	}
	p->sky_zenith[3] = s.sky_enabled ? 1.0f : 0.0f;
	for (float& option : p->composite_options)
	{
		option = 1.0f;
	}

	if (plan != nullptr)
	{
		std::memset(plan, 0, sizeof(*plan));
		plan->di_active = diActive ? 1 : 0;
		plan->denoiser = s.denoiser ? 1 : 0;
		plan->atrous_iterations = std::min(std::max(s.atrous_iterations, 0), 5);
		plan->reference_accumulate = reference ? 1 : 0;
		plan->reference_weight_frames = state->reference_frames;
		plan->surface_light_is_di = restirDi ? 1 : 0;
		plan->display = s.display ? 1 : 0;
		plan->taa = taa ? 1 : 0;
		plan->exposure = s.display && s.auto_exposure ? 1 : 0;
		plan->specular = s.specular_gi ? 1 : 0;
		plan->gi_from_cache = p->radiance_cache > 0.5f && s.cache_only_gi ? 1 : 0;
		if (plan->gi_from_cache)
		{
			plan->denoiser = 0;
		}
		std::memcpy(plan->unjittered_view_proj, unjittered, sizeof(unjittered));
	}
	return RESTIR_OK;
}

void oracle_frame_advance(const RestirParams* params, const RestirFramePlan* plan, const RestirFrameInput* input,
	RestirFrameState* state)
{
	std::memcpy(state->previous_view_proj, params->view_proj, sizeof(state->previous_view_proj));
	for (int k = 0; k < 3; ++k)
	{
		state->previous_eye[k] = input->eye[k];
	}
	state->history_valid = 1;
	state->frame_number += 1u;
	state->di_valid = plan != nullptr && plan->di_active && !state->reference_accumulating ? 1 : 0;
	if (state->reference_accumulating)
	{
		state->reference_frames += 1u;
	}
	if (plan != nullptr)
	{
		std::memcpy(state->previous_unjittered_view_proj, plan->unjittered_view_proj,
			sizeof(state->previous_unjittered_view_proj));
		state->taa_valid = plan->taa;
		state->exposure_valid = plan->exposure;
	}
}

int oracle_display_params(const float* inv_view_proj, const float* previous_unjittered_view_proj, uint32_t width,
	uint32_t height, int taa, int taa_history_valid, int auto_exposure, int exposure_valid, float adaptation_speed,
	float delta_time, float exposure_ev, int tonemapper, int pass_through, int reference_view, RestirDisplayParams* out)
{
	if (inv_view_proj == nullptr || previous_unjittered_view_proj == nullptr || out == nullptr || width == 0u
		|| height == 0u || tonemapper < RESTIR_TONEMAP_ACES || tonemapper > RESTIR_TONEMAP_CLAMP || reference_view < 0
		|| reference_view > 2)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	std::memset(out, 0, sizeof(*out));
	std::memcpy(out->inv_view_proj, inv_view_proj, sizeof(out->inv_view_proj));
	std::memcpy(out->previous_view_proj, previous_unjittered_view_proj, sizeof(out->previous_view_proj));
	out->taa = taa != 0 && pass_through == 0 ? 1.0f : 0.0f;
	out->taa_history_valid = taa_history_valid ? 1.0f : 0.0f;
	out->origin_bottom_left = 0.0f;
	// The exposure moves toward this frame's value by 1 - e^(-speed dt) (cs_exposure.sc).
	out->exposure_adapt = 1.0f - std::exp(-adaptation_speed * delta_time);
	out->exposure_reset = exposure_valid ? 0.0f : 1.0f;
	out->exposure_ev = exposure_ev;
	out->auto_exposure = auto_exposure ? 1.0f : 0.0f;
	out->tonemapper = float(tonemapper);
	out->pass_through = pass_through ? 1.0f : 0.0f;
	out->reference_view = float(reference_view);
	out->width = width;
	out->height = height;
	return RESTIR_OK;
}

/* The seeded procedural scenes (RESTIR_SCENE_*), from the generator source
 * the product uses: a handle, described by oracle_mesh_describe. */
void* oracle_mesh_procedural(int kind, uint32_t seed, uint32_t target_triangles)
{
	restir::Mesh* mesh = new (std::nothrow) restir::Mesh();
	if (mesh == nullptr)
	{
		return nullptr;
	}
	switch (kind)
	{
	case RESTIR_SCENE_CORNELL:
		*mesh = restir::makeCornell();
		break;
	case RESTIR_SCENE_COURTYARD:
		*mesh = restir::makeCourtyard(seed, target_triangles);
		break;
	case RESTIR_SCENE_CITY:
		*mesh = restir::makeCity(seed, target_triangles);
		break;
	case RESTIR_SCENE_CITY_LIT:
		*mesh = restir::makeCity(seed, target_triangles, 2048);
		break;
	default:
		delete mesh;
		return nullptr;
	}
	return mesh;
}

int oracle_mesh_describe(void* handle, RestirMeshDesc* out)
{
	const restir::Mesh* mesh = static_cast<const restir::Mesh*>(handle);
	if (mesh == nullptr || out == nullptr)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	std::memset(out, 0, sizeof(*out));
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
	return RESTIR_OK;
}

void oracle_mesh_destroy(void* handle)
{
	delete static_cast<restir::Mesh*>(handle);
}

} // extern "C"
