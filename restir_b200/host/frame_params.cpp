// The uniforms of one frame, as Renderer::render derives them
// (src/renderer.cpp:435-731), and the state it carries to the next
// (renderer.cpp:1119-1124).
#include "../../include/restir_cache.h"
#include "../../include/restir_display.h"
#include "../../include/restir_frame.h"
#include "bvh_build.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace
{

// renderer.cpp:51-85, settings.h:28-34
constexpr float kReferenceSceneRadius = 1.75f;
constexpr int kShadowFaceBorder = 4;
constexpr float kGridMinCellSize = 0.02f;
constexpr float kGridCellPixels = 6.0f;
constexpr uint32_t kReferenceJitterCount = 1024;
constexpr uint32_t kTaaJitterCount = 8;
constexpr float kJacobianClamp = 10.0f;
constexpr float kOutlierClamp = 8.0f;
constexpr float kBoilingFilter = 4.0f;
constexpr float kCameraFovY = 48.0f;
constexpr double kPiD = 3.14159265358979323846;

float halton(uint32_t index, uint32_t base)
{
	float result = 0.0f;
	float fraction = 1.0f;
	for (uint32_t value = index; value > 0; value /= base)
	{
		fraction /= float(base);
		result += fraction * float(value % base);
	}
	return result;
}

void copy16(float* out, const float* in)
{
	std::memcpy(out, in, 16 * sizeof(float));
}

} // namespace

extern "C" void restir_settings_default(RestirSettings* s)
{
	std::memset(s, 0, sizeof(*s));
	s->light_color[0] = s->light_color[1] = s->light_color[2] = 1.0f;
	s->light_intensity = 1.0f;
	s->extra_lights = 0;
	s->extra_intensity = 0.3f;
	s->extra_seed = 1;
	s->sky_enabled = 1;
	const float zenith[3] = { 0.30f, 0.50f, 0.95f };
	const float horizon[3] = { 0.85f, 0.88f, 0.92f };
	const float ground[3] = { 0.32f, 0.29f, 0.26f };
	std::memcpy(s->sky_zenith, zenith, sizeof(zenith));
	std::memcpy(s->sky_horizon, horizon, sizeof(horizon));
	std::memcpy(s->sky_ground, ground, sizeof(ground));
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
	s->grid_table_size = 65536;
	s->grid_cell_capacity = 32;
	s->grid_mode = RESTIR_GRID_ATOMIC;
	s->wavefront = 1;
	s->radiance_cache = 0;
	s->cache_training_samples = 65536;
	s->wave_visibility = 0;
	s->taa = 1;
	s->auto_exposure = 0;
	s->tonemapper = RESTIR_TONEMAP_AGX;
	s->exposure_ev = 0.0f;
	s->adaptation_speed = 1.5f;
	s->display = 1;
	s->bvh_on_device = 1;
	s->specular_gi = 1;
}

extern "C" int restir_frame_params(const RestirSettings* requested, const RestirMeshDesc* scene, uint32_t light_count,
	const RestirBvhDesc* bvh, const RestirFrameInput* input, const RestirFrameState* state, RestirParams* p,
	RestirFramePlan* plan)
{
	if (requested == nullptr || scene == nullptr || input == nullptr || state == nullptr || p == nullptr
		|| input->width == 0 || input->height == 0 || requested->gi_divisor <= 0 || requested->shadow_face_size <= 2 * kShadowFaceBorder)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	// While the reference accumulates, every biased shortcut is off
	// (renderer.cpp:437-451).
	RestirSettings s = *requested;
	bool diValid = state->di_valid != 0;
	if (state->reference_accumulating)
	{
		s.temporal_taps = 0;
		s.spatial_taps = 0;
		s.denoiser = 0;
		s.clamp_jacobian = 0;
		s.clamp_outliers = 0;
		s.boiling_filter = 0;
		s.di_spatial_taps = 0;
		diValid = false;
	}
	std::memset(p, 0, sizeof(*p));
	const uint32_t width = input->width, height = input->height;
	const float radius = scene->radius;
	const float center[3] = { scene->center[0], scene->center[1], scene->center[2] };

	float view[16], projection[16];
	restir_camera_matrices(input->eye, input->yaw, input->pitch, float(width) / float(height), center, radius, view, projection);
	float unjittered[16];
	restir::multiply(projection, view, unjittered);
	// TAA integrates a Halton (2, 3) sub-pixel jitter over 8 frames; the
	// reference accumulation over 1024 (renderer.cpp:472-488). The scene passes
	// use the jittered matrices, TAA reprojects with the unjittered ones.
	const bool taa = s.taa != 0 && s.display != 0 && !state->reference_accumulating;
	if (taa || state->reference_accumulating)
	{
		// clip.xy += jitter * clip.w.
		const uint32_t index = (state->frame_number % (state->reference_accumulating ? kReferenceJitterCount : kTaaJitterCount)) + 1;
		const float jitterX = (halton(index, 2) - 0.5f) * 2.0f / float(width);
		const float jitterY = (halton(index, 3) - 0.5f) * 2.0f / float(height);
		for (int c = 0; c < 4; ++c)
		{
			projection[0 * 4 + c] += jitterX * projection[3 * 4 + c];
			projection[1 * 4 + c] += jitterY * projection[3 * 4 + c];
		}
	}
	restir::multiply(projection, view, p->view_proj);
	if (!restir::invert(p->view_proj, p->inv_view_proj))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	copy16(p->prev_view_proj, state->previous_view_proj);

	const float sceneScale = radius / kReferenceSceneRadius;
	const float lightScale = s.light_intensity * sceneScale * sceneScale;
	for (int k = 0; k < 3; ++k)
	{
		p->light_position[k] = s.light_position[k];
		p->light_color[k] = s.light_color[k] * lightScale;
		p->camera_position[k] = input->eye[k];
		p->prev_camera_position[k] = state->previous_eye[k];
	}
	p->light_position[3] = 1.0f;
	p->light_color[3] = 1.0f;
	p->camera_position[3] = 1.0f;
	p->prev_camera_position[3] = 1.0f;

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

	// The light list and DI (renderer.cpp:624-700).
	const bool restirDi = s.direct_lighting == 0;
	const bool bvhPresent = bvh != nullptr && bvh->node_count > 0;
	const bool diActive = restirDi && light_count > 0 && bvhPresent;
	const bool emitters = s.emissive_lighting != 0;
	p->surface_light_scale = restirDi ? 1.0f : (emitters ? 1.0f : 0.0f);
	p->emission_scale = restirDi ? 0.0f : (emitters ? 1.0f : 0.0f);
	p->di_light_count = int32_t(light_count);
	p->di_candidates = s.di_candidates;
	p->di_spatial_taps = s.di_spatial_taps;
	p->di_history_valid = diValid ? 1.0f : 0.0f;

	p->initial_candidates = s.initial_candidates;
	p->temporal_taps = s.temporal_taps;
	p->spatial_taps = s.spatial_taps;
	p->trace_steps = s.trace_steps;

	p->grid_min_cell = kGridMinCellSize * sceneScale;
	p->grid_pixel_size = float(2.0 * std::tan(0.5 * double(kCameraFovY) * kPiD / 180.0)) / float(p->gi_height);
	p->grid_cell_pixels = kGridCellPixels;
	p->world_space_reuse = s.world_space_reuse ? 1.0f : 0.0f;
	p->grid_table_size = s.grid_table_size;
	p->grid_cell_capacity = s.grid_cell_capacity;
	p->grid_mode = s.grid_mode;
	p->ray_mode = s.ray_mode;
	// The radiance cache replaces the history-based bounce; reference
	// accumulation keeps the plain method.
	p->radiance_cache = (s.radiance_cache && s.wavefront && !state->reference_accumulating) ? 1.0f : 0.0f;
	p->cache_training_samples = s.cache_training_samples < RESTIR_CACHE_MAX_BATCH ? s.cache_training_samples
		: RESTIR_CACHE_MAX_BATCH;
	p->wave_visibility = s.wave_visibility ? 1.0f : 0.0f;
	p->composite_specular = s.specular_gi ? 1.0f : 0.0f;

	// The shadow atlas (renderer.cpp:527-593): six faces of a slightly wider
	// field of view than 90 degrees, a border of 4 texels.
	const uint32_t face = uint32_t(s.shadow_face_size);
	const float tanHalf = float(face) / float(face - 2 * kShadowFaceBorder);
	const float shadowFar = 2.5f * radius;
	p->shadow_far = shadowFar;
	p->shadow_tan_half_fov = tanHalf;
	p->shadow_inv_face_size = 1.0f / float(face);
	p->shadows_enabled = s.shadows ? 1.0f : 0.0f;
	p->shadow_face_size = face;
	float shadowProjection[16];
	restir::perspectiveRH(float(2.0 * std::atan(double(tanHalf))), 1.0f, 0.01f * radius, shadowFar, shadowProjection);
	const float directions[6][3] = { { 1, 0, 0 }, { -1, 0, 0 }, { 0, 1, 0 }, { 0, -1, 0 }, { 0, 0, 1 }, { 0, 0, -1 } };
	for (int f = 0; f < 6; ++f)
	{
		const float up[3] = { 0.0f, f == 2 || f == 3 ? 0.0f : 1.0f, f == 2 || f == 3 ? 1.0f : 0.0f };
		const float at[3] = { s.light_position[0] + directions[f][0], s.light_position[1] + directions[f][1],
			s.light_position[2] + directions[f][2] };
		float faceView[16];
		restir::lookAtRH(s.light_position, at, up, faceView);
		restir::multiply(shadowProjection, faceView, p->shadow_view_proj[f]);
		restir::invert(p->shadow_view_proj[f], p->shadow_inv_view_proj[f]);
	}

	for (int k = 0; k < 3; ++k)
	{
		p->sky_zenith[k] = s.sky_zenith[k] * s.sky_intensity;
		p->sky_horizon[k] = s.sky_horizon[k] * s.sky_intensity;
		p->sky_ground[k] = s.sky_ground[k] * s.sky_intensity;
	}
	p->sky_zenith[3] = s.sky_enabled ? 1.0f : 0.0f;
	p->composite_options[0] = 1.0f;
	p->composite_options[1] = 1.0f;
	p->composite_options[2] = 1.0f;
	p->composite_options[3] = 1.0f;

	if (plan != nullptr)
	{
		plan->di_active = diActive ? 1 : 0;
		plan->denoiser = s.denoiser ? 1 : 0;
		plan->atrous_iterations = std::min(std::max(s.atrous_iterations, 0), 5);
		plan->reference_accumulate = state->reference_accumulating ? 1 : 0;
		plan->reference_weight_frames = state->reference_frames;
		plan->surface_light_is_di = restirDi ? 1 : 0;
		plan->display = s.display ? 1 : 0;
		plan->taa = taa ? 1 : 0;
		plan->exposure = s.display && s.auto_exposure ? 1 : 0;
		plan->specular = s.specular_gi ? 1 : 0;
		plan->gi_from_cache = p->radiance_cache > 0.5f && s.cache_only_gi ? 1 : 0;
		if (plan->gi_from_cache)
		{
			plan->denoiser = 0; // the cache's values carry no sampling noise
		}
		copy16(plan->unjittered_view_proj, unjittered);
	}
	return RESTIR_OK;
}

extern "C" void restir_frame_advance(const RestirParams* params, const RestirFramePlan* plan, const RestirFrameInput* input,
	RestirFrameState* state)
{
	copy16(state->previous_view_proj, params->view_proj);
	for (int k = 0; k < 3; ++k)
	{
		state->previous_eye[k] = input->eye[k];
	}
	state->history_valid = 1;
	state->frame_number += 1;
	// DI history is valid after a frame that ran DI; the reference mode
	// clears it again before every frame (renderer.cpp:449, 683-688).
	state->di_valid = plan != nullptr && plan->di_active && !state->reference_accumulating ? 1 : 0;
	if (state->reference_accumulating)
	{
		state->reference_frames += 1;
	}
	// TAA and auto exposure history (renderer.cpp:1004-1045, 1120).
	if (plan != nullptr)
	{
		copy16(state->previous_unjittered_view_proj, plan->unjittered_view_proj);
		state->taa_valid = plan->taa;
		state->exposure_valid = plan->exposure;
	}
}
