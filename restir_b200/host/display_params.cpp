// restir_display_params: the display passes' uniforms as src/renderer.cpp
// sets them (auto exposure 993-999, TAA 1022-1034, tone mapping 1101-1115).
#include "../../include/restir_display.h"

#include <cmath>
#include <cstring>

extern "C" int restir_display_params(const float* inv_view_proj, const float* previous_unjittered_view_proj,
	uint32_t width, uint32_t height, int taa, int taa_history_valid, int auto_exposure, int exposure_valid,
	float adaptation_speed, float delta_time, float exposure_ev, int tonemapper, int pass_through,
	int reference_view, RestirDisplayParams* out)
{
	if (inv_view_proj == nullptr || previous_unjittered_view_proj == nullptr || out == nullptr || width == 0 || height == 0
		|| tonemapper < RESTIR_TONEMAP_ACES || tonemapper > RESTIR_TONEMAP_CLAMP || reference_view < 0 || reference_view > 2)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	std::memset(out, 0, sizeof(*out));
	std::memcpy(out->inv_view_proj, inv_view_proj, sizeof(out->inv_view_proj));
	std::memcpy(out->previous_view_proj, previous_unjittered_view_proj, sizeof(out->previous_view_proj));
	// A data view (pass_through) neither runs TAA nor moves the exposure
	// (renderer.cpp:475, 989).
	out->taa = (taa != 0 && pass_through == 0) ? 1.0f : 0.0f;
	out->taa_history_valid = taa_history_valid ? 1.0f : 0.0f;
	out->origin_bottom_left = 0.0f;
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
