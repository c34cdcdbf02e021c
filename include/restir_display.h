/*
 * restir-b200: the display passes that follow the composite, as CUDA image
 * kernels behind the same C ABI as restir_gpu.h.
 *
 *   restir_exposure  auto exposure (shaders/cs_exposure.sc:30-82,
 *                    dispatched at src/renderer.cpp:987-1010)
 *   restir_taa       temporal anti-aliasing (shaders/fs_taa.sc:111-172,
 *                    submitted at src/renderer.cpp:1012-1046)
 *   restir_tonemap   exposure and tone mapping to the display
 *                    (shaders/fs_tonemap.sc:122-162, shaders/tonemap.sh:17-122,
 *                    submitted at src/renderer.cpp:1096-1117)
 *   restir_display   the three in the reference's order as two launches: the
 *                    exposure reduction, then TAA and tone mapping fused per
 *                    pixel (the TAA target is still written, rounded to half
 *                    as the reference's RGBA16F target holds it, and the tone
 *                    mapping reads that rounded value).
 *
 * Conventions, as for the other passes (restir_numeric.h): row 0 at the top
 * unless origin_bottom_left; a pixel's texture coordinate is
 * ((x + 0.5) / width, (y + 0.5) / height); point-sampled targets clamp to the
 * edge. The TAA history is sampled bilinearly (renderer.cpp creates it
 * without point-sampling flags): taps at floor(uv * size - 0.5) and the next
 * texel, clamped to the edge, weights from the fraction, blended as
 * mix(mix(c00, c10, fx), mix(c01, c11, fx), fy) with mix(a, b, t) =
 * a * (1 - t) + b * t. log2, exp2 and pow are restir_numeric.h's.
 *
 * Formats: hdr, TAA history and TAA output RGBA16F (4 halves per pixel);
 * depth D32F; the display BGRA8 (bytes B, G, R, A; the tone mapping's
 * gamma-encoded colour, alpha 1); the exposure state one uint32 holding the
 * float bits of the adapted log2 luminance (the reference's b_exposure[0]).
 */
#ifndef RESTIR_DISPLAY_H
#define RESTIR_DISPLAY_H

#include "restir_gpu.h"

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Tone mapping operators (src/settings.h:38-46, shaders/tonemap.sh:10-14). */
#define RESTIR_TONEMAP_ACES 0
#define RESTIR_TONEMAP_AGX 1
#define RESTIR_TONEMAP_NEUTRAL 2
#define RESTIR_TONEMAP_REINHARD 3
#define RESTIR_TONEMAP_CLAMP 4

/* The display passes' uniforms, as renderer.cpp sets them. */
typedef struct RestirDisplayParams
{
	float inv_view_proj[16];      /* u_sceneInvViewProj: this frame's, jittered (row-major, clip = M v) */
	float previous_view_proj[16]; /* u_taaPreviousViewProj: last frame's, unjittered */
	float taa_history_valid;      /* u_taaInfo.x */
	float origin_bottom_left;     /* u_taaInfo.y */
	float exposure_adapt;         /* u_exposureAdapt.x: 1 - exp(-adaptationSpeed * deltaTime) */
	float exposure_reset;         /* u_exposureAdapt.y: 1 jumps to this frame's value */
	float exposure_ev;            /* u_tonemap.x */
	float auto_exposure;          /* u_tonemap.y */
	float tonemapper;             /* u_tonemap.z: RESTIR_TONEMAP_* */
	float pass_through;           /* u_tonemap.w: the image is already display colour */
	float reference_view;         /* u_referenceView.x: 0 image, 1 reference, 2 error map */
	float taa;                    /* restir_display only: 1 runs TAA, 0 tone-maps hdr itself */
	uint32_t width;
	uint32_t height;
} RestirDisplayParams;

/* Fills RestirDisplayParams the way renderer.cpp does for one frame: the
 * matrices from the caller, taa_history_valid / exposure_reset from the
 * caller's history flags, exposure_adapt = 1 - exp(-adaptation_speed *
 * delta_time) (renderer.cpp:993-999), the rest from the settings' values. */
int restir_display_params(const float* inv_view_proj, const float* previous_unjittered_view_proj,
	uint32_t width, uint32_t height, int taa, int taa_history_valid, int auto_exposure, int exposure_valid,
	float adaptation_speed, float delta_time, float exposure_ev, int tonemapper, int pass_through,
	int reference_view, RestirDisplayParams* out);

/* Auto exposure (cs_exposure.sc): one block of 16x16 threads samples a 64x64
 * grid over hdr (4x4 points per thread, alpha > 0.5 only), sums
 * clamp(log2(max(luminance, 1e-6)), -12, 12) by a shared-memory tree in the
 * shader's order, and moves exposure[0] towards the mean by exposure_adapt
 * (or sets it, on exposure_reset or when the stored value is not within
 * +-12). An image with no geometry sample leaves exposure[0] unchanged. */
int restir_exposure(const RestirDisplayParams* params, const uint16_t* hdr, uint32_t* exposure, void* stream);

/* TAA (fs_taa.sc): out = the current frame blended into the reprojected,
 * Catmull-Rom filtered, YCoCg-clipped history; out = hdr where the history
 * is invalid or the reprojection leaves the screen. out must not alias hdr
 * or history. */
int restir_taa(const RestirDisplayParams* params, const uint16_t* hdr, const float* depth,
	const uint16_t* history, uint16_t* out, void* stream);

/* Tone mapping (fs_tonemap.sc): display = toGamma(tonemap(hdr * exposure)),
 * the background colour (0.125, 0.141, 0.169) where alpha < 0.5, hdr itself
 * with pass_through; reference_view 1 shows the reference mean instead of
 * hdr, 2 the turbo map of the relative luminance error against it.
 * reference_mean / reference_alpha: restir_reference_accumulate's planes
 * (may be null when reference_view is 0); exposure may be null unless
 * auto_exposure. */
int restir_tonemap(const RestirDisplayParams* params, const uint16_t* hdr, const uint32_t* exposure,
	const double* reference_mean, const uint8_t* reference_alpha, uint8_t* display, void* stream);

/* The display chain of renderer.cpp:987-1117 in two launches: restir_exposure
 * on hdr when auto_exposure (and not pass_through), then, per pixel, TAA into
 * taa_out (when taa) and tone mapping of that value (of hdr without taa) into
 * display. Outputs equal those of the separate calls. taa_out / history /
 * depth may be null without taa. */
int restir_display(const RestirDisplayParams* params, const uint16_t* hdr, const float* depth,
	const uint16_t* history, uint16_t* taa_out, uint32_t* exposure, const double* reference_mean,
	const uint8_t* reference_alpha, uint8_t* display, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RESTIR_DISPLAY_H */
