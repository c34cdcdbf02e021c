"""ctypes mirrors of the C structs in include/restir_gpu.h and include/restir_host.h.

Field order and types must match the headers exactly; tests/test_abi.py checks
the sizes against the compiled library.
"""
from __future__ import annotations

import ctypes as C

f4 = C.c_float * 4
m16 = C.c_float * 16
f3 = C.c_float * 3


class RestirParams(C.Structure):
    _fields_ = [
        ("view_proj", m16), ("inv_view_proj", m16), ("prev_view_proj", m16),
        ("shadow_view_proj", m16 * 6), ("shadow_inv_view_proj", m16 * 6),
        ("light_position", f4), ("light_color", f4), ("camera_position", f4), ("prev_camera_position", f4),
        ("frame_index", C.c_float), ("history_valid", C.c_float), ("origin_bottom_left", C.c_float),
        ("multiple_bounces", C.c_float),
        ("width", C.c_uint32), ("height", C.c_uint32), ("gi_width", C.c_uint32), ("gi_height", C.c_uint32),
        ("scene_scale", C.c_float), ("boiling_filter", C.c_float), ("jacobian_clamp", C.c_float),
        ("outlier_clamp", C.c_float),
        ("surface_light_scale", C.c_float), ("emission_scale", C.c_float),
        ("initial_candidates", C.c_int32), ("temporal_taps", C.c_int32), ("spatial_taps", C.c_int32),
        ("trace_steps", C.c_int32),
        ("grid_min_cell", C.c_float), ("grid_pixel_size", C.c_float), ("grid_cell_pixels", C.c_float),
        ("world_space_reuse", C.c_float), ("grid_table_size", C.c_uint32), ("grid_cell_capacity", C.c_uint32),
        ("grid_mode", C.c_uint32),
        ("ray_mode", C.c_int32),
        ("di_light_count", C.c_int32), ("di_candidates", C.c_int32), ("di_spatial_taps", C.c_int32),
        ("di_history_valid", C.c_float),
        ("shadow_far", C.c_float), ("shadow_tan_half_fov", C.c_float), ("shadow_inv_face_size", C.c_float),
        ("shadows_enabled", C.c_float), ("shadow_face_size", C.c_uint32),
        ("sky_zenith", f4), ("sky_horizon", f4), ("sky_ground", f4),
        ("composite_options", f4),
        ("radiance_cache", C.c_float), ("cache_training_samples", C.c_uint32), ("wave_visibility", C.c_float),
        ("composite_specular", C.c_float),
    ]


class RestirScene(C.Structure):
    _fields_ = [
        ("bvh", C.c_void_p), ("node_count", C.c_uint32), ("triangle_offset", C.c_uint32),
        ("triangle_count", C.c_uint32), ("lights", C.c_void_p), ("light_count", C.c_uint32),
        ("triangle_normals", C.c_void_p), ("materials", C.c_void_p), ("material_count", C.c_uint32),
    ]


class RestirGBuffer(C.Structure):
    _fields_ = [("albedo", C.c_void_p), ("normal", C.c_void_p), ("emissive", C.c_void_p),
                ("shading_normal", C.c_void_p), ("depth", C.c_void_p)]


class RestirGiReservoirs(C.Structure):
    _fields_ = [("sample", C.c_void_p), ("receiver", C.c_void_p), ("normal", C.c_void_p)]


class RestirGiHistory(C.Structure):
    _fields_ = [("sample", C.c_void_p), ("receiver", C.c_void_p), ("normal", C.c_void_p),
                ("color", C.c_void_p), ("moments", C.c_void_p)]


class RestirDiReservoirs(C.Structure):
    _fields_ = [("sample", C.c_void_p), ("receiver", C.c_void_p), ("normal", C.c_void_p)]


class RestirMeshDesc(C.Structure):
    _fields_ = [
        ("triangle_count", C.c_uint32), ("positions", C.c_void_p), ("normals", C.c_void_p),
        ("triangle_material", C.c_void_p), ("material_count", C.c_uint32), ("materials", C.c_void_p),
        ("bounds_min", f3), ("bounds_max", f3), ("center", f3), ("radius", C.c_float),
        ("light_position", f3), ("camera_eye", f3), ("camera_yaw", C.c_float), ("camera_pitch", C.c_float),
        ("sky", C.c_int), ("two_sided", C.c_void_p),
    ]


class RestirBvhDesc(C.Structure):
    _fields_ = [
        ("data", C.c_void_p), ("float_count", C.c_uint64), ("node_count", C.c_uint32),
        ("triangle_offset", C.c_uint32), ("triangle_count", C.c_uint32), ("depth", C.c_uint32),
        ("triangle_normals", C.c_void_p), ("order", C.c_void_p), ("emitter_count", C.c_uint32),
        ("emitters", C.c_void_p), ("build_ms", C.c_double),
    ]


class RestirLightsDesc(C.Structure):
    _fields_ = [("data", C.c_void_p), ("count", C.c_uint32), ("triangles", C.c_uint32)]


class RestirSettings(C.Structure):
    _fields_ = [
        ("light_position", f3), ("light_color", f3), ("light_intensity", C.c_float),
        ("extra_lights", C.c_int), ("extra_intensity", C.c_float), ("extra_seed", C.c_int),
        ("sky_enabled", C.c_int), ("sky_zenith", f3), ("sky_horizon", f3), ("sky_ground", f3),
        ("sky_intensity", C.c_float),
        ("multiple_bounces", C.c_int), ("shadows", C.c_int), ("denoiser", C.c_int),
        ("world_space_reuse", C.c_int), ("emissive_lighting", C.c_int), ("ray_mode", C.c_int),
        ("direct_lighting", C.c_int), ("clamp_jacobian", C.c_int), ("clamp_outliers", C.c_int),
        ("boiling_filter", C.c_int),
        ("gi_divisor", C.c_int), ("shadow_face_size", C.c_int), ("atrous_iterations", C.c_int),
        ("initial_candidates", C.c_int), ("temporal_taps", C.c_int), ("spatial_taps", C.c_int),
        ("trace_steps", C.c_int), ("di_candidates", C.c_int), ("di_spatial_taps", C.c_int),
        ("grid_table_size", C.c_uint32), ("grid_cell_capacity", C.c_uint32), ("grid_mode", C.c_uint32),
        ("wavefront", C.c_uint32), ("radiance_cache", C.c_uint32), ("cache_training_samples", C.c_uint32),
        ("wave_visibility", C.c_uint32),
        ("taa", C.c_int), ("auto_exposure", C.c_int), ("tonemapper", C.c_int), ("exposure_ev", C.c_float),
        ("adaptation_speed", C.c_float), ("display", C.c_int), ("bvh_on_device", C.c_int), ("specular_gi", C.c_int),
        ("cache_only_gi", C.c_int), ("cache_learning_rate", C.c_float),
        ("extra_light_orbit", C.c_float),
    ]


class RestirFrameInput(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("eye", f3), ("yaw", C.c_float),
                ("pitch", C.c_float), ("delta_time", C.c_float)]


class RestirFrameState(C.Structure):
    _fields_ = [
        ("frame_number", C.c_uint32), ("history_valid", C.c_int), ("di_valid", C.c_int),
        ("previous_view_proj", m16), ("previous_eye", f3), ("reference_accumulating", C.c_int),
        ("reference_frames", C.c_uint32), ("previous_unjittered_view_proj", m16), ("taa_valid", C.c_int),
        ("exposure_valid", C.c_int),
    ]


class RestirMetrics(C.Structure):
    _fields_ = [("valid", C.c_int), ("relative_mse", C.c_double), ("bias", C.c_double), ("error", C.c_double * 4),
                ("pass_ms", C.c_float * 13), ("reference_frames", C.c_uint32)]


class RestirFramePlan(C.Structure):
    """Which passes a frame runs, as Renderer::render decides (renderer.cpp:627-1094)."""
    _fields_ = [
        ("di_active", C.c_int), ("denoiser", C.c_int), ("atrous_iterations", C.c_int),
        ("reference_accumulate", C.c_int), ("reference_weight_frames", C.c_uint32),
        ("surface_light_is_di", C.c_int), ("display", C.c_int), ("taa", C.c_int), ("exposure", C.c_int),
        ("specular", C.c_int), ("gi_from_cache", C.c_int),
        ("unjittered_view_proj", m16),
    ]


# --- include/restir_display.h -------------------------------------------------------------------------

TONEMAP_ACES, TONEMAP_AGX, TONEMAP_NEUTRAL, TONEMAP_REINHARD, TONEMAP_CLAMP = range(5)


class RestirDisplayParams(C.Structure):
    _fields_ = [
        ("inv_view_proj", m16), ("previous_view_proj", m16), ("taa_history_valid", C.c_float),
        ("origin_bottom_left", C.c_float), ("exposure_adapt", C.c_float), ("exposure_reset", C.c_float),
        ("exposure_ev", C.c_float), ("auto_exposure", C.c_float), ("tonemapper", C.c_float),
        ("pass_through", C.c_float), ("reference_view", C.c_float), ("taa", C.c_float),
        ("width", C.c_uint32), ("height", C.c_uint32),
    ]


# --- include/restir_cache.h ---------------------------------------------------------------------------

CACHE_LEVELS = 16
CACHE_FEATURES = 2
CACHE_WEIGHTS = 4 * 64 * 64 + 16 * 64
CACHE_PARTIAL_STRIDE = CACHE_WEIGHTS + 64


class RestirCacheConfig(C.Structure):
    _fields_ = [
        ("bounds_min", f3), ("bounds_max", f3), ("table_log2", C.c_uint32), ("n_min", C.c_float),
        ("n_max", C.c_float), ("learning_rate", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
        ("epsilon", C.c_float), ("initial_loss_scale", C.c_float), ("seed", C.c_uint32),
    ]


class RestirCacheLayout(C.Structure):
    _fields_ = [
        ("weights", C.c_uint64), ("weights_bf16", C.c_uint64), ("weight_m", C.c_uint64), ("weight_v", C.c_uint64),
        ("weight_grad", C.c_uint64), ("weight_partials", C.c_uint64), ("table", C.c_uint64),
        ("table_half", C.c_uint64), ("table_m", C.c_uint64), ("table_v", C.c_uint64), ("table_grad", C.c_uint64),
        ("table_grad_fixed", C.c_uint64), ("scalars", C.c_uint64), ("bytes", C.c_uint64), ("entries", C.c_uint32), ("partial_blocks", C.c_uint32),
        ("level_scale", C.c_float * CACHE_LEVELS), ("level_dense", C.c_uint32 * CACHE_LEVELS),
    ]


class RestirCacheScalars(C.Structure):
    _fields_ = [
        ("loss_scale", C.c_float), ("step", C.c_uint32), ("clean_steps", C.c_uint32), ("skipped_steps", C.c_uint32),
        ("loss", C.c_float), ("nonfinite", C.c_uint32), ("samples", C.c_uint32), ("blocks", C.c_uint32),
        ("beta1_power", C.c_float), ("beta2_power", C.c_float), ("pad", C.c_uint32 * 6),
    ]


class RestirBatchTuning(C.Structure):
    _fields_ = [("tracer_threads", C.c_uint32), ("tracer_blocks_per_sm", C.c_uint32), ("ms_per_frame", C.c_float)]
