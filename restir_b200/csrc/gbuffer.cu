// The two raster passes of the reference, restated as ray casts.
//
// restir_gbuffer_primary replaces the geometry view (renderer.cpp:595-612,
// vs_scene.sc + fs_gbuffer.sc): one primary ray per pixel centre through
// the (jittered) inverse view-projection, nearest triangle whose shading
// normal faces the camera (fs_gbuffer.sc:45-55 discards the others unless
// two-sided), written to the reference's four targets and depth.
//
// restir_shadow_atlas replaces the six shadow views (renderer.cpp:527-593,
// fs_shadow.sc): one ray per atlas texel centre from the light through its
// face's frustum, nearest triangle of either side, distance / far.
//
// Both are closest-hit rays with a full traversal stack, ties to the lower
// triangle index, one thread per pixel in 8x8 tiles (coherent rays share
// node fetches through L1).
#include "bvh.cuh"
#include "screen.cuh"

namespace restir
{
namespace
{

__global__ void __launch_bounds__(64) gbufferKernel(const RestirParams P, BvhView bvh, const float4* __restrict__ normals,
	const float4* __restrict__ materials, RestirGBuffer gb)
{
	const int x = int(blockIdx.x * 8 + threadIdx.x % 8);
	const int y = int(blockIdx.y * 8 + threadIdx.x / 8);
	const int W = int(P.width), H = int(P.height);
	if (x >= W || y >= H)
	{
		return;
	}
	const int i = y * W + x;
	const V2 texel = v2(1.0f / float(W), 1.0f / float(H));
	const V2 uv = pixelUv(x, y, texel);
	const V3 camera = v3(P.camera_position[0], P.camera_position[1], P.camera_position[2]);
	const float ndcX = uv.x * 2.0f - 1.0f;
	const float ndcY = toClipSpaceY(P, uv.y * 2.0f - 1.0f);
	const V3 nearPoint = clipToWorld(P.inv_view_proj, v3(ndcX, ndcY, 0.0f));
	const V3 farPoint = clipToWorld(P.inv_view_proj, v3(ndcX, ndcY, 1.0f));
	const V3 span = farPoint - nearPoint;
	const float rayLength = length(span);
	const V3 direction = span / rayLength;
	float distance = rayLength;
	const int hit = traceNearestFiltered(bvh, nearPoint, direction, distance, [&](int t)
	{
		float4 n = __ldg(normals + t);
		return n.w > 0.5f || dot(v3(n.x, n.y, n.z), camera - bvh.vertex(t, 0)) > 0.0f;
	});
	if (hit < 0)
	{
		const V4 zero = v4(0.0f, 0.0f, 0.0f, 0.0f);
		storeU8(gb.albedo, i, zero);
		storeU8(gb.normal, i, zero);
		storeH4(gb.emissive, i, zero);
		storeU8(gb.shading_normal, i, zero);
		gb.depth[i] = 1.0f;
		return;
	}
	const V3 position = nearPoint + direction * distance;
	const V4 clip = mul(P.view_proj, v4(position, 1.0f));
	const float4 nn = __ldg(normals + hit);
	const V3 worldNormal = normalize(v3(nn.x, nn.y, nn.z));
	const V3 toCamera = normalize(camera - position);
	const float facing = dot(worldNormal, camera - bvh.vertex(hit, 0)) > 0.0f ? 1.0f : -1.0f;
	V3 normal = worldNormal * facing;
	const float normalView = dot(normal, toCamera);
	if (normalView < 0.05f)
	{
		normal = normalize(normal + toCamera * (0.05f - normalView));
	}
	const int material = int(bvh.row(bvh.triangleOffset + hit * 4).w + 0.5f);
	const float4 m0 = __ldg(materials + 2 * material);
	const float4 m1 = __ldg(materials + 2 * material + 1);
	const V3 encoded = worldNormal * facing * 0.5f + 0.5f;
	storeU8(gb.albedo, i, v4(m0.x, m0.y, m0.z, m0.w));
	storeU8(gb.normal, i, v4(encoded, m1.w));
	storeH4(gb.emissive, i, v4(m1.x, m1.y, m1.z, 1.0f));
	storeU8(gb.shading_normal, i, v4(normal * 0.5f + 0.5f, 1.0f));
	gb.depth[i] = clip.z / clip.w;
}

__global__ void __launch_bounds__(64) shadowAtlasKernel(const RestirParams P, BvhView bvh, float* __restrict__ atlas)
{
	const int f = int(P.shadow_face_size);
	const int W = 3 * f, H = 2 * f;
	const int x = int(blockIdx.x * 8 + threadIdx.x % 8);
	const int y = int(blockIdx.y * 8 + threadIdx.x / 8);
	if (x >= W || y >= H)
	{
		return;
	}
	const bool originBottomLeft = P.origin_bottom_left > 0.5f;
	const int column = x / f;
	const int row = y / f;
	const int face = column + 3 * (originBottomLeft ? 1 - row : row);
	const float inverseFace = 1.0f / float(f);
	const V2 local = v2((float(x - column * f) + 0.5f) * inverseFace, (float(y - row * f) + 0.5f) * inverseFace);
	const float ndcX = local.x * 2.0f - 1.0f;
	const float ndcY = originBottomLeft ? local.y * 2.0f - 1.0f : 1.0f - local.y * 2.0f;
	const V3 nearPoint = clipToWorld(P.shadow_inv_view_proj[face], v3(ndcX, ndcY, 0.0f));
	const V3 farPoint = clipToWorld(P.shadow_inv_view_proj[face], v3(ndcX, ndcY, 1.0f));
	const V3 span = farPoint - nearPoint;
	const float rayLength = length(span);
	const V3 direction = span / rayLength;
	float distance = rayLength;
	const int hit = traceNearestFiltered(bvh, nearPoint, direction, distance, [](int) { return true; });
	float value = 1.0f;
	if (hit >= 0)
	{
		const V3 light = v3(P.light_position[0], P.light_position[1], P.light_position[2]);
		value = length(nearPoint + direction * distance - light) / P.shadow_far;
	}
	atlas[y * W + x] = value;
}

} // namespace
} // namespace restir

using namespace restir;

extern "C" int restir_gbuffer_primary(const RestirParams* params, const RestirScene* scene, const RestirGBuffer* gbuffer,
	void* stream)
{
	if (params == nullptr || scene == nullptr || gbuffer == nullptr || gbuffer->albedo == nullptr || gbuffer->normal == nullptr
		|| gbuffer->emissive == nullptr || gbuffer->shading_normal == nullptr || gbuffer->depth == nullptr
		|| scene->triangle_normals == nullptr || scene->materials == nullptr || params->width == 0 || params->height == 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	dim3 grid((params->width + 7) / 8, (params->height + 7) / 8);
	gbufferKernel<<<grid, 64, 0, asStream(stream)>>>(*params, makeBvhView(scene),
		reinterpret_cast<const float4*>(scene->triangle_normals), reinterpret_cast<const float4*>(scene->materials), *gbuffer);
	return launchStatus();
}

extern "C" int restir_shadow_atlas(const RestirParams* params, const RestirScene* scene, float* atlas, void* stream)
{
	if (params == nullptr || scene == nullptr || atlas == nullptr || params->shadow_face_size == 0)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const uint32_t f = params->shadow_face_size;
	dim3 grid((3 * f + 7) / 8, (2 * f + 7) / 8);
	shadowAtlasKernel<<<grid, 64, 0, asStream(stream)>>>(*params, makeBvhView(scene), atlas);
	return launchStatus();
}
