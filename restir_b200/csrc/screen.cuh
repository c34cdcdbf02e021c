// Screen-space conventions of the passes (restir.sh:150-199, di.sh:71-76),
// with bgfx shaderlib's clip-space helpers fixed as the ABI fixes them: NDC
// depth in [0, 1], texture row 0 at the top unless origin_bottom_left.
#pragma once

#include "common.cuh"

namespace restir
{

__device__ __forceinline__ float toClipSpaceY(const RestirParams& P, float y)
{
	return P.origin_bottom_left > 0.5f ? y : -y;
}

__device__ __forceinline__ V3 clipToWorld(const float* inverse, V3 clip)
{
	V4 w = mul(inverse, v4(clip, 1.0f));
	return v3(w.x / w.w, w.y / w.w, w.z / w.w);
}

__device__ __forceinline__ V3 reconstructWorldPosition(const RestirParams& P, V2 uv, float depth)
{
	V3 clip = v3(uv.x * 2.0f - 1.0f, uv.y * 2.0f - 1.0f, depth);
	clip.y = toClipSpaceY(P, clip.y);
	return clipToWorld(P.inv_view_proj, clip);
}

__device__ __forceinline__ V2 clipToUv(const RestirParams& P, V4 clip)
{
	float originSign = P.origin_bottom_left > 0.5f ? 1.0f : -1.0f;
	V2 c = v2(clip.x, clip.y * originSign);
	return v2(c.x / clip.w * 0.5f + 0.5f, c.y / clip.w * 0.5f + 0.5f);
}

__device__ __forceinline__ bool isOnScreen(V2 uv)
{
	return uv.x > 0.001f && uv.x < 0.999f && uv.y > 0.001f && uv.y < 0.999f;
}

__device__ __forceinline__ V3 decodeNormal(const uint8_t* normal, int i)
{
	V4 n = loadU8(normal, i);
	return normalize(v3(n.x * 2.0f - 1.0f, n.y * 2.0f - 1.0f, n.z * 2.0f - 1.0f));
}

// Texture coordinate of a pixel centre: (x + 0.5) * (1 / size).
__device__ __forceinline__ V2 pixelUv(int x, int y, V2 texel)
{
	return v2((float(x) + 0.5f) * texel.x, (float(y) + 0.5f) * texel.y);
}

} // namespace restir
