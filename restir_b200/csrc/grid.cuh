// World-space hash grid of GI reservoirs (shaders/hashgrid.sh): keys, lookup
// and the two passes that build it each frame (cs_grid_clear.sc,
// cs_grid_insert.sc). Buffer: uint32 [checksums T][counts T][entries T*C].
#pragma once

#include "common.cuh"

namespace restir
{

#define kGridInvalid 0xffffffffu
#define kGridMaxProbes 8u

__device__ __forceinline__ uint32_t gridHash(uint32_t v)
{
	return pcg(v);
}

__device__ __forceinline__ uint32_t gridChecksumHash(uint32_t v)
{
	v ^= v >> 15u;
	v *= 2246822519u;
	v ^= v >> 13u;
	v *= 3266489917u;
	v ^= v >> 16u;
	return v;
}

struct GridView
{
	const uint32_t* data;
	uint32_t tableSize;
	uint32_t capacity;
	float minCell;
	float pixelSize;
	float cellPixels;
	bool worldSpace;
	V3 camera;

	__device__ __forceinline__ uint32_t mask() const { return tableSize - 1u; }

	// hashgrid.sh:82-87, with floor(log2) from the exponent and exp2 of an
	// integer built exactly (include/restir_numeric.h).
	__device__ __forceinline__ float cellSize(V3 p) const
	{
		float target = distance(p, camera) * pixelSize * cellPixels;
		float level = float(rn_floor_log2(fmaxf(target / minCell, 1.0f)));
		return minCell * rn_exp2i(int(level));
	}
};

__host__ __device__ inline GridView makeGridView(const RestirParams* p, const uint32_t* data, const float* camera)
{
	GridView g;
	g.data = data;
	g.tableSize = p->grid_table_size;
	g.capacity = p->grid_cell_capacity;
	g.minCell = p->grid_min_cell;
	g.pixelSize = p->grid_pixel_size;
	g.cellPixels = p->grid_cell_pixels;
	g.worldSpace = p->world_space_reuse > 0.5f;
	g.camera = { camera[0], camera[1], camera[2] };
	return g;
}

__device__ __forceinline__ uint32_t gridNormalBucket(V3 n)
{
	V3 a = vabs(n);
	uint32_t bucket = n.z >= 0.0f ? 4u : 5u;
	if (a.x >= a.y && a.x >= a.z)
	{
		bucket = n.x >= 0.0f ? 0u : 1u;
	}
	else if (a.y >= a.z)
	{
		bucket = n.y >= 0.0f ? 2u : 3u;
	}
	return bucket;
}

__device__ __forceinline__ V3 gridJitter(V3 p, V3 n, float cellSize, float r0, float r1)
{
	V3 tangent = normalize(fabsf(n.y) < 0.99f ? cross(n, v3(0.0f, 1.0f, 0.0f)) : cross(n, v3(1.0f, 0.0f, 0.0f)));
	V3 bitangent = cross(n, tangent);
	return p + (tangent * (r0 - 0.5f) + bitangent * (r1 - 0.5f)) * cellSize;
}

__device__ __forceinline__ void gridKey(V3 p, V3 n, float cellSize, uint32_t tableMask, uint32_t& slot, uint32_t& checksum)
{
	V3 c = v3(floorf(p.x / cellSize), floorf(p.y / cellSize), floorf(p.z / cellSize));
	int cx = int(c.x), cy = int(c.y), cz = int(c.z);
	uint32_t level = __float_as_uint(cellSize);
	uint32_t bucket = gridNormalBucket(n);
	slot = gridHash(level + gridHash(bucket + gridHash(uint32_t(cx) + gridHash(uint32_t(cy) + gridHash(uint32_t(cz)))))) & tableMask;
	uint32_t sum = gridChecksumHash(level ^ gridChecksumHash(bucket ^ gridChecksumHash(
		uint32_t(cx) ^ gridChecksumHash(uint32_t(cy) ^ gridChecksumHash(uint32_t(cz) + 0x9e3779b9u)))));
	checksum = sum > 1u ? sum : 1u;
}

// hashgrid.sh:132-150
__device__ __forceinline__ uint32_t gridFindCell(const GridView& g, uint32_t slot0, uint32_t checksum)
{
	for (uint32_t probe = 0u; probe < kGridMaxProbes; ++probe)
	{
		uint32_t slot = (slot0 + probe) & g.mask();
		uint32_t stored = __ldg(g.data + slot);
		if (stored == checksum)
		{
			return slot;
		}
		if (stored == 0u)
		{
			break;
		}
	}
	return kGridInvalid;
}

// hashgrid.sh:155-177
__device__ __forceinline__ uint32_t gridPickEntry(const GridView& g, V3 p, V3 n, float r0, float r1, float r2)
{
	float size = g.cellSize(p);
	V3 jittered = gridJitter(p, n, size, r0, r1);
	uint32_t slot, checksum;
	gridKey(jittered, n, size, g.mask(), slot, checksum);
	uint32_t cell = gridFindCell(g, slot, checksum);
	if (cell == kGridInvalid)
	{
		return kGridInvalid;
	}
	uint32_t count = min(__ldg(g.data + g.tableSize + cell), g.capacity);
	if (count == 0u)
	{
		return kGridInvalid;
	}
	uint32_t index = min(uint32_t(r2 * float(count)), count - 1u);
	return __ldg(g.data + 2u * g.tableSize + cell * g.capacity + index);
}

} // namespace restir
