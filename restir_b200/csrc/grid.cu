// Hash grid passes: restir_grid_clear (cs_grid_clear.sc:12-21) and
// restir_grid_insert (cs_grid_insert.sc:40-73, gridInsert hashgrid.sh:182-200).
//
// Insertion is warp-aggregated: lanes whose receivers fall in the same cell
// (neighbouring pixels usually do) find each other with __match_any_sync,
// and one leader claims the slot and reserves all their entries with a
// single atomicAdd, instead of one CAS probe sequence and one atomic per
// pixel. In the deterministic mode each cell keeps its C lowest pixel
// indices in increasing order, by an atomicMin cascade down the cell's
// entries (each lane carries the larger value onwards), which leaves the
// same list whatever the arrival order.
#include "grid.cuh"
#include "screen.cuh"

namespace restir
{

__device__ unsigned int g_restirStatus = 0;
__device__ unsigned long long g_restirCounters[RESTIR_COUNTERS] = {};
__device__ int g_restirCounting = 0;

namespace
{

__global__ void __launch_bounds__(256) gridClearKernel(uint4* counts, uint32_t countVectors, uint4* entries, uint32_t entryVectors)
{
	uint32_t stride = gridDim.x * blockDim.x;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < countVectors; i += stride)
	{
		counts[i] = make_uint4(0u, 0u, 0u, 0u);
	}
	if (entries != nullptr)
	{
		for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < entryVectors; i += stride)
		{
			entries[i] = make_uint4(kGridInvalid, kGridInvalid, kGridInvalid, kGridInvalid);
		}
	}
}

__global__ void __launch_bounds__(256) gridInsertKernel(const RestirParams P, const float* __restrict__ depth,
	const uint8_t* __restrict__ normal, uint32_t* grid)
{
	const int w = int(P.gi_width), h = int(P.gi_height);
	const int W = int(P.width), H = int(P.height);
	const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
	const uint32_t T = P.grid_table_size;
	const uint32_t C = P.grid_cell_capacity;
	bool active = i < w * h;
	uint32_t slot = 0u, checksum = 0u;
	if (active)
	{
		int x = i % w, y = i / w;
		V2 texel = v2(1.0f / float(w), 1.0f / float(h));
		V2 uv = pixelUv(x, y, texel);
		int g = texelIndex(uv, W, H);
		float d = loadF1(depth, g);
		if (d >= kSkyDepth)
		{
			active = false;
		}
		else
		{
			V3 position = reconstructWorldPosition(P, uv, d);
			V3 n = decodeNormal(normal, g);
			uint32_t rng = pcg(uint32_t(x) + pcg(uint32_t(y) + pcg(uint32_t(P.frame_index) ^ 0x5bd1e995u)));
			GridView view = makeGridView(&P, grid, P.camera_position);
			float size = view.cellSize(position);
			float r0 = nextRandom(rng);
			float r1 = nextRandom(rng);
			V3 jittered = gridJitter(position, n, size, r0, r1);
			gridKey(jittered, n, size, T - 1u, slot, checksum);
		}
	}

	// Lanes of the same cell: one leader claims the slot and counts them all.
	const unsigned lane = threadIdx.x & 31u;
	unsigned long long key = active ? (static_cast<unsigned long long>(slot) << 32) | checksum : ~0ull;
	unsigned peers = __match_any_sync(0xffffffffu, key);
	int leader = __ffs(peers) - 1;
	unsigned rank = __popc(peers & ((1u << lane) - 1u));
	uint32_t claimed = kGridInvalid;
	uint32_t base = 0u;
	if (active && int(lane) == leader)
	{
		for (uint32_t probe = 0u; probe < kGridMaxProbes; ++probe)
		{
			uint32_t s = (slot + probe) & (T - 1u);
			uint32_t previous = atomicCAS(grid + s, 0u, checksum);
			if (previous == 0u || previous == checksum)
			{
				claimed = s;
				base = atomicAdd(grid + T + s, uint32_t(__popc(peers)));
				break;
			}
		}
		if (claimed == kGridInvalid)
		{
			raiseStatus(2u);
		}
	}
	claimed = __shfl_sync(0xffffffffu, claimed, leader);
	base = __shfl_sync(0xffffffffu, base, leader);
	if (!active || claimed == kGridInvalid)
	{
		return;
	}
	uint32_t* entries = grid + 2u * T + claimed * C;
	if (P.grid_mode == RESTIR_GRID_DETERMINISTIC)
	{
		uint32_t value = uint32_t(i);
		for (uint32_t k = 0u; k < C && value != kGridInvalid; ++k)
		{
			uint32_t old = atomicMin(entries + k, value);
			value = old > value ? old : value;
		}
	}
	else
	{
		uint32_t index = base + rank;
		if (index < C)
		{
			entries[index] = uint32_t(i);
		}
	}
}

} // namespace

} // namespace restir

using namespace restir;

extern "C" int restir_grid_clear(const RestirParams* params, uint32_t* grid, void* stream)
{
	if (params == nullptr || grid == nullptr || params->grid_table_size < 4u
		|| (params->grid_table_size & (params->grid_table_size - 1u)) != 0u || params->grid_cell_capacity == 0u)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const uint32_t T = params->grid_table_size;
	const uint32_t C = params->grid_cell_capacity;
	const uint32_t countVectors = (2u * T) / 4u;
	const bool entries = params->grid_mode == RESTIR_GRID_DETERMINISTIC;
	const uint32_t entryVectors = entries ? (T * C) / 4u : 0u;
	const uint32_t work = countVectors > entryVectors ? countVectors : entryVectors;
	uint32_t blocks = (work + 255u) / 256u;
	blocks = blocks < 148u * 8u ? blocks : 148u * 8u;
	gridClearKernel<<<blocks, 256, 0, asStream(stream)>>>(reinterpret_cast<uint4*>(grid), countVectors,
		entries ? reinterpret_cast<uint4*>(grid + 2u * T) : nullptr, entryVectors);
	return launchStatus();
}

extern "C" int restir_grid_insert(const RestirParams* params, const RestirGBuffer* gbuffer, uint32_t* grid, void* stream)
{
	if (params == nullptr || gbuffer == nullptr || grid == nullptr || gbuffer->depth == nullptr || gbuffer->normal == nullptr
		|| params->gi_width == 0u || params->gi_height == 0u || params->grid_table_size < 4u
		|| (params->grid_table_size & (params->grid_table_size - 1u)) != 0u)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	const uint32_t pixels = params->gi_width * params->gi_height;
	gridInsertKernel<<<(pixels + 255u) / 256u, 256, 0, asStream(stream)>>>(*params, gbuffer->depth, gbuffer->normal, grid);
	return launchStatus();
}

extern "C" int restir_counters(int enable, uint64_t* counters)
{
	unsigned long long values[RESTIR_COUNTERS] = {};
	if (cudaDeviceSynchronize() != cudaSuccess
		|| cudaMemcpyFromSymbol(values, g_restirCounters, sizeof(values)) != cudaSuccess)
	{
		return RESTIR_ERROR_LAUNCH;
	}
	const unsigned long long zero[RESTIR_COUNTERS] = {};
	const int flag = enable != 0 ? 1 : 0;
	if (cudaMemcpyToSymbol(g_restirCounters, zero, sizeof(zero)) != cudaSuccess
		|| cudaMemcpyToSymbol(g_restirCounting, &flag, sizeof(flag)) != cudaSuccess)
	{
		return RESTIR_ERROR_LAUNCH;
	}
	if (counters != nullptr)
	{
		for (int i = 0; i < RESTIR_COUNTERS; ++i)
		{
			counters[i] = values[i];
		}
	}
	return RESTIR_OK;
}

extern "C" int restir_status(uint32_t* flags)
{
	unsigned int value = 0;
	unsigned int zero = 0;
	if (cudaMemcpyFromSymbol(&value, g_restirStatus, sizeof(value)) != cudaSuccess
		|| cudaMemcpyToSymbol(g_restirStatus, &zero, sizeof(zero)) != cudaSuccess)
	{
		return RESTIR_ERROR_LAUNCH;
	}
	if (flags != nullptr)
	{
		*flags = value;
	}
	return RESTIR_OK;
}
