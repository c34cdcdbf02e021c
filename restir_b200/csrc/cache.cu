// The radiance cache (include/restir_cache.h): multiresolution hash-grid
// encoding, a 64-wide MLP on the tcgen05 tensor cores, its backward pass,
// and Adam.
//
// The MLP runs "fully fused" per tile of 128 queries, one query per thread
// and per TMEM lane: the layer's input tile (128 x 64 bfloat16) and the
// weights sit in shared memory as umma.cuh's core matrices, one thread
// issues the tile's MMAs (K = 16 each) into a 128 x 64 FP32 accumulator in
// TMEM, and every thread reads its own row back (tcgen05.ld), applies the
// ReLU, rounds to bfloat16 and writes the next layer's input row. The
// training kernel keeps every layer's activations in shared memory for the
// backward pass and accumulates the weight gradients of all its tiles in
// TMEM (dW = dZ^T H, with K = the 128 rows of a tile), then writes one row
// of per-block partial sums; a reduction kernel sums the rows in a fixed
// order. The hash-table gradient is scattered with atomics onto 64-bit
// fixed-point sums, whose integer addition does not depend on the order the
// atomics land in, so a training step is deterministic.
#include "common.cuh"
#include "umma.cuh"

#include "../../include/restir_cache.h"

namespace restir
{
namespace
{

constexpr int kTile = 128;
constexpr uint32_t kWaitPolls = 1u << 22;
constexpr uint32_t kStatusTensor = 8u;  // a tensor-core step failed (status word bit 3)
constexpr int kWeightLayerBytes = 64 * 64 * 2;
constexpr int kWeightBytes = RESTIR_CACHE_WEIGHTS * 2;  // 34816
constexpr int kTileBytes = kTile * 64 * 2;              // 16384

__host__ __device__ constexpr int weightOffset(int layer)
{
	return layer * 64 * 64;
}

struct CacheView
{
	const uint16_t* weightsBf16;
	const uint16_t* tableHalf;
	float boundsMin[3];
	float boundsMax[3];
	float levelScale[RESTIR_CACHE_LEVELS];
	uint32_t denseLevels;  // bit l: level l indexed densely
	uint32_t entries;
};

CacheView makeView(const RestirCacheConfig& cfg, const RestirCacheLayout& l, const void* state)
{
	const char* base = static_cast<const char*>(state);
	CacheView v;
	v.weightsBf16 = reinterpret_cast<const uint16_t*>(base + l.weights_bf16);
	v.tableHalf = reinterpret_cast<const uint16_t*>(base + l.table_half);
	for (int i = 0; i < 3; ++i)
	{
		v.boundsMin[i] = cfg.bounds_min[i];
		v.boundsMax[i] = cfg.bounds_max[i];
	}
	v.denseLevels = 0;
	for (int level = 0; level < RESTIR_CACHE_LEVELS; ++level)
	{
		v.levelScale[level] = l.level_scale[level];
		v.denseLevels |= l.level_dense[level] ? (1u << level) : 0u;
	}
	v.entries = l.entries;
	return v;
}

// --- the encoding ----------------------------------------------------------------

// The 8 corners of the query's cell on one level: table indices and
// trilinear weights, corner d = (d & 1, d >> 1 & 1, d >> 2).
struct LevelCorners
{
	uint32_t index[8];
	float weight[8];
};

__device__ __forceinline__ float unitCoordinate(float p, float lo, float hi)
{
	return fminf(fmaxf((p - lo) / (hi - lo), 0.0f), 1.0f);
}

// The table slot of corner (x, y, z): corners are stored in 2x2x2 bricks of
// 8 consecutive entries (32 bytes of half features, one L2 sector), so a
// cell's 8 corners fall in 1, 2, 4 or 8 sectors (3.4 on average) instead of
// up to 8. A dense level numbers the bricks x + y * b + z * b^2; a hashed
// level hashes the brick coordinates (XOR of the coordinates times 1,
// 2654435761, 805459861, as Mueller et al. 2022 hash corners) onto the
// table's entries / 8 bricks.
__device__ __forceinline__ uint32_t brickIndex(bool dense, uint32_t x, uint32_t y, uint32_t z, uint32_t bricks,
	uint32_t entries)
{
	const uint32_t local = (x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2);
	const uint32_t bx = x >> 1, by = y >> 1, bz = z >> 1;
	const uint32_t brick = dense ? bx + by * bricks + bz * bricks * bricks
		: ((bx * 1u) ^ (by * 2654435761u) ^ (bz * 805459861u)) & ((entries >> 3) - 1u);
	return brick * 8u + local;
}

__device__ __forceinline__ void levelCorners(const CacheView& c, int level, const float unit[3], LevelCorners& out)
{
	const float scale = c.levelScale[level];
	const int resolution = int(scale);
	int cell[3];
	float frac[3];
	for (int a = 0; a < 3; ++a)
	{
		const float g = unit[a] * scale;
		cell[a] = min(int(floorf(g)), resolution - 1);
		frac[a] = g - float(cell[a]);
	}
	const bool dense = (c.denseLevels >> level) & 1u;
	const uint32_t bricks = uint32_t(resolution + 2) >> 1;  // bricks across a dense level
	for (int d = 0; d < 8; ++d)
	{
		const uint32_t x = uint32_t(cell[0] + (d & 1));
		const uint32_t y = uint32_t(cell[1] + ((d >> 1) & 1));
		const uint32_t z = uint32_t(cell[2] + (d >> 2));
		const float wx = (d & 1) ? frac[0] : 1.0f - frac[0];
		const float wy = ((d >> 1) & 1) ? frac[1] : 1.0f - frac[1];
		const float wz = (d >> 2) ? frac[2] : 1.0f - frac[2];
		out.weight[d] = wx * wy * wz;
		out.index[d] = brickIndex(dense, x, y, z, bricks, c.entries);
	}
}

__device__ __forceinline__ void unitPosition(const CacheView& c, const float4& q0, float unit[3])
{
	unit[0] = unitCoordinate(q0.x, c.boundsMin[0], c.boundsMax[0]);
	unit[1] = unitCoordinate(q0.y, c.boundsMin[1], c.boundsMax[1]);
	unit[2] = unitCoordinate(q0.z, c.boundsMin[2], c.boundsMax[2]);
}

// Two floats as a pair of bfloat16 (lo in the low half), one cvt
// instruction. The conversion rounds to nearest even as restir_numeric.h's
// rn_float_to_bf16 does, so the bits are the same for every non-NaN input.
__device__ __forceinline__ uint32_t packBf16(float lo, float hi)
{
	uint32_t pair;
	asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(pair) : "f"(hi), "f"(lo));
	return pair;
}

// The two halves of a pair of FP16 features as floats (exact conversions).
__device__ __forceinline__ void unpackHalf2(uint32_t pair, float& lo, float& hi)
{
	asm("{\n\t.reg .b16 l, h;\n\tmov.b32 {l, h}, %2;\n\tcvt.f32.f16 %0, l;\n\tcvt.f32.f16 %1, h;\n\t}"
		: "=f"(lo), "=f"(hi) : "r"(pair));
}

// A float as FP16, rounded to nearest even (rn_float_to_half's bits for
// every non-NaN input).
__device__ __forceinline__ uint16_t toHalf(float f)
{
	uint16_t h;
	asm("cvt.rn.f16.f32 %0, %1;" : "=h"(h) : "f"(f));
	return h;
}

__device__ __forceinline__ uint4 choose(bool p, const uint4& a, const uint4& b)
{
	return make_uint4(p ? a.x : b.x, p ? a.y : b.y, p ? a.z : b.z, p ? a.w : b.w);
}

// Entry (b0 + 2 b1) of a 16-byte half brick (4 entries: local x + 2 y).
__device__ __forceinline__ uint32_t pickEntry(const uint4& h, bool b0, bool b1)
{
	const uint32_t lo = b0 ? h.y : h.x;
	const uint32_t hi = b0 ? h.w : h.z;
	return b1 ? hi : lo;
}

// A whole brick (8 entries, 32 bytes: one L2 sector) in one 256-bit load;
// a brick starts on a 32-byte boundary (the table is 256-byte aligned and a
// level is a whole number of bricks).
struct Brick
{
	uint4 lo;  // the z = 0 plane: locals 0-3
	uint4 hi;  // the z = 1 plane: locals 4-7
};

__device__ __forceinline__ Brick loadBrick(const uint4* p)
{
	Brick b;
	asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
		: "=r"(b.lo.x), "=r"(b.lo.y), "=r"(b.lo.z), "=r"(b.lo.w), "=r"(b.hi.x), "=r"(b.hi.y), "=r"(b.hi.z), "=r"(b.hi.w)
		: "l"(p));
	return b;
}

// The feature pairs of a cell's 8 corners on one level, each brick read
// once. Along an axis where the cell's coordinate is even both corners lie
// in one brick; where it is odd they lie in neighbouring bricks. So the
// corners sit in (1 + odd x)(1 + odd y)(1 + odd z) bricks, 3.4 on average:
// those are loaded whole (the others are predicated off) instead of 8
// 4-byte loads in as many sectors, and each corner picks its entry. The
// values are the ones levelCorners' indices address.
__device__ __forceinline__ void levelPairs(const CacheView& c, int level, const int cell[3], uint32_t pair[8])
{
	const bool dense = (c.denseLevels >> level) & 1u;
	const uint32_t bricks = uint32_t(int(c.levelScale[level]) + 2) >> 1;
	const uint32_t mask = (c.entries >> 3) - 1u;
	const uint32_t bx = uint32_t(cell[0]) >> 1, by = uint32_t(cell[1]) >> 1, bz = uint32_t(cell[2]) >> 1;
	const bool ox = cell[0] & 1, oy = cell[1] & 1, oz = cell[2] & 1;
	// brickIndex's terms per axis, for brick offsets 0 and 1.
	uint32_t tx[2], ty[2], tz[2];
	for (uint32_t k = 0; k < 2; ++k)
	{
		tx[k] = dense ? bx + k : (bx + k) * 1u;
		ty[k] = dense ? (by + k) * bricks : (by + k) * 2654435761u;
		tz[k] = dense ? (bz + k) * bricks * bricks : (bz + k) * 805459861u;
	}
	const uint4* table = reinterpret_cast<const uint4*>(c.tableHalf) + size_t(level) * (c.entries >> 2);
	// plane[ez][dy][dx]: the 4 entries (local x + 2 y) of corner plane z = cell z + ez
	// in brick column (dx, dy): with z even both planes are the brick's; with z
	// odd plane 0 is the upper half of brick z and plane 1 the lower half of brick z + 1.
	uint4 plane[2][2][2];
#pragma unroll
	for (int dy = 0; dy < 2; ++dy)
	{
#pragma unroll
		for (int dx = 0; dx < 2; ++dx)
		{
			Brick b0 = { make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u) };
			Brick b1 = b0;
			if ((dx == 0 || ox) && (dy == 0 || oy))
			{
				const uint32_t column = dense ? tx[dx] + ty[dy] : tx[dx] ^ ty[dy];
				const uint32_t brick0 = dense ? column + tz[0] : (column ^ tz[0]) & mask;
				b0 = loadBrick(table + size_t(brick0) * 2u);
				if (oz)
				{
					const uint32_t brick1 = dense ? column + tz[1] : (column ^ tz[1]) & mask;
					b1 = loadBrick(table + size_t(brick1) * 2u);
				}
			}
			plane[0][dy][dx] = choose(oz, b0.hi, b0.lo);
			plane[1][dy][dx] = choose(oz, b1.lo, b0.hi);
		}
	}
	// Corner (ex, ey, ez): column (ox & ex, oy & ey), entry ((ox ^ ex), (oy ^ ey)).
#pragma unroll
	for (int ez = 0; ez < 2; ++ez)
	{
#pragma unroll
		for (int ey = 0; ey < 2; ++ey)
		{
#pragma unroll
			for (int ex = 0; ex < 2; ++ex)
			{
				const bool cx = ox && ex, cy = oy && ey;
				const uint4 lo = choose(cx, plane[ez][0][1], plane[ez][0][0]);
				const uint4 hi = choose(cx, plane[ez][1][1], plane[ez][1][0]);
				pair[ex + 2 * ey + 4 * ez] = pickEntry(choose(cy, hi, lo), ox != bool(ex), oy != bool(ey));
			}
		}
	}
}


// The 64 network inputs of one query as bfloat16, 8 per 16-byte chunk. The
// levels are unrolled so that the gathers of all levels can be in flight
// together; each level still sums its corners in order d = 0..7.
__device__ inline void queryFeatures(const CacheView& c, const float4* query, uint4 chunk[8])
{
	const float4 q0 = query[0], q1 = query[1], q2 = query[2], q3 = query[3];
	float unit[3];
	unitPosition(c, q0, unit);
	uint32_t packed[32];
#pragma unroll
	for (int level = 0; level < RESTIR_CACHE_LEVELS; ++level)
	{
		const float scale = c.levelScale[level];
		const int resolution = int(scale);
		int cell[3];
		float frac[3];
		for (int a = 0; a < 3; ++a)
		{
			const float g = unit[a] * scale;
			cell[a] = min(int(floorf(g)), resolution - 1);
			frac[a] = g - float(cell[a]);
		}
		uint32_t pair[8];
		levelPairs(c, level, cell, pair);
		LevelCorners corners;
		for (int d = 0; d < 8; ++d)
		{
			const float wx = (d & 1) ? frac[0] : 1.0f - frac[0];
			const float wy = ((d >> 1) & 1) ? frac[1] : 1.0f - frac[1];
			const float wz = (d >> 2) ? frac[2] : 1.0f - frac[2];
			corners.weight[d] = wx * wy * wz;
		}
		float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
		for (int d = 0; d < 8; ++d)
		{
			float h0, h1;
			unpackHalf2(pair[d], h0, h1);
			f0 = f0 + corners.weight[d] * h0;
			f1 = f1 + corners.weight[d] * h1;
		}
		packed[level] = packBf16(f0, f1);
	}
	// Inputs 32..42: direction, normal, roughness, albedo, then the constant 1.
	packed[16] = packBf16(q2.x, q2.y);
	packed[17] = packBf16(q2.z, q1.x);
	packed[18] = packBf16(q1.y, q1.z);
	packed[19] = packBf16(q0.w, q3.x);
	packed[20] = packBf16(q3.y, q3.z);
	packed[21] = packBf16(1.0f, 0.0f);
#pragma unroll
	for (int i = 22; i < 32; ++i)
	{
		packed[i] = 0u;
	}
#pragma unroll
	for (int k = 0; k < 8; ++k)
	{
		chunk[k] = make_uint4(packed[4 * k], packed[4 * k + 1], packed[4 * k + 2], packed[4 * k + 3]);
	}
}

// --- shared-memory tiles -------------------------------------------------------------

// Row r of a 64-column tile from 8 chunks of 8 bfloat16.
__device__ __forceinline__ void storeRow(uint8_t* tile, int r, const uint4 chunk[8])
{
	for (int k = 0; k < 8; ++k)
	{
		*reinterpret_cast<uint4*>(tile + umma::coreOffset(uint32_t(r), uint32_t(8 * k), 64u)) = chunk[k];
	}
}

__device__ __forceinline__ uint16_t rowElement(const uint8_t* tile, int r, int k, int columns)
{
	return *reinterpret_cast<const uint16_t*>(tile + umma::coreOffset(uint32_t(r), uint32_t(k), uint32_t(columns)));
}

// All weights (bfloat16 [out][in]) into shared memory, layer by layer.
__device__ __forceinline__ void loadWeights(uint8_t* smem, const uint16_t* weights)
{
	const uint4* source = reinterpret_cast<const uint4*>(weights);
	for (int chunk = int(threadIdx.x); chunk < RESTIR_CACHE_WEIGHTS / 8; chunk += int(blockDim.x))
	{
		const int element = chunk * 8;
		const int layer = element < 4 * 4096 ? element / 4096 : 4;
		const int local = element - weightOffset(layer);
		const int out = local / 64, in = local % 64;
		*reinterpret_cast<uint4*>(smem + layer * kWeightLayerBytes + umma::coreOffset(uint32_t(out), uint32_t(in), 64u))
			= __ldg(source + chunk);
	}
}

// ReLU of 16 accumulator columns into 2 chunks of bfloat16.
__device__ __forceinline__ void reluChunks(const float* v, uint4* chunk)
{
	uint32_t h[8];
	for (int i = 0; i < 8; ++i)
	{
		h[i] = packBf16(fmaxf(v[2 * i], 0.0f), fmaxf(v[2 * i + 1], 0.0f));
	}
	chunk[0] = make_uint4(h[0], h[1], h[2], h[3]);
	chunk[1] = make_uint4(h[4], h[5], h[6], h[7]);
}

// The CTA's tensor-core context: its TMEM columns, its mbarrier and phase.
struct TensorContext
{
	uint32_t tmem = 0;
	uint32_t barrier = 0;
	uint32_t phase = 0;
	bool ok = true;
	int group = 0;  // the tile group of 128 threads that owns the context (named barrier 1 + group)
};

// The 128 threads of tile group g meet at named barrier 1 + g (barrier 0 is
// __syncthreads'), so the groups of a block run their tiles independently.
__device__ __forceinline__ void groupSync(int group)
{
	asm volatile("bar.sync %0, 128;" ::"r"(group + 1) : "memory");
}

// The group's barrier as a vote: true if `p` holds in all its 128 threads.
__device__ __forceinline__ bool groupAll(int group, bool p)
{
	uint32_t all;
	asm volatile(
		"{\n\t.reg .pred p, q;\n\t"
		"setp.ne.u32 p, %1, 0;\n\t"
		"bar.red.and.pred q, %2, 128, p;\n\t"
		"selp.u32 %0, 1, 0, q;\n\t}\n"
		: "=r"(all)
		: "r"(p ? 1u : 0u), "r"(group + 1)
		: "memory");
	return all != 0u;
}

// Every thread waits for the barrier's current phase, at most `polls` polls;
// a wait that gives up raises status bit 3 and marks the context failed (the
// kernel then skips its remaining tensor-core steps and frees its TMEM).
__device__ __forceinline__ void awaitBarrier(TensorContext& t, uint32_t polls)
{
	bool done = umma::barrierWait(t.barrier, t.phase, polls);
	t.phase ^= 1u;
	done = groupAll(t.group, done);
	if (!done)
	{
		if ((threadIdx.x & (kTile - 1)) == 0)
		{
			raiseStatus(kStatusTensor);
		}
		t.ok = false;
	}
	umma::fenceAfterSync();
}

// Commit by the issuing thread (the group's first), then every thread of the
// group waits for the MMAs. A commit tracks the MMAs its own thread issued,
// so the groups of a block complete independently.
__device__ __forceinline__ void completeMmas(TensorContext& t)
{
	if ((threadIdx.x & (kTile - 1)) == 0)
	{
		umma::commit(t.barrier);
	}
	awaitBarrier(t, kWaitPolls);
}

// The failure path of the bounded wait, with no MMA: an mbarrier that no one
// arrives at, waited on as completeMmas waits (restir_cache_wait_check).
__global__ void __launch_bounds__(128) waitCheckKernel(uint32_t polls, uint32_t* result)
{
	__shared__ __align__(8) uint64_t barrier;
	TensorContext t;
	t.barrier = umma::smemAddress(&barrier);
	t.phase = 0;
	t.ok = true;
	t.tmem = 0;
	t.group = 0;
	if (threadIdx.x == 0)
	{
		umma::barrierInit(t.barrier, 1);
	}
	__syncthreads();
	awaitBarrier(t, polls);
	if (threadIdx.x == 0)
	{
		*result = t.ok ? 1u : 0u;
	}
}

// The descriptors address the tiles from the start of dynamic shared memory,
// which must be 1024-byte aligned: the MMA reads a misaligned tile as if it
// started at the aligned address below it. (Static __shared__ variables in a
// kernel move the dynamic region; these kernels have none.)
__device__ __forceinline__ bool alignedTiles(const uint8_t* smem)
{
	if ((umma::smemAddress(smem) & 1023u) == 0u)
	{
		return true;
	}
	if (threadIdx.x == 0)
	{
		raiseStatus(kStatusTensor);
	}
	return false;
}

// Before the issuing thread reads shared memory written by all threads or
// overwrites TMEM they read: every thread fences, then the block syncs.
__device__ __forceinline__ void handOff()
{
	umma::fenceSharedForAsync();
	umma::fenceBeforeSync();
	__syncthreads();
	umma::fenceAfterSync();
}

// The same within one tile group.
__device__ __forceinline__ void groupHandOff(int group)
{
	umma::fenceSharedForAsync();
	umma::fenceBeforeSync();
	groupSync(group);
	umma::fenceAfterSync();
}

// D (128 x n) = A (128 x 64, K-major tile) * W^T for one layer with n outputs.
__device__ __forceinline__ void issueLayer(uint32_t tmemD, const uint8_t* a, const uint8_t* w, int n)
{
	const uint32_t instr = umma::instrDescriptorBf16(128u, uint32_t(n), 0u, 0u);
	const uint32_t aBase = umma::smemAddress(a), wBase = umma::smemAddress(w);
	for (int s = 0; s < 4; ++s)
	{
		umma::mma(tmemD, umma::smemDescriptor(aBase + 256u * s, 128u, 1024u), umma::smemDescriptor(wBase + 256u * s, 128u, 1024u),
			instr, s > 0);
	}
}

// --- forward ----------------------------------------------------------------------------

// A forward block runs kGroups tile groups of 128 threads (4 warps each),
// which share one copy of the weights in shared memory and each own an
// activation tile, an mbarrier and 64 TMEM columns: the weights are paid
// once per block, so more tiles are in flight per SM, and each group's
// gathers overlap the other groups' MMA chains. Named barriers keep the
// groups independent. Blocks per SM: 4 of 1 group (128 registers a thread),
// 3 of 2 (80), 2 of 4 (64). With the encoding's whole-brick loads, on
// 2,073,600 random queries: 1 group 0.934 ms, 2 groups 0.947, 4 groups 1.132
// (at 64 registers the 16 levels' brick loads spill); the renderer uses 1.
constexpr int kForwardGroups = 1;

template<int kGroups>
struct ForwardShape
{
	static constexpr int threads = kTile * kGroups;
	static constexpr int blocksPerSm = kGroups == 1 ? 4 : (kGroups == 2 ? 3 : 2);
	static constexpr int smem = kWeightBytes + kGroups * kTileBytes + 64;
	static constexpr uint32_t columns = 64u * uint32_t(kGroups);
};

template<int kMode, int kGroups>  // kMode 0: half4 cache values, 1: 16 raw floats, 2: the 64 inputs
__global__ void __launch_bounds__(ForwardShape<kGroups>::threads, ForwardShape<kGroups>::blocksPerSm)
	forwardKernel(CacheView c, const float4* __restrict__ queries, uint32_t n, void* __restrict__ output)
{
	extern __shared__ __align__(1024) uint8_t smem[];
	const int tid = int(threadIdx.x);
	const int warp = tid >> 5;
	const int group = tid / kTile;
	const int r = tid % kTile;  // the thread's row of its group's tile and its TMEM lane
	uint8_t* weights = smem;
	uint8_t* act = smem + kWeightBytes + group * kTileBytes;
	uint64_t* barriers = reinterpret_cast<uint64_t*>(smem + kWeightBytes + kGroups * kTileBytes);
	uint32_t* slot = reinterpret_cast<uint32_t*>(barriers + kGroups);
	const uint32_t tiles = (n + kTile - 1) / kTile;

	if (kMode == 2)
	{
		for (uint32_t row = blockIdx.x * blockDim.x + uint32_t(tid); row < n; row += gridDim.x * blockDim.x)
		{
			uint4 chunk[8];
			queryFeatures(c, queries + size_t(row) * 4, chunk);
			uint4* out = static_cast<uint4*>(output) + size_t(row) * 8;
			for (int k = 0; k < 8; ++k)
			{
				out[k] = chunk[k];
			}
		}
		return;
	}

	if (!alignedTiles(smem))
	{
		return;
	}
	loadWeights(weights, c.weightsBf16);
	if (tid < kGroups)
	{
		umma::barrierInit(umma::smemAddress(barriers + tid), 1);
	}
	if (warp == 0)
	{
		umma::tmemAllocate(umma::smemAddress(slot), ForwardShape<kGroups>::columns);
	}
	umma::fenceBeforeSync();
	__syncthreads();
	umma::fenceAfterSync();
	const uint32_t tmemBase = *slot;
	TensorContext t;
	t.tmem = tmemBase + 64u * uint32_t(group);
	t.barrier = umma::smemAddress(barriers + group);
	t.phase = 0;
	t.ok = true;
	t.group = group;
	// A warp reads the TMEM lanes of its quarter of the group: 32 * (warp % 4).
	const uint32_t laneBase = uint32_t((warp & 3) * 32) << 16;

	for (uint32_t tile = blockIdx.x * kGroups + uint32_t(group); tile < tiles && t.ok; tile += gridDim.x * kGroups)
	{
		const uint32_t row = tile * kTile + uint32_t(r);
		uint4 chunk[8];
		if (row < n)
		{
			queryFeatures(c, queries + size_t(row) * 4, chunk);
		}
		else
		{
			for (int k = 0; k < 8; ++k)
			{
				chunk[k] = make_uint4(0u, 0u, 0u, 0u);
			}
		}
		storeRow(act, r, chunk);
		for (int layer = 0; layer < 5 && t.ok; ++layer)
		{
			groupHandOff(group);
			const int width = layer < 4 ? 64 : 16;
			if (r == 0)
			{
				issueLayer(t.tmem, act, weights + layer * kWeightLayerBytes, width);
			}
			completeMmas(t);
			if (!t.ok)
			{
				break;
			}
			if (layer < 4)
			{
				for (int q = 0; q < 4; ++q)
				{
					float v[16];
					umma::tmemLoad16(t.tmem + laneBase + uint32_t(16 * q), v);
					uint4 relu[2];
					reluChunks(v, relu);
					*reinterpret_cast<uint4*>(act + umma::coreOffset(uint32_t(r), uint32_t(16 * q), 64u)) = relu[0];
					*reinterpret_cast<uint4*>(act + umma::coreOffset(uint32_t(r), uint32_t(16 * q + 8), 64u)) = relu[1];
				}
			}
			else
			{
				float v[16];
				umma::tmemLoad16(t.tmem + laneBase, v);
				if (row < n)
				{
					if (kMode == 0)
					{
						ushort4 h;
						h.x = toHalf(fmaxf(v[0], 0.0f));
						h.y = toHalf(fmaxf(v[1], 0.0f));
						h.z = toHalf(fmaxf(v[2], 0.0f));
						h.w = toHalf(queries[size_t(row) * 4 + 1].w > 0.5f ? 1.0f : 0.0f);
						static_cast<ushort4*>(output)[row] = h;
					}
					else
					{
						float4* out = static_cast<float4*>(output) + size_t(row) * 4;
						for (int k = 0; k < 4; ++k)
						{
							out[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
						}
					}
				}
			}
		}
	}
	umma::fenceBeforeSync();
	__syncthreads();
	if (warp == 0)
	{
		umma::fenceAfterSync();
		umma::tmemFree(tmemBase, ForwardShape<kGroups>::columns);
	}
}

// --- training: forward, loss, backward -------------------------------------------------

// Shared memory: weights, the output gradient (128 x 16), the hidden
// gradient, the input and the four hidden activations (128 x 64 each). The
// output gradient is read as a 128-row MN-major operand of which only 16
// rows exist; the rows past it fall on the following tiles and produce
// accumulator rows that are never read.
constexpr int kTrainDOut = kWeightBytes;
constexpr int kTrainDZ = kTrainDOut + kTile * 16 * 2;
constexpr int kTrainX = kTrainDZ + kTileBytes;
constexpr int kTrainH = kTrainX + kTileBytes;      // H1..H4
constexpr int kTrainBarrier = kTrainH + 4 * kTileBytes;
constexpr int kTrainSmem = kTrainBarrier + 64;
// TMEM columns: [0, 64) the layer accumulator, then dW0..dW4 64 each.
constexpr uint32_t kTrainColumns = 512;

__device__ __forceinline__ uint64_t kMajor(const uint8_t* tile, int kStep, int columns)
{
	return umma::smemDescriptor(umma::smemAddress(tile) + 256u * uint32_t(kStep), 128u, uint32_t(columns / 8) * 128u);
}

// The tile read transposed: rows are the reduction dimension.
__device__ __forceinline__ uint64_t mnMajor(const uint8_t* tile, int kStep, int columns)
{
	const uint32_t rowGroup = uint32_t(columns / 8) * 128u;
	return umma::smemDescriptor(umma::smemAddress(tile) + 2u * rowGroup * uint32_t(kStep), rowGroup, 128u);
}

struct TrainArgs
{
	CacheView c;
	const float4* queries;
	const float4* targets;
	uint32_t n;
	const float* scalars;   // RestirCacheScalars: loss_scale first
	uint32_t* nonfinite;    // RestirCacheScalars::nonfinite
	float* partials;        // [blocks][RESTIR_CACHE_PARTIAL_STRIDE]
	unsigned long long* tableGradFixed; // the table gradient in fixed point (kGradientFixedScale)
};

// The hash table's gradient is summed in 64-bit fixed point, units of 2^-32
// of the loss-scaled gradient: integer addition is associative, so the sum
// of the samples' scattered contributions does not depend on the order the
// atomics land in, and a training step is reproducible bit for bit. One
// contribution of magnitude 2^20 or more (or not finite) marks the step
// non-finite instead (the loss-scale logic then halves the scale and skips
// it); a sum stays within range below 2^11 such contributions per entry.
constexpr float kGradientFixedScale = 4294967296.0f; // 2^32
constexpr float kGradientFixedLimit = 1048576.0f;    // 2^20

__device__ __forceinline__ void scatterFixed(unsigned long long* target, float value, bool& overflow)
{
	if (!(fabsf(value) < kGradientFixedLimit))
	{
		overflow = true;
		return;
	}
	atomicAdd(target, static_cast<unsigned long long>(__float2ll_rn(value * kGradientFixedScale)));
}

__global__ void __launch_bounds__(kTile, 1) trainKernel(TrainArgs a)
{
	extern __shared__ __align__(1024) uint8_t smem[];
	uint8_t* weights = smem;
	uint8_t* dOut = smem + kTrainDOut;
	uint8_t* dZ = smem + kTrainDZ;
	uint8_t* x = smem + kTrainX;
	uint8_t* hidden[4] = { smem + kTrainH, smem + kTrainH + kTileBytes, smem + kTrainH + 2 * kTileBytes,
		smem + kTrainH + 3 * kTileBytes };
	uint64_t* barrier = reinterpret_cast<uint64_t*>(smem + kTrainBarrier);
	uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kTrainBarrier + 8);
	float* lossWarp = reinterpret_cast<float*>(smem + kTrainBarrier + 16);
	const int tid = int(threadIdx.x);
	const int warp = tid >> 5;
	const uint32_t tiles = (a.n + kTile - 1) / kTile;
	const float lossScale = a.scalars[0];
	const float gradientScale = 2.0f / (3.0f * float(a.n));
	if (!alignedTiles(smem))
	{
		return;
	}

	loadWeights(weights, a.c.weightsBf16);
	TensorContext t;
	t.barrier = umma::smemAddress(barrier);
	t.phase = 0;
	t.ok = true;
	if (tid == 0)
	{
		umma::barrierInit(t.barrier, 1);
	}
	if (warp == 0)
	{
		umma::tmemAllocate(umma::smemAddress(slot), kTrainColumns);
	}
	umma::fenceBeforeSync();
	__syncthreads();
	umma::fenceAfterSync();
	t.tmem = *slot;
	const uint32_t laneBase = uint32_t(warp * 32) << 16;
	const uint32_t instrBackward = umma::instrDescriptorBf16(128u, 64u, 0u, 1u);
	const uint32_t instrWeights = umma::instrDescriptorBf16(128u, 64u, 1u, 1u);
	float lossSum = 0.0f;
	bool first = true;

	for (uint32_t tile = blockIdx.x; tile < tiles && t.ok; tile += gridDim.x)
	{
		const uint32_t row = tile * kTile + uint32_t(tid);
		const bool valid = row < a.n;
		uint4 chunk[8];
		if (valid)
		{
			queryFeatures(a.c, a.queries + size_t(row) * 4, chunk);
		}
		else
		{
			for (int k = 0; k < 8; ++k)
			{
				chunk[k] = make_uint4(0u, 0u, 0u, 0u);
			}
		}
		storeRow(x, tid, chunk);

		// Forward, keeping every activation.
		float prediction[3] = { 0.0f, 0.0f, 0.0f };
		for (int layer = 0; layer < 5 && t.ok; ++layer)
		{
			handOff();
			const uint8_t* input = layer == 0 ? x : hidden[layer - 1];
			if (tid == 0)
			{
				issueLayer(t.tmem, input, weights + layer * kWeightLayerBytes, layer < 4 ? 64 : 16);
			}
			completeMmas(t);
			if (!t.ok)
			{
				break;
			}
			if (layer < 4)
			{
				for (int q = 0; q < 4; ++q)
				{
					float v[16];
					umma::tmemLoad16(t.tmem + laneBase + uint32_t(16 * q), v);
					uint4 relu[2];
					reluChunks(v, relu);
					*reinterpret_cast<uint4*>(hidden[layer] + umma::coreOffset(uint32_t(tid), uint32_t(16 * q), 64u)) = relu[0];
					*reinterpret_cast<uint4*>(hidden[layer] + umma::coreOffset(uint32_t(tid), uint32_t(16 * q + 8), 64u)) = relu[1];
				}
			}
			else
			{
				float v[16];
				umma::tmemLoad16(t.tmem + laneBase, v);
				prediction[0] = v[0];
				prediction[1] = v[1];
				prediction[2] = v[2];
			}
		}
		if (!t.ok)
		{
			break;
		}

		// Relative L2 loss and its gradient (scaled), 16 columns of which 3 used.
		uint16_t g[16];
		for (int i = 0; i < 16; ++i)
		{
			g[i] = 0;
		}
		if (valid)
		{
			const float4 target = __ldg(a.targets + row);
			const float tv[3] = { target.x, target.y, target.z };
			const float weight = target.w;
			for (int ch = 0; ch < 3; ++ch)
			{
				const float y = prediction[ch];
				const float denominator = y * y + 0.01f;
				const float difference = y - tv[ch];
				lossSum = lossSum + weight * (difference * difference / denominator);
				g[ch] = rn_float_to_bf16(difference / denominator * gradientScale * lossScale * weight);
			}
		}
		for (int k = 0; k < 2; ++k)
		{
			*reinterpret_cast<uint4*>(dOut + umma::coreOffset(uint32_t(tid), uint32_t(8 * k), 16u)) = make_uint4(
				uint32_t(g[8 * k]) | (uint32_t(g[8 * k + 1]) << 16), uint32_t(g[8 * k + 2]) | (uint32_t(g[8 * k + 3]) << 16),
				uint32_t(g[8 * k + 4]) | (uint32_t(g[8 * k + 5]) << 16), uint32_t(g[8 * k + 6]) | (uint32_t(g[8 * k + 7]) << 16));
		}

		// Backward, layer 4 down to the input.
		for (int layer = 4; layer >= 0 && t.ok; --layer)
		{
			handOff();
			const uint8_t* gradient = layer == 4 ? dOut : dZ;  // dZ of this layer's outputs
			const int outputs = layer == 4 ? 16 : 64;
			const uint8_t* input = layer == 0 ? x : hidden[layer - 1];
			if (tid == 0)
			{
				// dW[layer] += dZ^T X over the tile's 128 rows.
				const uint32_t dW = t.tmem + 64u * uint32_t(layer + 1);
				for (int s = 0; s < 8; ++s)
				{
					umma::mma(dW, mnMajor(gradient, s, outputs), mnMajor(input, s, 64), instrWeights, !(first && s == 0));
				}
				// dX = dZ W[layer]: W read transposed (its outputs are the reduction).
				const uint8_t* w = weights + layer * kWeightLayerBytes;
				for (int s = 0; s < outputs / 16; ++s)
				{
					umma::mma(t.tmem, kMajor(gradient, s, outputs), mnMajor(w, s, 64), instrBackward, s > 0);
				}
			}
			completeMmas(t);
			if (!t.ok)
			{
				break;
			}
			if (layer > 0)
			{
				// dZ of the layer below: dX times the ReLU's derivative.
				const uint8_t* h = hidden[layer - 1];
				for (int q = 0; q < 4; ++q)
				{
					float v[16];
					umma::tmemLoad16(t.tmem + laneBase + uint32_t(16 * q), v);
					uint16_t d[16];
					for (int i = 0; i < 16; ++i)
					{
						// The ReLU passed a positive value (bfloat16 bits nonzero, sign clear).
						const uint16_t bits = rowElement(h, tid, 16 * q + i, 64);
						const bool active = bits != 0 && (bits & 0x8000u) == 0;
						d[i] = active ? rn_float_to_bf16(v[i]) : uint16_t(0);
					}
					for (int k = 0; k < 2; ++k)
					{
						*reinterpret_cast<uint4*>(dZ + umma::coreOffset(uint32_t(tid), uint32_t(16 * q + 8 * k), 64u)) = make_uint4(
							uint32_t(d[8 * k]) | (uint32_t(d[8 * k + 1]) << 16), uint32_t(d[8 * k + 2]) | (uint32_t(d[8 * k + 3]) << 16),
							uint32_t(d[8 * k + 4]) | (uint32_t(d[8 * k + 5]) << 16), uint32_t(d[8 * k + 6]) | (uint32_t(d[8 * k + 7]) << 16));
					}
				}
			}
			else
			{
				// The encoding's gradient, scattered onto the hash table (the
				// TMEM loads are warp-wide, the scatter per valid row).
				float dx[32];
				umma::tmemLoad16(t.tmem + laneBase, dx);
				umma::tmemLoad16(t.tmem + laneBase + 16u, dx + 16);
				if (!valid)
				{
					continue;
				}
				float unit[3];
				unitPosition(a.c, a.queries[size_t(row) * 4], unit);
				bool overflow = false;
				for (int level = 0; level < RESTIR_CACHE_LEVELS; ++level)
				{
					LevelCorners corners;
					levelCorners(a.c, level, unit, corners);
					unsigned long long* grad = a.tableGradFixed + (size_t(level) * a.c.entries) * 2;
					for (int d = 0; d < 8; ++d)
					{
						scatterFixed(grad + size_t(corners.index[d]) * 2, corners.weight[d] * dx[2 * level], overflow);
						scatterFixed(grad + size_t(corners.index[d]) * 2 + 1, corners.weight[d] * dx[2 * level + 1],
							overflow);
					}
				}
				if (overflow)
				{
					atomicOr(a.nonfinite, 1u);
				}
			}
		}
		first = false;
	}

	// This block's weight gradients (rows 0-63 of each dW accumulator live in
	// the lanes of warps 0 and 1) and loss sum.
	umma::fenceBeforeSync();
	__syncthreads();
	umma::fenceAfterSync();
	float* partial = a.partials + size_t(blockIdx.x) * RESTIR_CACHE_PARTIAL_STRIDE;
	if (warp < 2)
	{
		for (int layer = 0; layer < 5; ++layer)
		{
			const int outputs = layer < 4 ? 64 : 16;
			for (int q = 0; q < 4; ++q)
			{
				float v[16];
				umma::tmemLoad16(t.tmem + laneBase + 64u * uint32_t(layer + 1) + uint32_t(16 * q), v);
				if (tid < outputs)
				{
					for (int i = 0; i < 16; ++i)
					{
						partial[weightOffset(layer) + tid * 64 + 16 * q + i] = (first || !t.ok) ? 0.0f : v[i];
					}
				}
			}
		}
	}
	// Loss: a fixed-order sum over the block.
	for (int offset = 16; offset > 0; offset >>= 1)
	{
		lossSum += __shfl_down_sync(0xffffffffu, lossSum, offset);
	}
	if ((tid & 31) == 0)
	{
		lossWarp[warp] = lossSum;
	}
	umma::fenceBeforeSync();
	__syncthreads();
	if (tid == 0)
	{
		partial[RESTIR_CACHE_WEIGHTS] = ((lossWarp[0] + lossWarp[1]) + lossWarp[2]) + lossWarp[3];
	}
	if (warp == 0)
	{
		umma::fenceAfterSync();
		umma::tmemFree(t.tmem, kTrainColumns);
	}
}

// --- reduction and Adam -------------------------------------------------------------------

struct StepArgs
{
	float* weights;
	uint16_t* weightsBf16;
	float* weightM;
	float* weightV;
	float* weightGrad;
	const float* partials;
	float* table;
	uint16_t* tableHalf;
	float* tableM;
	float* tableV;
	float* tableGrad;
	unsigned long long* tableGradFixed;
	RestirCacheScalars* scalars;
	uint32_t tableCount;
	float learningRate, beta1, beta2, epsilon;
};

__device__ __forceinline__ bool finite(float x)
{
	return (rn_float_bits(x) & 0x7f800000u) != 0x7f800000u;
}

// Weight gradients: the blocks' partial rows summed in block order, unscaled;
// the table gradient converted from its fixed-point sum and unscaled; the
// non-finite flag; the mean loss.
__global__ void reduceKernel(StepArgs s, uint32_t blocks, uint32_t samples)
{
	const float inverseScale = 1.0f / s.scalars->loss_scale;
	bool bad = false;
	const uint32_t stride = gridDim.x * blockDim.x;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < RESTIR_CACHE_WEIGHTS + s.tableCount; i += stride)
	{
		if (i < RESTIR_CACHE_WEIGHTS)
		{
			float sum = 0.0f;
			for (uint32_t b = 0; b < blocks; ++b)
			{
				sum = sum + s.partials[size_t(b) * RESTIR_CACHE_PARTIAL_STRIDE + i];
			}
			const float g = sum * inverseScale;
			s.weightGrad[i] = g;
			bad = bad || !finite(g);
		}
		else
		{
			const uint32_t j = i - RESTIR_CACHE_WEIGHTS;
			const long long fixed = static_cast<long long>(s.tableGradFixed[j]);
			const float g = float(double(fixed) * (1.0 / double(kGradientFixedScale))) * inverseScale;
			s.tableGrad[j] = g;
			bad = bad || !finite(g);
		}
	}
	if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31u) == 0u)
	{
		atomicOr(&s.scalars->nonfinite, 1u);
	}
	if (blockIdx.x == 0 && threadIdx.x == 0)
	{
		float loss = 0.0f;
		for (uint32_t b = 0; b < blocks; ++b)
		{
			loss = loss + s.partials[size_t(b) * RESTIR_CACHE_PARTIAL_STRIDE + RESTIR_CACHE_WEIGHTS];
		}
		s.scalars->loss = samples > 0 ? loss / (3.0f * float(samples)) : 0.0f;
		s.scalars->samples = samples;
		s.scalars->blocks = blocks;
	}
}

// Step bookkeeping before the update: the running powers of beta1, beta2.
__global__ void adamBeginKernel(StepArgs s)
{
	RestirCacheScalars* c = s.scalars;
	if (c->nonfinite == 0u)
	{
		c->step += 1u;
		c->beta1_power = c->beta1_power * s.beta1;
		c->beta2_power = c->beta2_power * s.beta2;
	}
}

__device__ __forceinline__ float adamUpdate(float w, float g, float& m, float& v, float lr, float b1, float b2, float eps,
	float correction1, float correction2)
{
	m = b1 * m + (1.0f - b1) * g;
	v = b2 * v + (1.0f - b2) * (g * g);
	const float mHat = m / correction1;
	const float vHat = v / correction2;
	return w - lr * mHat / (sqrtf(vHat) + eps);
}

__global__ void adamKernel(StepArgs s)
{
	const RestirCacheScalars* c = s.scalars;
	if (c->nonfinite != 0u)
	{
		return;
	}
	const float correction1 = 1.0f - c->beta1_power;
	const float correction2 = 1.0f - c->beta2_power;
	const uint32_t stride = gridDim.x * blockDim.x;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < RESTIR_CACHE_WEIGHTS + s.tableCount; i += stride)
	{
		if (i < RESTIR_CACHE_WEIGHTS)
		{
			// The padding rows of the output layer (outputs 3-15) stay zero.
			if (i >= uint32_t(weightOffset(4)) + 3u * 64u)
			{
				continue;
			}
			float m = s.weightM[i], v = s.weightV[i];
			const float w = adamUpdate(s.weights[i], s.weightGrad[i], m, v, s.learningRate, s.beta1, s.beta2, s.epsilon,
				correction1, correction2);
			s.weightM[i] = m;
			s.weightV[i] = v;
			s.weights[i] = w;
			s.weightsBf16[i] = rn_float_to_bf16(w);
		}
		else
		{
			const uint32_t j = i - RESTIR_CACHE_WEIGHTS;
			float m = s.tableM[j], v = s.tableV[j];
			const float w = adamUpdate(s.table[j], s.tableGrad[j], m, v, s.learningRate, s.beta1, s.beta2, s.epsilon,
				correction1, correction2);
			s.tableM[j] = m;
			s.tableV[j] = v;
			s.table[j] = w;
			s.tableHalf[j] = rn_float_to_half(w);
		}
	}
}

// Loss-scale bookkeeping after the update.
__global__ void adamEndKernel(StepArgs s)
{
	RestirCacheScalars* c = s.scalars;
	if (c->nonfinite != 0u)
	{
		c->loss_scale = fmaxf(c->loss_scale * 0.5f, 1.0f);
		c->clean_steps = 0u;
		c->skipped_steps += 1u;
		c->nonfinite = 0u;
		return;
	}
	c->clean_steps += 1u;
	if (c->clean_steps >= 1000u)
	{
		c->loss_scale = fminf(c->loss_scale * 2.0f, 65536.0f);
		c->clean_steps = 0u;
	}
}

__device__ __forceinline__ float uniformSigned(uint32_t seed, uint32_t i)
{
	const uint32_t h = pcg(seed ^ pcg(i));
	return float(h >> 8) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
}

__global__ void initKernel(StepArgs s, uint32_t seed, float initialLossScale)
{
	const uint32_t stride = gridDim.x * blockDim.x;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < RESTIR_CACHE_WEIGHTS + s.tableCount; i += stride)
	{
		if (i < RESTIR_CACHE_WEIGHTS)
		{
			const bool output = i >= uint32_t(weightOffset(4));
			const float bound = output ? 0.29924947f : 0.21650635f;  // sqrt(6 / (64 + 3)), sqrt(6 / 128)
			float w = uniformSigned(seed, i) * bound;
			if (output && i >= uint32_t(weightOffset(4)) + 3u * 64u)
			{
				w = 0.0f;
			}
			s.weights[i] = w;
			s.weightsBf16[i] = rn_float_to_bf16(w);
			s.weightM[i] = 0.0f;
			s.weightV[i] = 0.0f;
			s.weightGrad[i] = 0.0f;
		}
		else
		{
			const uint32_t j = i - RESTIR_CACHE_WEIGHTS;
			const float w = uniformSigned(seed ^ 0x9e3779b9u, j) * 1e-4f;
			s.table[j] = w;
			s.tableHalf[j] = rn_float_to_half(w);
			s.tableM[j] = 0.0f;
			s.tableV[j] = 0.0f;
			s.tableGrad[j] = 0.0f;
			s.tableGradFixed[j] = 0ull;
		}
	}
	if (blockIdx.x == 0 && threadIdx.x == 0)
	{
		RestirCacheScalars c = {};
		c.loss_scale = initialLossScale;
		c.beta1_power = 1.0f;
		c.beta2_power = 1.0f;
		*s.scalars = c;
	}
}

StepArgs stepArgs(const RestirCacheConfig& cfg, const RestirCacheLayout& l, void* state)
{
	char* base = static_cast<char*>(state);
	StepArgs s;
	s.weights = reinterpret_cast<float*>(base + l.weights);
	s.weightsBf16 = reinterpret_cast<uint16_t*>(base + l.weights_bf16);
	s.weightM = reinterpret_cast<float*>(base + l.weight_m);
	s.weightV = reinterpret_cast<float*>(base + l.weight_v);
	s.weightGrad = reinterpret_cast<float*>(base + l.weight_grad);
	s.partials = reinterpret_cast<const float*>(base + l.weight_partials);
	s.table = reinterpret_cast<float*>(base + l.table);
	s.tableHalf = reinterpret_cast<uint16_t*>(base + l.table_half);
	s.tableM = reinterpret_cast<float*>(base + l.table_m);
	s.tableV = reinterpret_cast<float*>(base + l.table_v);
	s.tableGrad = reinterpret_cast<float*>(base + l.table_grad);
	s.tableGradFixed = reinterpret_cast<unsigned long long*>(base + l.table_grad_fixed);
	s.scalars = reinterpret_cast<RestirCacheScalars*>(base + l.scalars);
	s.tableCount = uint32_t(RESTIR_CACHE_LEVELS) * l.entries * RESTIR_CACHE_FEATURES;
	s.learningRate = cfg.learning_rate;
	s.beta1 = cfg.beta1;
	s.beta2 = cfg.beta2;
	s.epsilon = cfg.epsilon;
	return s;
}

int smCount()
{
	static int sms = 0;
	if (sms == 0)
	{
		int device = 0;
		sms = 148;
		if (cudaGetDevice(&device) == cudaSuccess)
		{
			cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
		}
	}
	return sms;
}

bool prepare(const RestirCacheConfig* cfg, const void* state, RestirCacheLayout& l)
{
	return cfg != nullptr && state != nullptr && (reinterpret_cast<uintptr_t>(state) & 255u) == 0u
		&& restir_cache_layout(cfg, &l) == RESTIR_OK;
}

template<int kMode, int kGroups>
void launchForwardShape(const CacheView& view, const float4* queries, uint32_t n, void* output, void* stream)
{
	using Shape = ForwardShape<kGroups>;
	static bool configured = false;
	if (!configured)
	{
		cudaFuncSetAttribute(forwardKernel<kMode, kGroups>, cudaFuncAttributeMaxDynamicSharedMemorySize, Shape::smem);
		configured = true;
	}
	const uint32_t tiles = (n + kTile - 1) / kTile;
	// At most the blocks that fit on the SMs at once (shared memory, registers
	// and TMEM: blocksPerSm x columns <= 512); each loops over tiles.
	const uint32_t blocks = min((tiles + kGroups - 1) / kGroups, uint32_t(smCount() * Shape::blocksPerSm));
	forwardKernel<kMode, kGroups><<<blocks, Shape::threads, Shape::smem, asStream(stream)>>>(view, queries, n, output);
}

template<int kMode>
int launchForward(const RestirCacheConfig* cfg, const void* state, const float* queries, uint32_t n, void* output,
	void* stream)
{
	RestirCacheLayout l;
	if (!prepare(cfg, state, l) || (n > 0u && (queries == nullptr || output == nullptr)))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	if (n == 0u)
	{
		return RESTIR_OK;
	}
	launchForwardShape<kMode, kForwardGroups>(makeView(*cfg, l, state), reinterpret_cast<const float4*>(queries), n, output,
		stream);
	return launchStatus();
}

} // namespace
} // namespace restir

using namespace restir;

extern "C" int restir_cache_init(const RestirCacheConfig* cfg, void* state, void* stream)
{
	RestirCacheLayout l;
	if (!prepare(cfg, state, l))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	StepArgs s = stepArgs(*cfg, l, state);
	cudaStream_t st = asStream(stream);
	cudaMemsetAsync(static_cast<char*>(state) + l.weight_partials, 0,
		size_t(l.partial_blocks) * RESTIR_CACHE_PARTIAL_STRIDE * 4, st);
	initKernel<<<smCount() * 4, 256, 0, st>>>(s, cfg->seed, cfg->initial_loss_scale);
	return launchStatus();
}

extern "C" int restir_cache_query(const RestirCacheConfig* cfg, const void* state, const float* queries, uint32_t n,
	uint16_t* output, void* stream)
{
	return launchForward<0>(cfg, state, queries, n, output, stream);
}

extern "C" int restir_cache_forward(const RestirCacheConfig* cfg, const void* state, const float* queries, uint32_t n,
	float* outputs, void* stream)
{
	return launchForward<1>(cfg, state, queries, n, outputs, stream);
}

extern "C" int restir_cache_features(const RestirCacheConfig* cfg, const void* state, const float* queries, uint32_t n,
	uint16_t* features, void* stream)
{
	return launchForward<2>(cfg, state, queries, n, features, stream);
}

extern "C" int restir_cache_gradients(const RestirCacheConfig* cfg, void* state, const float* queries, const float* targets,
	uint32_t n, void* stream)
{
	RestirCacheLayout l;
	if (!prepare(cfg, state, l) || n > RESTIR_CACHE_MAX_BATCH || (n > 0u && (queries == nullptr || targets == nullptr)))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	StepArgs s = stepArgs(*cfg, l, state);
	cudaStream_t st = asStream(stream);
	cudaMemsetAsync(s.tableGradFixed, 0, size_t(s.tableCount) * 8, st);
	const uint32_t tiles = (n + kTile - 1) / kTile;
	const uint32_t blocks = n == 0u ? 0u : min(tiles, min(uint32_t(smCount()), l.partial_blocks));
	if (blocks > 0u)
	{
		static bool configured = false;
		if (!configured)
		{
			cudaFuncSetAttribute(trainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
			configured = true;
		}
		TrainArgs a;
		a.c = makeView(*cfg, l, state);
		a.queries = reinterpret_cast<const float4*>(queries);
		a.targets = reinterpret_cast<const float4*>(targets);
		a.n = n;
		a.scalars = reinterpret_cast<const float*>(s.scalars);
		a.partials = reinterpret_cast<float*>(static_cast<char*>(state) + l.weight_partials);
		a.tableGradFixed = s.tableGradFixed;
		a.nonfinite = &s.scalars->nonfinite;
		trainKernel<<<blocks, kTile, kTrainSmem, st>>>(a);
	}
	reduceKernel<<<smCount() * 4, 256, 0, st>>>(s, blocks, n);
	return launchStatus();
}

extern "C" int restir_cache_adam(const RestirCacheConfig* cfg, void* state, void* stream)
{
	RestirCacheLayout l;
	if (!prepare(cfg, state, l))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	StepArgs s = stepArgs(*cfg, l, state);
	cudaStream_t st = asStream(stream);
	adamBeginKernel<<<1, 1, 0, st>>>(s);
	adamKernel<<<smCount() * 4, 256, 0, st>>>(s);
	adamEndKernel<<<1, 1, 0, st>>>(s);
	return launchStatus();
}

extern "C" int restir_cache_train(const RestirCacheConfig* cfg, void* state, const float* queries, const float* targets,
	uint32_t n, void* stream)
{
	const int status = restir_cache_gradients(cfg, state, queries, targets, n, stream);
	return status != RESTIR_OK ? status : restir_cache_adam(cfg, state, stream);
}

// A check of the tensor-core steps' bounded wait, no counterpart in the
// reference: one block waits, as completeMmas does, on an mbarrier that no
// one arrives at, for at most `polls` polls; the wait gives up, raises status
// bit 3 and the kernel returns. result (device): 0 when the wait gave up.
extern "C" int restir_cache_wait_check(uint32_t polls, uint32_t* result, void* stream)
{
	if (result == nullptr || polls == 0u || polls > kWaitPolls)
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	waitCheckKernel<<<1, 128, 0, asStream(stream)>>>(polls, result);
	return launchStatus();
}
