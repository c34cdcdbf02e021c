// Host side of the radiance cache's C ABI (include/restir_cache.h): the
// default configuration and the state block's layout, including the
// resolution of each hash-grid level.
#include "restir_cache.h"
#include "restir_gpu.h"

#include <cmath>

namespace
{

uint64_t alignUp(uint64_t x)
{
	return (x + 255u) & ~uint64_t(255u);
}

// Rows of per-block weight-gradient partials the training kernel may write
// (one per resident block; 148 SMs on a B200).
constexpr uint32_t kPartialBlocks = 256;

} // namespace

extern "C" void restir_cache_config_default(RestirCacheConfig* cfg)
{
	if (cfg == nullptr)
	{
		return;
	}
	for (int i = 0; i < 3; ++i)
	{
		cfg->bounds_min[i] = 0.0f;
		cfg->bounds_max[i] = 1.0f;
	}
	cfg->table_log2 = 18;
	cfg->n_min = 16.0f;
	cfg->n_max = 2048.0f;
	cfg->learning_rate = 1e-2f;
	cfg->beta1 = 0.9f;
	cfg->beta2 = 0.99f;
	cfg->epsilon = 1e-15f;
	cfg->initial_loss_scale = 128.0f;
	cfg->seed = 1337u;
}

extern "C" int restir_cache_layout(const RestirCacheConfig* cfg, RestirCacheLayout* layout)
{
	if (cfg == nullptr || layout == nullptr || cfg->table_log2 < 12 || cfg->table_log2 > 22 || !(cfg->n_min >= 1.0f)
		|| !(cfg->n_max >= cfg->n_min) || !(cfg->learning_rate > 0.0f) || !(cfg->initial_loss_scale > 0.0f))
	{
		return RESTIR_ERROR_INVALID_ARGUMENT;
	}
	for (int i = 0; i < 3; ++i)
	{
		if (!(cfg->bounds_max[i] > cfg->bounds_min[i]))
		{
			return RESTIR_ERROR_INVALID_ARGUMENT;
		}
	}
	RestirCacheLayout l = {};
	l.entries = 1u << cfg->table_log2;
	l.partial_blocks = kPartialBlocks;
	const uint64_t weights = RESTIR_CACHE_WEIGHTS;
	const uint64_t table = uint64_t(RESTIR_CACHE_LEVELS) * l.entries * RESTIR_CACHE_FEATURES;
	uint64_t at = 0;
	auto take = [&](uint64_t bytes) -> uint64_t
	{
		const uint64_t offset = at;
		at = alignUp(at + bytes);
		return offset;
	};
	l.weights = take(weights * 4);
	l.weights_bf16 = take(weights * 2);
	l.weight_m = take(weights * 4);
	l.weight_v = take(weights * 4);
	l.weight_grad = take(weights * 4);
	l.weight_partials = take(uint64_t(kPartialBlocks) * RESTIR_CACHE_PARTIAL_STRIDE * 4);
	l.table = take(table * 4);
	l.table_half = take(table * 2);
	l.table_m = take(table * 4);
	l.table_v = take(table * 4);
	l.table_grad = take(table * 4);
	l.table_grad_fixed = take(table * 8);
	l.scalars = take(sizeof(RestirCacheScalars));
	l.bytes = at;
	// Level l at floor(n_min * b^l) cells across the box, b the growth factor
	// from n_min to n_max over the levels (computed in double, then exact).
	const double growth = std::exp((std::log(double(cfg->n_max)) - std::log(double(cfg->n_min)))
		/ double(RESTIR_CACHE_LEVELS - 1));
	for (int level = 0; level < RESTIR_CACHE_LEVELS; ++level)
	{
		const double resolution = std::floor(double(cfg->n_min) * std::pow(growth, double(level)) + 1e-9);
		l.level_scale[level] = float(resolution);
		// Dense when the level's 2x2x2 bricks of corners, 8 entries each, fit the table.
		const double bricks = std::floor((resolution + 2.0) / 2.0);
		l.level_dense[level] = 8.0 * bricks * bricks * bricks <= double(l.entries) ? 1u : 0u;
	}
	*layout = l;
	return RESTIR_OK;
}

extern "C" uint64_t restir_cache_state_bytes(const RestirCacheConfig* cfg)
{
	RestirCacheLayout l;
	return restir_cache_layout(cfg, &l) == RESTIR_OK ? l.bytes : 0;
}
