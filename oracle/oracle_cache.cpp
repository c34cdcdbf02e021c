/*
 * ORACLE (test infrastructure): the radiance cache of include/restir_cache.h
 * restated on the CPU, to check the CUDA kernels.
 *
 * The reference renderer has no cache, so this restates the published
 * algorithms the header names: the multiresolution hash encoding (Mueller,
 * Evans, Schied, Keller 2022, section 3: per-level trilinear interpolation of
 * hashed corner features, hash = XOR of the coordinates times the primes
 * 1, 2654435761, 805459861, dense indexing where a level fits; here applied
 * to 2x2x2 bricks of corners stored together), a ReLU MLP
 * without biases, the relative L2 loss of neural radiance caching (Mueller,
 * Rousselle, Novak, Keller 2021, section 5: (y - t)^2 / (sg(y)^2 + 0.01)),
 * its gradients by backpropagation, and Adam (Kingma and Ba 2015,
 * algorithm 1, with bias correction).
 *
 *   - The encoding is computed in the same binary32 operations as the CUDA
 *     kernel (no contraction), so the network inputs are bit-exact.
 *   - The MLP is evaluated in binary64 on the same bfloat16 weights and
 *     inputs, rounding each hidden activation to bfloat16 where the kernel
 *     does; the kernel accumulates in binary32 on the tensor cores, so
 *     outputs and gradients agree to a tolerance, not bit for bit.
 *   - Adam runs in binary32 in the kernel's order of operations: bit-exact
 *     for the same gradients.
 */
#include "../include/restir_cache.h"
#include "../include/restir_gpu.h"
#include "../include/restir_numeric.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace
{

struct Corners
{
	uint32_t index[8];
	float weight[8];
};

float unitCoordinate(float p, float lo, float hi)
{
	float u = (p - lo) / (hi - lo);
	u = u > 0.0f ? u : 0.0f;
	return u < 1.0f ? u : 1.0f;
}

void corners(const RestirCacheLayout& l, int level, const float unit[3], Corners& out)
{
	const float scale = l.level_scale[level];
	const int resolution = int(scale);
	int cell[3];
	float frac[3];
	for (int a = 0; a < 3; ++a)
	{
		const float g = unit[a] * scale;
		cell[a] = std::min(int(std::floor(g)), resolution - 1);
		frac[a] = g - float(cell[a]);
	}
	const uint32_t bricks = uint32_t(resolution + 2) / 2u;
	for (int d = 0; d < 8; ++d)
	{
		const int bx = d & 1, by = (d >> 1) & 1, bz = d >> 2;
		const uint32_t x = uint32_t(cell[0] + bx), y = uint32_t(cell[1] + by), z = uint32_t(cell[2] + bz);
		const float wx = bx ? frac[0] : 1.0f - frac[0];
		const float wy = by ? frac[1] : 1.0f - frac[1];
		const float wz = bz ? frac[2] : 1.0f - frac[2];
		const float wxy = wx * wy;
		out.weight[d] = wxy * wz;
		// 2x2x2 bricks of 8 consecutive entries (restir_cache.h).
		const uint32_t local = (x % 2u) + 2u * (y % 2u) + 4u * (z % 2u);
		const uint32_t cx = x / 2u, cy = y / 2u, cz = z / 2u;
		const uint32_t brick = l.level_dense[level] ? cx + cy * bricks + cz * bricks * bricks
			: ((cx * 1u) ^ (cy * 2654435761u) ^ (cz * 805459861u)) % (l.entries / 8u);
		out.index[d] = brick * 8u + local;
	}
}

void unitPosition(const RestirCacheConfig& cfg, const float* q, float unit[3])
{
	for (int a = 0; a < 3; ++a)
	{
		unit[a] = unitCoordinate(q[a], cfg.bounds_min[a], cfg.bounds_max[a]);
	}
}

void features(const RestirCacheConfig& cfg, const RestirCacheLayout& l, const uint16_t* tableHalf, const float* q,
	uint16_t* out)
{
	float unit[3];
	unitPosition(cfg, q, unit);
	for (int level = 0; level < RESTIR_CACHE_LEVELS; ++level)
	{
		Corners c;
		corners(l, level, unit, c);
		const uint16_t* row = tableHalf + size_t(level) * l.entries * 2;
		float f0 = 0.0f, f1 = 0.0f;
		for (int d = 0; d < 8; ++d)
		{
			const float p0 = c.weight[d] * rn_half_to_float(row[size_t(c.index[d]) * 2]);
			const float p1 = c.weight[d] * rn_half_to_float(row[size_t(c.index[d]) * 2 + 1]);
			f0 = f0 + p0;
			f1 = f1 + p1;
		}
		out[2 * level] = rn_float_to_bf16(f0);
		out[2 * level + 1] = rn_float_to_bf16(f1);
	}
	// direction, normal, roughness, albedo, constant 1
	const float extra[11] = { q[8], q[9], q[10], q[4], q[5], q[6], q[3], q[12], q[13], q[14], 1.0f };
	for (int i = 0; i < 11; ++i)
	{
		out[32 + i] = rn_float_to_bf16(extra[i]);
	}
	for (int i = 43; i < 64; ++i)
	{
		out[i] = 0;
	}
}

int layerOutputs(int layer)
{
	return layer < 4 ? 64 : 16;
}

double bf(uint16_t b)
{
	return double(rn_bf16_to_float(b));
}

bool positive(uint16_t b)
{
	return b != 0 && (b & 0x8000u) == 0;
}

// Forward through the MLP; acts[l] are the bfloat16 inputs of layer l
// (acts[0] the features), out the 16 outputs.
void forward(const uint16_t* w, const uint16_t* x, uint16_t acts[5][64], double out[16])
{
	std::memcpy(acts[0], x, 64 * sizeof(uint16_t));
	for (int layer = 0; layer < 5; ++layer)
	{
		const uint16_t* wl = w + layer * 64 * 64;
		for (int o = 0; o < layerOutputs(layer); ++o)
		{
			double z = 0.0;
			for (int k = 0; k < 64; ++k)
			{
				z += bf(wl[o * 64 + k]) * bf(acts[layer][k]);
			}
			if (layer < 4)
			{
				const float zf = float(z);
				acts[layer + 1][o] = rn_float_to_bf16(zf > 0.0f ? zf : 0.0f);
			}
			else
			{
				out[o] = z;
			}
		}
	}
}

} // namespace

/* The layout (level resolutions, dense levels, entries) is an input: the
 * configuration the kernels ran with, from restir_cache_layout. */
extern "C" void oracle_cache_features(const RestirCacheConfig* cfg, const RestirCacheLayout* layout,
	const uint16_t* table_half, const float* queries, uint32_t n, uint16_t* out)
{
	const RestirCacheLayout& l = *layout;
	for (uint32_t i = 0; i < n; ++i)
	{
		features(*cfg, l, table_half, queries + size_t(i) * 16, out + size_t(i) * 64);
	}
}

extern "C" void oracle_cache_forward(const uint16_t* weights_bf16, const uint16_t* inputs, uint32_t n, double* outputs)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		uint16_t acts[5][64];
		forward(weights_bf16, inputs + size_t(i) * 64, acts, outputs + size_t(i) * 16);
	}
}

/* Gradients of the mean relative L2 loss over n samples: weight_grad
 * [RESTIR_CACHE_WEIGHTS] and table_grad [levels * entries * features], both
 * unscaled; loss the mean. The output gradient is formed in binary32 from
 * the binary32 prediction, scaled by loss_scale and rounded to bfloat16, as
 * are the hidden-layer gradients, like the kernel. */
extern "C" void oracle_cache_gradients(const RestirCacheConfig* cfg, const RestirCacheLayout* layout,
	const uint16_t* weights_bf16, const uint16_t* table_half, const float* queries, const float* targets, uint32_t n,
	float loss_scale, double* weight_grad, double* table_grad, double* loss)
{
	const RestirCacheLayout& l = *layout;
	const size_t tableCount = size_t(RESTIR_CACHE_LEVELS) * l.entries * RESTIR_CACHE_FEATURES;
	std::fill(weight_grad, weight_grad + RESTIR_CACHE_WEIGHTS, 0.0);
	std::fill(table_grad, table_grad + tableCount, 0.0);
	double lossSum = 0.0;
	const float gradientScale = 2.0f / (3.0f * float(n));
	for (uint32_t i = 0; i < n; ++i)
	{
		const float* q = queries + size_t(i) * 16;
		uint16_t x[64];
		features(*cfg, l, table_half, q, x);
		uint16_t acts[5][64];
		double out[16];
		forward(weights_bf16, x, acts, out);
		// Output gradient (16 wide, 3 used).
		uint16_t dz[64] = {};
		const float weight = targets[size_t(i) * 4 + 3];
		for (int c = 0; c < 3; ++c)
		{
			const float y = float(out[c]);
			const float t = targets[size_t(i) * 4 + c];
			const float denominator = y * y + 0.01f;
			const float difference = y - t;
			const float term = difference * difference / denominator;
			lossSum += double(weight * term);
			dz[c] = rn_float_to_bf16(difference / denominator * gradientScale * loss_scale * weight);
		}
		for (int layer = 4; layer >= 0; --layer)
		{
			const int outputs = layerOutputs(layer);
			const uint16_t* wl = weights_bf16 + layer * 64 * 64;
			double* gl = weight_grad + layer * 64 * 64;
			double dx[64];
			for (int k = 0; k < 64; ++k)
			{
				double s = 0.0;
				for (int o = 0; o < outputs; ++o)
				{
					gl[o * 64 + k] += bf(dz[o]) * bf(acts[layer][k]);
					s += bf(dz[o]) * bf(wl[o * 64 + k]);
				}
				dx[k] = s;
			}
			if (layer > 0)
			{
				for (int k = 0; k < 64; ++k)
				{
					dz[k] = positive(acts[layer][k]) ? rn_float_to_bf16(float(dx[k])) : uint16_t(0);
				}
			}
			else
			{
				float unit[3];
				unitPosition(*cfg, q, unit);
				for (int level = 0; level < RESTIR_CACHE_LEVELS; ++level)
				{
					Corners c;
					corners(l, level, unit, c);
					double* g = table_grad + size_t(level) * l.entries * 2;
					for (int d = 0; d < 8; ++d)
					{
						g[size_t(c.index[d]) * 2] += double(c.weight[d]) * float(dx[2 * level]);
						g[size_t(c.index[d]) * 2 + 1] += double(c.weight[d]) * float(dx[2 * level + 1]);
					}
				}
			}
		}
	}
	for (int i = 0; i < RESTIR_CACHE_WEIGHTS; ++i)
	{
		weight_grad[i] /= double(loss_scale);
	}
	for (size_t i = 0; i < tableCount; ++i)
	{
		table_grad[i] /= double(loss_scale);
	}
	*loss = n > 0 ? lossSum / (3.0 * double(n)) : 0.0;
}

/* One Adam step over count parameters in binary32, the kernel's operations:
 * correction1 = 1 - beta1^t, correction2 = 1 - beta2^t given as powers. */
extern "C" void oracle_cache_adam(const RestirCacheConfig* cfg, uint32_t count, float* w, float* m, float* v,
	const float* g, float beta1_power, float beta2_power)
{
	const float b1 = cfg->beta1, b2 = cfg->beta2, lr = cfg->learning_rate, eps = cfg->epsilon;
	const float correction1 = 1.0f - beta1_power;
	const float correction2 = 1.0f - beta2_power;
	for (uint32_t i = 0; i < count; ++i)
	{
		const float a1 = b1 * m[i];
		const float a2 = (1.0f - b1) * g[i];
		m[i] = a1 + a2;
		const float gg = g[i] * g[i];
		const float c1 = b2 * v[i];
		const float c2 = (1.0f - b2) * gg;
		v[i] = c1 + c2;
		const float mHat = m[i] / correction1;
		const float vHat = v[i] / correction2;
		const float step = lr * mHat;
		w[i] = w[i] - step / (std::sqrt(vHat) + eps);
	}
}
