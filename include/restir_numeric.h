/*
 * Numeric conventions of the restir-b200 ABI.
 *
 * The reference's passes are shader code whose transcendental functions,
 * texture encodings and rounding are left to each graphics backend. This
 * library fixes them, so that its CUDA kernels and a CPU restatement of the
 * same passes agree bit for bit:
 *
 *   - Every float operation is a single IEEE-754 binary32 operation rounded
 *     to nearest even. No multiply-add is contracted (kernels are compiled
 *     with --fmad=false, host code with -ffp-contract=off), division and
 *     square root are correctly rounded, denormals are kept.
 *   - Unorm8 targets (the reference's BGRA8 G-buffer, renderer.cpp:1363-1366)
 *     store round(clamp(x, 0, 1) * 255) and read back u / 255.
 *   - Half targets (the reference's RGBA16F, renderer.cpp:1385-1422) store
 *     IEEE binary16 rounded to nearest even.
 *   - sin, cos and exp are evaluated by the functions below (Cody-Waite
 *     argument reduction and Taylor polynomials, no table), floor(log2(x)) is
 *     read from the exponent field, and exp2 of an integer is built from it.
 *     The reference calls GLSL's sin/cos/exp/log2/exp2 (restir.sh:201-212,
 *     hashgrid.sh:82-87, svgf.sh:26-36, fs_svgf_atrous.sc:373), whose
 *     precision GLSL does not specify.
 *
 * Everything here is header-only and compiles both as host C/C++ and as CUDA
 * device code.
 */
#ifndef RESTIR_NUMERIC_H
#define RESTIR_NUMERIC_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#	define RN_HD __host__ __device__ __forceinline__
#else
#	define RN_HD static inline
#endif

#ifdef __cplusplus
extern "C++" {
#endif

RN_HD uint32_t rn_float_bits(float x)
{
#if defined(__CUDA_ARCH__)
	return __float_as_uint(x);
#else
	uint32_t u;
	memcpy(&u, &x, 4);
	return u;
#endif
}

RN_HD float rn_bits_float(uint32_t u)
{
#if defined(__CUDA_ARCH__)
	return __uint_as_float(u);
#else
	float x;
	memcpy(&x, &u, 4);
	return x;
#endif
}

/* 2^n as a float, for -126 <= n <= 127 (exact). */
RN_HD float rn_exp2i(int n)
{
	return rn_bits_float((uint32_t)(n + 127) << 23);
}

/* floor(log2(x)) for a finite, normal, positive x: its unbiased exponent. */
RN_HD int rn_floor_log2(float x)
{
	return (int)((rn_float_bits(x) >> 23) & 0xffu) - 127;
}

/* Round to nearest integer value, ties away from zero, for |x| < 2^22. */
RN_HD float rn_round(float x)
{
	float t = x < 0.0f ? -x : x;
	float r = (float)(int)(t + 0.5f);
	return x < 0.0f ? -r : r;
}

/* pi / 2 split into three floats (Cody and Waite): the first two have few
 * significant bits, so k times them is exact for |k| < 2^15. */
#define RN_PIO2_HI 1.5703125f
#define RN_PIO2_MID 4.837512969970703125e-04f
#define RN_PIO2_LO 7.549790126404332e-08f
#define RN_TWO_OVER_PI 6.3661977236758134308e-01f

/* sin and cos of x, both, for |x| < 2^15. Cody-Waite reduction to
 * [-pi/4, pi/4], then the Taylor series of sin to x^11 and cos to x^12. */
RN_HD void rn_sincos(float x, float* s, float* c)
{
	float k = rn_round(x * RN_TWO_OVER_PI);
	float r = x - k * RN_PIO2_HI;
	r = r - k * RN_PIO2_MID;
	r = r - k * RN_PIO2_LO;
	float r2 = r * r;
	/* sin: r - r^3/3! + r^5/5! - r^7/7! + r^9/9! - r^11/11! */
	float ps = -2.5052108385441718775e-08f;
	ps = ps * r2 + 2.7557319223985890653e-06f;
	ps = ps * r2 + -1.9841269841269841253e-04f;
	ps = ps * r2 + 8.3333333333333332177e-03f;
	ps = ps * r2 + -1.6666666666666665741e-01f;
	float sr = r + (r * r2) * ps;
	/* cos: 1 - r^2/2! + r^4/4! - r^6/6! + r^8/8! - r^10/10! + r^12/12! */
	float pc = 2.0876756987868098979e-09f;
	pc = pc * r2 + -2.7557319223985888276e-07f;
	pc = pc * r2 + 2.4801587301587301566e-05f;
	pc = pc * r2 + -1.3888888888888889419e-03f;
	pc = pc * r2 + 4.1666666666666664354e-02f;
	pc = pc * r2 + -0.5f;
	float cr = 1.0f + r2 * pc;
	int q = ((int)k) & 3;
	float sv = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
	float cv = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
	*s = sv;
	*c = cv;
}

RN_HD float rn_sin(float x)
{
	float s, c;
	rn_sincos(x, &s, &c);
	return s;
}

RN_HD float rn_cos(float x)
{
	float s, c;
	rn_sincos(x, &s, &c);
	return c;
}

/* ln 2 split the same way: k times the first part is exact for |k| < 2^9. */
#define RN_LN2_HI 6.93145751953125e-01f
#define RN_LN2_LO 1.428606765330187e-06f
#define RN_LOG2E 1.44269504088896338700e+00f

/* e^x. Reduction x = k ln2 + r with |r| <= ln2/2, Taylor series of e^r to
 * r^8, then scaling by 2^k in two exact steps (one rounding into the
 * denormal range). */
RN_HD float rn_exp(float x)
{
	if (x != x)
	{
		return x;
	}
	if (x > 88.72283935546875f)
	{
		return rn_bits_float(0x7f800000u);
	}
	if (x < -103.97208f)
	{
		return 0.0f;
	}
	float k = rn_round(x * RN_LOG2E);
	float r = x - k * RN_LN2_HI;
	r = r - k * RN_LN2_LO;
	float p = 2.4801587301587302e-05f;       /* 1/8! */
	p = p * r + 1.9841269841269841e-04f;     /* 1/7! */
	p = p * r + 1.3888888888888889e-03f;     /* 1/6! */
	p = p * r + 8.3333333333333332e-03f;     /* 1/5! */
	p = p * r + 4.1666666666666664e-02f;     /* 1/4! */
	p = p * r + 1.6666666666666666e-01f;     /* 1/3! */
	p = p * r + 0.5f;
	p = p * r + 1.0f;
	p = p * r + 1.0f;
	int n = (int)k;
	int n1 = n / 2;
	int n2 = n - n1;
	return (p * rn_exp2i(n1)) * rn_exp2i(n2);
}

#define RN_LN2 6.93147180559945309417e-01f
#define RN_TWO_OVER_LN2 2.88539008177792681472e+00f

/* log2(x). x = m * 2^e with m in [sqrt(1/2), sqrt(2)), then
 * log2(m) = (2 / ln 2) * atanh(s), s = (m - 1) / (m + 1), by the series
 * atanh(s) = s + s^3/3 + ... + s^11/11 (|s| <= 0.172). Zero gives -infinity,
 * a negative x or NaN gives NaN, +infinity itself. */
RN_HD float rn_log2(float x)
{
	if (!(x > 0.0f))
	{
		return x == 0.0f ? rn_bits_float(0xff800000u) : rn_bits_float(0x7fc00000u);
	}
	uint32_t bits = rn_float_bits(x);
	if (bits >= 0x7f800000u)
	{
		return x;
	}
	int e = 0;
	if (bits < 0x00800000u)
	{
		/* Denormal: scale by 2^23 into the normal range. */
		bits = rn_float_bits(x * 8388608.0f);
		e = -23;
	}
	e += (int)(bits >> 23) - 127;
	float m = rn_bits_float((bits & 0x007fffffu) | 0x3f800000u);
	if (m >= 1.41421356237309504880f)
	{
		m = m * 0.5f;
		e += 1;
	}
	float s = (m - 1.0f) / (m + 1.0f);
	float s2 = s * s;
	float p = 9.0909090909090909e-02f;   /* 1/11 */
	p = p * s2 + 1.1111111111111111e-01f; /* 1/9 */
	p = p * s2 + 1.4285714285714285e-01f; /* 1/7 */
	p = p * s2 + 2.0000000000000001e-01f; /* 1/5 */
	p = p * s2 + 3.3333333333333331e-01f; /* 1/3 */
	p = p * s2 + 1.0f;
	return (float)e + (s * p) * RN_TWO_OVER_LN2;
}

/* 2^x: x = k + r with k = round(x), |r| <= 1/2, 2^r = e^(r ln 2) by rn_exp,
 * then scaling by 2^k in two exact steps as rn_exp does. */
RN_HD float rn_exp2(float x)
{
	if (x != x)
	{
		return x;
	}
	if (x >= 128.0f)
	{
		return rn_bits_float(0x7f800000u);
	}
	if (x < -150.0f)
	{
		return 0.0f;
	}
	float k = rn_round(x);
	float r = x - k;
	int n = (int)k;
	int n1 = n / 2;
	int n2 = n - n1;
	return (rn_exp(r * RN_LN2) * rn_exp2i(n1)) * rn_exp2i(n2);
}

/* x^y for x >= 0 (GLSL's pow, whose result for x < 0 is undefined; callers
 * pass abs(x) or clamped values): 2^(y log2 x), with 0^y = 0 for y > 0. */
RN_HD float rn_pow(float x, float y)
{
	if (x == 0.0f)
	{
		return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : rn_bits_float(0x7f800000u));
	}
	return rn_exp2(y * rn_log2(x));
}

/* x^5 and x^64, by a fixed sequence of products (the reference's pow(x, 5.0)
 * and pow(x, 64.0), brdf.sh:460, svgf.sh:203). */
RN_HD float rn_pow5(float x)
{
	float x2 = x * x;
	return (x2 * x2) * x;
}

RN_HD float rn_pow64(float x)
{
	float y = x * x;
	y = y * y;
	y = y * y;
	y = y * y;
	y = y * y;
	return y * y;
}

/* IEEE binary16 from binary32, rounded to nearest even (NaN stays NaN). */
RN_HD uint16_t rn_float_to_half(float f)
{
	uint32_t x = rn_float_bits(f);
	uint32_t sign = (x >> 16) & 0x8000u;
	uint32_t exp = (x >> 23) & 0xffu;
	uint32_t mant = x & 0x7fffffu;
	if (exp == 0xffu)
	{
		return (uint16_t)(sign | 0x7c00u | (mant ? 0x200u : 0u));
	}
	int e = (int)exp - 127 + 15;
	if (e >= 31)
	{
		return (uint16_t)(sign | 0x7c00u);
	}
	if (e <= 0)
	{
		/* Denormal half (or zero): shift the full mantissa down. */
		if (e < -10)
		{
			return (uint16_t)sign;
		}
		uint32_t m = mant | 0x800000u;
		uint32_t shift = (uint32_t)(14 - e);
		uint32_t half = m >> shift;
		uint32_t rem = m & ((1u << shift) - 1u);
		uint32_t mid = 1u << (shift - 1u);
		if (rem > mid || (rem == mid && (half & 1u)))
		{
			++half;
		}
		return (uint16_t)(sign | half);
	}
	uint32_t half = ((uint32_t)e << 10) | (mant >> 13);
	uint32_t rem = mant & 0x1fffu;
	if (rem > 0x1000u || (rem == 0x1000u && (half & 1u)))
	{
		++half; /* may carry into the exponent, up to infinity: correct */
	}
	return (uint16_t)(sign | half);
}

/* Exact and branch-free (F. Giesen, "half to float done quic", 2012): the
 * exponent and mantissa shifted into binary32 position read as a float
 * 2^-112 times the half's magnitude, denormals included (the product is exact;
 * it needs denormal operands kept, as both builds do). Infinity and NaN keep
 * their mantissa bits under an all-ones exponent. */
RN_HD float rn_half_to_float(uint16_t h)
{
	uint32_t shifted = ((uint32_t)h & 0x7fffu) << 13;
	uint32_t magnitude = rn_float_bits(rn_bits_float(shifted) * 0x1p112f);
	if (((uint32_t)h & 0x7c00u) == 0x7c00u)
	{
		magnitude = shifted | 0x7f800000u;
	}
	return rn_bits_float(magnitude | (((uint32_t)h & 0x8000u) << 16));
}

/* Unorm8 store and load. */
RN_HD uint8_t rn_unorm8(float x)
{
	float c = x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x);
	if (c != c)
	{
		c = 0.0f;
	}
	return (uint8_t)(int)(c * 255.0f + 0.5f);
}

RN_HD float rn_unorm8_to_float(uint8_t u)
{
	return (float)u / 255.0f;
}

/* bfloat16 (the upper half of binary32) from binary32, rounded to nearest
 * even; NaN stays a quiet NaN. Used by the radiance cache's network inputs,
 * weights and activations. */
RN_HD uint16_t rn_float_to_bf16(float f)
{
	uint32_t x = rn_float_bits(f);
	if ((x & 0x7fffffffu) > 0x7f800000u)
	{
		return (uint16_t)((x >> 16) | 0x40u);
	}
	uint32_t rounding = 0x7fffu + ((x >> 16) & 1u);
	return (uint16_t)((x + rounding) >> 16);
}

RN_HD float rn_bf16_to_float(uint16_t b)
{
	return rn_bits_float((uint32_t)b << 16);
}

#ifdef __cplusplus
}
#endif

#endif /* RESTIR_NUMERIC_H */
