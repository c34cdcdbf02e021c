// The ReSTIR DI light list (layout of src/lights.h:5-17): emissive
// triangles, then extra point lights scattered through the middle 80% of the
// scene bounds in saturated colours, selected in proportion to their power
// (Lambertian triangle: pi * luminance * area; point light: 4 pi *
// luminance). The steps follow src/lights.cpp:40-119 so that the same scene
// gets the same list: the same seeded PCG stream for the extra lights, the
// same hue ramp, and a CDF accumulated in double precision whose last entry
// is exactly 1.
#include "bvh_build.h"

#include <cmath>

namespace restir
{
namespace
{

float luminance3(const float* c)
{
	return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
}

void hue(float h, float* rgb)
{
	for (int channel = 0; channel < 3; ++channel)
	{
		const float k = std::fmod(h * 6.0f + float(4 - 2 * channel) + 6.0f, 6.0f);
		rgb[channel] = 1.0f - std::fmax(0.0f, std::fmin(std::fmin(k, 4.0f - k), 1.0f)) * 0.8f;
	}
}

} // namespace

LightListResult buildLightList(const std::vector<Emitter>& emitters, int extraCount, float extraIntensity,
	uint32_t extraSeed, const float* boundsMin, const float* boundsMax, float intensityScale)
{
	LightListResult list;
	std::vector<float> power;
	auto append = [&](const float* v0, const float* v1, const float* v2, float type, float triangle,
		const float* emission, float p)
	{
		const float values[16] = {
			v0[0], v0[1], v0[2], type,
			v1[0], v1[1], v1[2], triangle,
			v2[0], v2[1], v2[2], 0.0f,
			emission[0], emission[1], emission[2], 0.0f,
		};
		list.data.insert(list.data.end(), values, values + 16);
		power.push_back(p);
	};
	for (const Emitter& e : emitters)
	{
		const float* a = e.vertices;
		const float* b = e.vertices + 3;
		const float* c = e.vertices + 6;
		const float ab[3] = { b[0] - a[0], b[1] - a[1], b[2] - a[2] };
		const float ac[3] = { c[0] - a[0], c[1] - a[1], c[2] - a[2] };
		const float n[3] = { ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0] };
		const float area = 0.5f * std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
		if (area <= 0.0f)
		{
			continue;
		}
		append(a, b, c, 0.0f, float(e.triangle), e.emission, 3.1415926535897932384626433832795f * luminance3(e.emission) * area);
	}
	list.triangles = uint32_t(power.size());
	Random random(extraSeed);
	for (int idx = 0; idx < extraCount; ++idx)
	{
		float position[3];
		for (int axis = 0; axis < 3; ++axis)
		{
			position[axis] = boundsMin[axis] + (boundsMax[axis] - boundsMin[axis]) * (0.1f + 0.8f * random.next());
		}
		float intensity[3];
		hue(random.next(), intensity);
		for (float& channel : intensity)
		{
			channel *= extraIntensity * intensityScale;
		}
		const float none[3] = { 0.0f, 0.0f, 0.0f };
		append(position, none, none, 1.0f, -1.0f, intensity, 4.0f * 3.1415926535897932384626433832795f * luminance3(intensity));
	}
	list.count = uint32_t(power.size());
	double total = 0.0;
	for (float p : power)
	{
		total += p;
	}
	double cumulative = 0.0;
	for (uint32_t idx = 0; idx < list.count; ++idx)
	{
		const double pmf = total > 0.0 ? power[idx] / total : 1.0 / double(list.count);
		cumulative += pmf;
		list.data[idx * 16 + 11] = idx + 1 == list.count ? 1.0f : float(cumulative);
		list.data[idx * 16 + 15] = float(pmf);
	}
	return list;
}

} // namespace restir
