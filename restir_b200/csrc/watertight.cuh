// Watertight ray/triangle intersection (Woop, Benthin and Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2(1), 2013): the ray is sheared so that
// it runs along +z, the three edge functions are evaluated in the sheared
// 2D plane (in double precision when one of them is exactly zero), and a hit
// on an edge shared by two triangles is reported by at least one of them.
// The production alternative to the reference's Moeller-Trumbore test
// (bvh.sh:44-71), whose rays can slip through shared edges.
#pragma once

#include "bvh.cuh"

namespace restir
{

struct WatertightRay
{
	int kx, ky, kz;
	float sx, sy, sz;
	V3 o;
};

__device__ __forceinline__ float component(V3 v, int k)
{
	return k == 0 ? v.x : (k == 1 ? v.y : v.z);
}

__device__ __forceinline__ WatertightRay makeWatertightRay(V3 o, V3 d)
{
	WatertightRay r;
	V3 a = vabs(d);
	int kz = a.x > a.y ? (a.x > a.z ? 0 : 2) : (a.y > a.z ? 1 : 2);
	int kx = kz + 1 == 3 ? 0 : kz + 1;
	int ky = kx + 1 == 3 ? 0 : kx + 1;
	if (component(d, kz) < 0.0f)
	{
		int t = kx;
		kx = ky;
		ky = t;
	}
	r.kx = kx;
	r.ky = ky;
	r.kz = kz;
	r.sx = component(d, kx) / component(d, kz);
	r.sy = component(d, ky) / component(d, kz);
	r.sz = 1.0f / component(d, kz);
	r.o = o;
	return r;
}

// Distance to the triangle, or -1; hits must lie in (0, tmax].
__device__ __forceinline__ float intersectWatertight(const WatertightRay& r, V3 v0, V3 v1, V3 v2, float tmax)
{
	V3 A = v0 - r.o;
	V3 B = v1 - r.o;
	V3 C = v2 - r.o;
	float az = component(A, r.kz), bz = component(B, r.kz), cz = component(C, r.kz);
	float ax = component(A, r.kx) - r.sx * az;
	float ay = component(A, r.ky) - r.sy * az;
	float bx = component(B, r.kx) - r.sx * bz;
	float by = component(B, r.ky) - r.sy * bz;
	float cx = component(C, r.kx) - r.sx * cz;
	float cy = component(C, r.ky) - r.sy * cz;
	float u = cx * by - cy * bx;
	float v = ax * cy - ay * cx;
	float w = bx * ay - by * ax;
	if (u == 0.0f || v == 0.0f || w == 0.0f)
	{
		u = float(double(cx) * double(by) - double(cy) * double(bx));
		v = float(double(ax) * double(cy) - double(ay) * double(cx));
		w = float(double(bx) * double(ay) - double(by) * double(ax));
	}
	if ((u < 0.0f || v < 0.0f || w < 0.0f) && (u > 0.0f || v > 0.0f || w > 0.0f))
	{
		return -1.0f;
	}
	float det = u + v + w;
	if (det == 0.0f)
	{
		return -1.0f;
	}
	float sz = r.sz;
	float t = u * (sz * az) + v * (sz * bz) + w * (sz * cz);
	float sign = det < 0.0f ? -1.0f : 1.0f;
	float signedT = t * sign;
	float absDet = det * sign;
	if (signedT <= 0.0f || signedT > tmax * absDet)
	{
		return -1.0f;
	}
	return t / det;
}

// Nearest watertight hit in (0, distance], ties to the lower triangle index,
// with conservative box tests.
__device__ inline int traceWatertight(const BvhView& b, V3 o, V3 d, float& distance)
{
	const WatertightRay ray = makeWatertightRay(o, d);
	return traceNearestFirst(b, o, d, distance, true,
		[&](int t, float tmax) { return intersectWatertight(ray, b.vertex(t, 0), b.vertex(t, 1), b.vertex(t, 2), tmax); },
		[](int) { return true; });
}

} // namespace restir
