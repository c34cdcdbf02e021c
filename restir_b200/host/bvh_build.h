// Host BVH builder and light list (the reference's src/bvh.cpp and
// src/lights.cpp layouts), and the camera conventions.
#pragma once

#include "mesh.h"

#include <atomic>
#include <cstdint>
#include <vector>

namespace restir
{

// A triangle whose material emits light (bvh.h:28-36).
struct Emitter
{
	uint32_t triangle = 0; // BVH order
	float vertices[9] = {};
	float emission[3] = {};
};

struct BvhResult
{
	std::vector<float> data;            // float4s: nodes, then triangles
	uint32_t nodeCount = 0;
	uint32_t triangleCount = 0;
	uint32_t triangleOffset = 0;        // in float4s
	uint32_t depth = 0;
	std::vector<uint32_t> order;        // BVH slot -> mesh triangle
	std::vector<float> triangleNormals; // float4 per BVH slot
	std::vector<Emitter> emitters;
	std::vector<float> emitterFloats;   // 13 per emitter, for the C ABI
	double buildMs = 0.0;
};

BvhResult buildBvh(const Mesh& mesh, int threads);

// Device copies of a BVH's node and triangle rows and its shading normals
// (cudaMalloc'd; the owner frees them with cudaFree).
struct DeviceBvh
{
	void* rows = nullptr;
	uint64_t rowsBytes = 0;
	void* normals = nullptr;
	uint64_t normalsBytes = 0;
};

// The same BVH built on the current CUDA device (csrc/bvh_build.cu), on a
// cudaStream_t; waits for it. Returns a RESTIR_* status. With device null the
// rows, order and normals are downloaded into result; otherwise they stay on
// the device in *device and result carries the counts and emitters only.
int buildBvhGpu(const Mesh& mesh, void* stream, BvhResult& result, DeviceBvh* device = nullptr);

struct LightListResult
{
	std::vector<float> data; // 16 floats per light
	uint32_t count = 0;
	uint32_t triangles = 0;
};

LightListResult buildLightList(const std::vector<Emitter>& emitters, int extraCount, float extraIntensity,
	uint32_t extraSeed, const float* boundsMin, const float* boundsMax, float intensityScale);

// Row-major 4x4 helpers (clip = M * v).
void lookAtRH(const float* eye, const float* at, const float* up, float* out);
void perspectiveRH(float fovyRadians, float aspect, float nearPlane, float farPlane, float* out);
void multiply(const float* a, const float* b, float* out); // out = a * b
bool invert(const float* m, float* out);                   // in double precision

} // namespace restir
