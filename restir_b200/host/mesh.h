// Host-side scene data: a triangle soup with per-triangle materials, and
// the procedural scenes that stand in for glTF models.
#pragma once

#include "../../include/restir_host.h"

#include <cstdint>
#include <vector>

namespace restir
{

struct Material
{
	float base[3] = { 0.73f, 0.73f, 0.73f };
	float roughness = 1.0f;
	float emission[3] = { 0.0f, 0.0f, 0.0f };
	float metallic = 0.0f;
};

struct Mesh
{
	std::vector<float> positions;      // 9 per triangle
	std::vector<float> normals;        // 3 per triangle
	std::vector<uint32_t> material;    // per triangle
	std::vector<uint8_t> twoSided;     // per triangle
	std::vector<Material> materials;
	float boundsMin[3] = { 0.0f, 0.0f, 0.0f };
	float boundsMax[3] = { 0.0f, 0.0f, 0.0f };
	float center[3] = { 0.0f, 0.0f, 0.0f };
	float radius = 1.0f;
	float lightPosition[3] = { 0.0f, 0.0f, 0.0f };
	float cameraEye[3] = { 0.0f, 0.0f, 0.0f };
	float cameraYaw = 0.0f;
	float cameraPitch = 0.0f;
	bool sky = true;
	std::vector<float> materialData;   // 8 per material, filled by finalize()

	uint32_t triangleCount() const { return uint32_t(material.size()); }
	// Bounds, centre, radius, default light position (scene.cpp:810-834),
	// the flat material array.
	void finalize();
};

Mesh makeCornell();
Mesh makeCourtyard(uint32_t seed, uint32_t targetTriangles);
Mesh makeCity(uint32_t seed, uint32_t targetTriangles, int emissivePanelCount = 128);

// A small deterministic generator (the PCG output function of lights.cpp:15-26).
struct Random
{
	uint32_t state;
	explicit Random(uint32_t seed) : state(seed * 2654435761u + 1u) {}
	uint32_t nextU32()
	{
		state = state * 747796405u + 2891336453u;
		uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
		return (word >> 22u) ^ word;
	}
	float next() { return float(nextU32() >> 8) * (1.0f / 16777216.0f); }
	float range(float lo, float hi) { return lo + (hi - lo) * next(); }
};

} // namespace restir
