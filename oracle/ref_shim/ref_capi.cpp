/*
 * ORACLE (test infrastructure): a C interface over the reference's own BVH
 * builder and light-list builder (pkonecki/restir src/bvh.cpp:253-393,
 * src/lights.cpp:40-119), compiled unmodified from the reference's sources
 * by oracle/Makefile into oracle/_ref/libref_bvh.so. Tests use it as the
 * layout oracle: the node and triangle records and the light CDF come from
 * the reference's code itself.
 */
#include "bvh.h"
#include "lights.h"

#include <cstring>
#include <vector>

namespace
{
SceneBvh g_bvh;
LightList g_lights;
}

bgfx::VertexLayout SceneVertex::ms_layout;

extern "C"
{

/* Builds the reference BVH over triangles (9 floats each), all with one
 * untextured material per triangle: material index, base colour (3 floats),
 * emission (3 floats), metallic. Returns the float count of the buffer. */
uint64_t ref_build_bvh(const float* positions, uint32_t triangleCount, const uint32_t* materialOfTriangle,
	const float* materialBase, const float* materialEmission, const float* materialMetallic, uint32_t materialCount,
	uint32_t* nodeCount, uint32_t* triangleOffset, uint32_t* depth)
{
	SceneMesh mesh;
	mesh.m_vertices.resize(size_t(triangleCount) * 3);
	mesh.m_indices.resize(size_t(triangleCount) * 3);
	for (uint32_t m = 0; m < materialCount; ++m)
	{
		SceneMaterial material;
		material.m_emissive[0] = materialEmission[3 * m + 0];
		material.m_emissive[1] = materialEmission[3 * m + 1];
		material.m_emissive[2] = materialEmission[3 * m + 2];
		mesh.m_materials.push_back(material);
	}
	for (uint32_t t = 0; t < triangleCount; ++t)
	{
		const uint32_t m = materialOfTriangle[t];
		for (int c = 0; c < 3; ++c)
		{
			SceneVertex& v = mesh.m_vertices[size_t(t) * 3 + c];
			std::memset(&v, 0, sizeof(v));
			std::memcpy(v.m_position, positions + size_t(t) * 9 + c * 3, 3 * sizeof(float));
			v.m_color[0] = materialBase[3 * m + 0];
			v.m_color[1] = materialBase[3 * m + 1];
			v.m_color[2] = materialBase[3 * m + 2];
			v.m_material[0] = 1.0f;
			v.m_material[1] = materialMetallic[m];
			mesh.m_indices[size_t(t) * 3 + c] = t * 3 + c;
		}
		SceneDraw draw;
		draw.m_firstIndex = t * 3;
		draw.m_indexCount = 3;
		draw.m_material = m;
		mesh.m_draws.push_back(draw);
	}
	g_bvh = buildBvh(mesh);
	*nodeCount = g_bvh.m_nodeCount;
	*triangleOffset = g_bvh.m_triangleOffset;
	*depth = g_bvh.m_depth;
	return g_bvh.m_data.size();
}

void ref_copy_bvh(float* out)
{
	std::memcpy(out, g_bvh.m_data.data(), g_bvh.m_data.size() * sizeof(float));
}

/* The light list of the last BVH's emitters plus extra point lights. */
uint32_t ref_build_lights(int extraCount, float extraIntensity, uint32_t extraSeed,
	const float* boundsMin, const float* boundsMax, float intensityScale, uint32_t* triangleLights)
{
	ExtraLights extra;
	extra.m_count = extraCount;
	extra.m_intensity = extraIntensity;
	extra.m_seed = extraSeed;
	g_lights = buildLightList(g_bvh.m_emitters, extra,
		bx::Vec3{ boundsMin[0], boundsMin[1], boundsMin[2] },
		bx::Vec3{ boundsMax[0], boundsMax[1], boundsMax[2] }, intensityScale);
	*triangleLights = g_lights.m_triangles;
	return g_lights.m_count;
}

void ref_copy_lights(float* out)
{
	std::memcpy(out, g_lights.m_data.data(), g_lights.m_data.size() * sizeof(float));
}

}
