// Seeded procedural scenes (the benchmark configurations' stand-ins for glTF
// models) and the scene description of scene.cpp:810-834 (describeScene).
#include "mesh.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace restir
{
namespace
{

struct V
{
	float x, y, z;
};

V operator+(V a, V b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
V operator-(V a, V b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
V operator*(V a, float s) { return { a.x * s, a.y * s, a.z * s }; }
float dotv(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V crossv(V a, V b) { return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }
V normalizev(V a)
{
	float l = std::sqrt(dotv(a, a));
	return l > 0.0f ? a * (1.0f / l) : a;
}

class Builder
{
public:
	explicit Builder(Mesh& mesh) : m_mesh(mesh) {}

	uint32_t material(float r, float g, float b, float roughness = 1.0f, float metallic = 0.0f, float er = 0.0f,
		float eg = 0.0f, float eb = 0.0f)
	{
		Material m;
		m.base[0] = r;
		m.base[1] = g;
		m.base[2] = b;
		m.roughness = roughness;
		m.metallic = metallic;
		m.emission[0] = er;
		m.emission[1] = eg;
		m.emission[2] = eb;
		m_mesh.materials.push_back(m);
		return uint32_t(m_mesh.materials.size() - 1);
	}

	// Wound so that the geometric normal agrees with the shading normal.
	void triangle(V a, V b, V c, V normal, uint32_t mat, bool twoSided = false)
	{
		if (dotv(crossv(b - a, c - a), normal) < 0.0f)
		{
			std::swap(b, c);
		}
		const V p[3] = { a, b, c };
		for (const V& q : p)
		{
			m_mesh.positions.push_back(q.x);
			m_mesh.positions.push_back(q.y);
			m_mesh.positions.push_back(q.z);
		}
		V n = normalizev(normal);
		m_mesh.normals.push_back(n.x);
		m_mesh.normals.push_back(n.y);
		m_mesh.normals.push_back(n.z);
		m_mesh.material.push_back(mat);
		m_mesh.twoSided.push_back(twoSided ? 1 : 0);
	}

	// The quad centre +- u +- v, facing normal.
	void quad(V c, V u, V v, V normal, uint32_t mat, bool twoSided = false)
	{
		V p00 = c - u - v, p10 = c + u - v, p11 = c + u + v, p01 = c - u + v;
		triangle(p00, p10, p11, normal, mat, twoSided);
		triangle(p00, p11, p01, normal, mat, twoSided);
	}

	// A box with half extents h, turned by yaw about +y, faces outwards.
	void box(V c, V h, float yaw, uint32_t mat)
	{
		float cs = std::cos(yaw), sn = std::sin(yaw);
		V ax = { cs, 0.0f, -sn }, ay = { 0.0f, 1.0f, 0.0f }, az = { sn, 0.0f, cs };
		V ex = ax * h.x, ey = ay * h.y, ez = az * h.z;
		quad(c + ex, ey, ez, ax, mat);
		quad(c - ex, ey, ez, ax * -1.0f, mat);
		quad(c + ey, ex, ez, ay, mat);
		quad(c - ey, ex, ez, ay * -1.0f, mat);
		quad(c + ez, ex, ey, az, mat);
		quad(c - ez, ex, ey, az * -1.0f, mat);
	}

	// A UV sphere of 16 segments and 17 rings: 512 triangles.
	void sphere(V c, float r, uint32_t mat)
	{
		const int segments = 16, rings = 17;
		auto point = [&](int ring, int segment)
		{
			float theta = float(M_PI) * float(ring) / float(rings);
			float phi = 2.0f * float(M_PI) * float(segment) / float(segments);
			return V{ std::sin(theta) * std::cos(phi), std::cos(theta), std::sin(theta) * std::sin(phi) };
		};
		for (int ring = 0; ring < rings; ++ring)
		{
			for (int segment = 0; segment < segments; ++segment)
			{
				V a = point(ring, segment), b = point(ring + 1, segment);
				V d = point(ring, segment + 1), e = point(ring + 1, segment + 1);
				if (ring != 0)
				{
					V n = normalizev((a + b + d) * (1.0f / 3.0f));
					triangle(c + a * r, c + b * r, c + d * r, n, mat);
				}
				if (ring != rings - 1)
				{
					V n = normalizev((b + e + d) * (1.0f / 3.0f));
					triangle(c + b * r, c + e * r, c + d * r, n, mat);
				}
			}
		}
	}

	// A semicircular arch of boxes over the x axis, of the given span.
	void arch(V c, float span, float thickness, float yaw, uint32_t mat, int pieces)
	{
		float cs = std::cos(yaw), sn = std::sin(yaw);
		float radius = 0.5f * span;
		for (int k = 0; k < pieces; ++k)
		{
			float a = float(M_PI) * (float(k) + 0.5f) / float(pieces);
			float lx = radius * std::cos(a), ly = radius * std::sin(a);
			V p = { c.x + lx * cs, c.y + ly, c.z - lx * sn };
			float piece = float(M_PI) * radius / float(pieces) * 0.5f;
			box(p, { piece, thickness, thickness }, yaw, mat);
		}
		box({ c.x + radius * cs, c.y * 0.5f, c.z - radius * sn }, { thickness, std::max(c.y * 0.5f, 0.05f), thickness }, yaw, mat);
		box({ c.x - radius * cs, c.y * 0.5f, c.z + radius * sn }, { thickness, std::max(c.y * 0.5f, 0.05f), thickness }, yaw, mat);
	}

private:
	Mesh& m_mesh;
};

} // namespace

void Mesh::finalize()
{
	for (int k = 0; k < 3; ++k)
	{
		boundsMin[k] = std::numeric_limits<float>::max();
		boundsMax[k] = -std::numeric_limits<float>::max();
	}
	for (size_t i = 0; i < positions.size(); i += 3)
	{
		for (int k = 0; k < 3; ++k)
		{
			boundsMin[k] = std::min(boundsMin[k], positions[i + k]);
			boundsMax[k] = std::max(boundsMax[k], positions[i + k]);
		}
	}
	float extent2 = 0.0f;
	for (int k = 0; k < 3; ++k)
	{
		center[k] = 0.5f * (boundsMin[k] + boundsMax[k]);
		float e = boundsMax[k] - boundsMin[k];
		extent2 += e * e;
	}
	radius = std::max(0.5f * std::sqrt(extent2), 1e-3f);
	materialData.resize(materials.size() * 8);
	for (size_t m = 0; m < materials.size(); ++m)
	{
		const Material& q = materials[m];
		float* d = &materialData[m * 8];
		d[0] = q.base[0];
		d[1] = q.base[1];
		d[2] = q.base[2];
		d[3] = q.roughness;
		d[4] = q.emission[0];
		d[5] = q.emission[1];
		d[6] = q.emission[2];
		d[7] = q.metallic;
	}
}

// The Cornell box: a 2-unit room open at +z (floor, ceiling, back, red left
// and green right walls), two white boxes 0.6 and 1.2 tall turned by -17 and
// +17 degrees, a 0.5 x 0.5 emissive panel of radiance 17 under the ceiling;
// the point light in front of the panel (describeScene), the camera of the
// reference's first view (main.cpp:57-60, 3.17 radii, yaw 0.64, pitch
// 0.255), the sky off (main.cpp:79-83).
Mesh makeCornell()
{
	Mesh mesh;
	Builder b(mesh);
	uint32_t white = b.material(0.73f, 0.73f, 0.73f);
	uint32_t red = b.material(0.63f, 0.065f, 0.05f);
	uint32_t green = b.material(0.14f, 0.45f, 0.091f);
	uint32_t light = b.material(0.78f, 0.78f, 0.78f, 1.0f, 0.0f, 17.0f, 17.0f, 17.0f);
	b.quad({ 0.0f, 0.0f, 0.0f }, { 1.0f, 0.0f, 0.0f }, { 0.0f, 0.0f, 1.0f }, { 0.0f, 1.0f, 0.0f }, white);
	b.quad({ 0.0f, 2.0f, 0.0f }, { 1.0f, 0.0f, 0.0f }, { 0.0f, 0.0f, 1.0f }, { 0.0f, -1.0f, 0.0f }, white);
	b.quad({ 0.0f, 1.0f, -1.0f }, { 1.0f, 0.0f, 0.0f }, { 0.0f, 1.0f, 0.0f }, { 0.0f, 0.0f, 1.0f }, white);
	b.quad({ -1.0f, 1.0f, 0.0f }, { 0.0f, 1.0f, 0.0f }, { 0.0f, 0.0f, 1.0f }, { 1.0f, 0.0f, 0.0f }, red);
	b.quad({ 1.0f, 1.0f, 0.0f }, { 0.0f, 1.0f, 0.0f }, { 0.0f, 0.0f, 1.0f }, { -1.0f, 0.0f, 0.0f }, green);
	b.quad({ 0.0f, 1.998f, 0.0f }, { 0.25f, 0.0f, 0.0f }, { 0.0f, 0.0f, 0.25f }, { 0.0f, -1.0f, 0.0f }, light);
	const float deg = float(M_PI) / 180.0f;
	b.box({ 0.33f, 0.3f, 0.3f }, { 0.3f, 0.3f, 0.3f }, -17.0f * deg, white);
	b.box({ -0.33f, 0.6f, -0.3f }, { 0.3f, 0.6f, 0.3f }, 17.0f * deg, white);
	mesh.finalize();
	const float offset = 0.15f * mesh.radius;
	mesh.lightPosition[0] = 0.0f;
	mesh.lightPosition[1] = 1.998f - offset;
	mesh.lightPosition[2] = 0.0f;
	const float distance = 3.17f * mesh.radius, yaw = 0.64f, pitch = 0.255f;
	const float cp = std::cos(pitch);
	const V forward = { -cp * std::sin(yaw), -std::sin(pitch), -cp * std::cos(yaw) };
	mesh.cameraEye[0] = mesh.center[0] - forward.x * distance;
	mesh.cameraEye[1] = mesh.center[1] - forward.y * distance;
	mesh.cameraEye[2] = mesh.center[2] - forward.z * distance;
	mesh.cameraYaw = yaw;
	mesh.cameraPitch = pitch;
	mesh.sky = false;
	return mesh;
}

namespace
{

// Camera of the reference's Sponza view (main.cpp:80-82): 0.45 radii from
// the centre, yaw pi/2 (looking down -x), pitch 0.255; light near the top.
void frameOpenScene(Mesh& mesh)
{
	mesh.finalize();
	const float distance = 0.45f * mesh.radius, yaw = 0.5f * float(M_PI), pitch = 0.255f;
	const float cp = std::cos(pitch);
	const V forward = { -cp * std::sin(yaw), -std::sin(pitch), -cp * std::cos(yaw) };
	mesh.cameraEye[0] = mesh.center[0] - forward.x * distance;
	mesh.cameraEye[1] = mesh.center[1] - forward.y * distance;
	mesh.cameraEye[2] = mesh.center[2] - forward.z * distance;
	mesh.cameraYaw = yaw;
	mesh.cameraPitch = pitch;
	mesh.lightPosition[0] = mesh.center[0];
	mesh.lightPosition[1] = mesh.boundsMax[1] - 0.15f * mesh.radius;
	mesh.lightPosition[2] = mesh.center[2];
	mesh.sky = true;
}

std::vector<uint32_t> randomMaterials(Builder& b, Random& random, int count)
{
	std::vector<uint32_t> ids;
	for (int k = 0; k < count; ++k)
	{
		ids.push_back(b.material(random.range(0.2f, 0.8f), random.range(0.2f, 0.8f), random.range(0.2f, 0.8f),
			random.range(0.05f, 1.0f), 0.0f));
	}
	return ids;
}

// Emissive panels (2 triangles each) of random colour, radiance 4-12.
void emissivePanels(Builder& b, Random& random, float half, float height, int panels)
{
	for (int k = 0; k < panels; ++k)
	{
		float e = random.range(4.0f, 12.0f);
		uint32_t m = b.material(0.8f, 0.8f, 0.8f, 1.0f, 0.0f, e * random.range(0.5f, 1.0f), e * random.range(0.5f, 1.0f),
			e * random.range(0.5f, 1.0f));
		V c = { random.range(-half, half), random.range(0.3f, height), random.range(-half, half) };
		float yaw = random.range(0.0f, 2.0f * float(M_PI));
		V n = { std::cos(yaw), 0.0f, std::sin(yaw) };
		b.quad(c, { -n.z * 0.25f, 0.0f, n.x * 0.25f }, { 0.0f, 0.25f, 0.0f }, n, m, true);
	}
}

} // namespace

// A walled courtyard of seeded random boxes and arches: albedo uniform in
// [0.2, 0.8], roughness in [0.05, 1], 128 emissive panels (256 triangles).
Mesh makeCourtyard(uint32_t seed, uint32_t targetTriangles)
{
	Mesh mesh;
	Builder b(mesh);
	Random random(seed);
	const float half = std::max(6.0f, 0.06f * std::sqrt(float(targetTriangles)));
	std::vector<uint32_t> mats = randomMaterials(b, random, 64);
	uint32_t ground = b.material(0.55f, 0.5f, 0.45f, 0.9f);
	b.quad({ 0.0f, 0.0f, 0.0f }, { half, 0.0f, 0.0f }, { 0.0f, 0.0f, half }, { 0.0f, 1.0f, 0.0f }, ground);
	const float wall = 4.0f;
	b.box({ 0.0f, 0.5f * wall, -half }, { half, 0.5f * wall, 0.2f }, 0.0f, ground);
	b.box({ 0.0f, 0.5f * wall, half }, { half, 0.5f * wall, 0.2f }, 0.0f, ground);
	b.box({ -half, 0.5f * wall, 0.0f }, { 0.2f, 0.5f * wall, half }, 0.0f, ground);
	b.box({ half, 0.5f * wall, 0.0f }, { 0.2f, 0.5f * wall, half }, 0.0f, ground);
	emissivePanels(b, random, half * 0.9f, 3.0f, 128);
	while (mesh.triangleCount() + 12 <= targetTriangles)
	{
		uint32_t m = mats[random.nextU32() % mats.size()];
		V c = { random.range(-half + 1.0f, half - 1.0f), 0.0f, random.range(-half + 1.0f, half - 1.0f) };
		float yaw = random.range(0.0f, 2.0f * float(M_PI));
		if (random.next() < 0.15f && mesh.triangleCount() + 120 <= targetTriangles)
		{
			float span = random.range(1.0f, 3.0f);
			b.arch({ c.x, random.range(0.8f, 2.0f), c.z }, span, 0.12f, yaw, m, 8);
		}
		else
		{
			V h = { random.range(0.1f, 0.8f), random.range(0.1f, 1.2f), random.range(0.1f, 0.8f) };
			c.y = h.y;
			b.box(c, h, yaw, m);
		}
	}
	frameOpenScene(mesh);
	return mesh;
}

// A city block: seeded boxes, spheres of 512 triangles and thin two-sided
// planes on a ground plane, with emissive panels (128 by default); about
// 80% of the triangles in spheres.
Mesh makeCity(uint32_t seed, uint32_t targetTriangles, int emissivePanelCount)
{
	Mesh mesh;
	Builder b(mesh);
	Random random(seed);
	const float half = std::max(8.0f, 0.02f * std::sqrt(float(targetTriangles)));
	std::vector<uint32_t> mats = randomMaterials(b, random, 128);
	uint32_t ground = b.material(0.5f, 0.5f, 0.5f, 0.8f);
	b.quad({ 0.0f, 0.0f, 0.0f }, { half, 0.0f, 0.0f }, { 0.0f, 0.0f, half }, { 0.0f, 1.0f, 0.0f }, ground);
	emissivePanels(b, random, half * 0.9f, 4.0f, emissivePanelCount);
	while (mesh.triangleCount() + 512 <= targetTriangles)
	{
		uint32_t m = mats[random.nextU32() % mats.size()];
		V c = { random.range(-half, half), 0.0f, random.range(-half, half) };
		float kind = random.next();
		if (kind < 0.8f)
		{
			float r = random.range(0.15f, 0.9f);
			c.y = r + random.range(0.0f, 3.0f) * (random.next() < 0.3f ? 1.0f : 0.0f);
			b.sphere(c, r, m);
		}
		else if (kind < 0.97f)
		{
			V h = { random.range(0.2f, 1.5f), random.range(0.2f, 3.0f), random.range(0.2f, 1.5f) };
			c.y = h.y;
			for (int k = 0; k < 8 && mesh.triangleCount() + 12 <= targetTriangles; ++k)
			{
				V q = { c.x + random.range(-3.0f, 3.0f), 0.0f, c.z + random.range(-3.0f, 3.0f) };
				V hq = { h.x * random.range(0.5f, 1.0f), h.y * random.range(0.3f, 1.0f), h.z * random.range(0.5f, 1.0f) };
				q.y = hq.y;
				b.box(q, hq, random.range(0.0f, 2.0f * float(M_PI)), mats[random.nextU32() % mats.size()]);
			}
		}
		else
		{
			for (int k = 0; k < 32; ++k)
			{
				float yaw = random.range(0.0f, 2.0f * float(M_PI));
				V n = { std::cos(yaw), random.range(-0.3f, 0.3f), std::sin(yaw) };
				n = normalizev(n);
				V u = normalizev(crossv(n, { 0.0f, 1.0f, 0.0f })) * random.range(0.3f, 1.5f);
				V v = normalizev(crossv(u, n)) * random.range(0.3f, 1.5f);
				V q = { c.x + random.range(-4.0f, 4.0f), random.range(0.5f, 4.0f), c.z + random.range(-4.0f, 4.0f) };
				b.quad(q, u, v, n, mats[random.nextU32() % mats.size()], true);
			}
		}
	}
	frameOpenScene(mesh);
	return mesh;
}

} // namespace restir
