// A minimal glTF 2.0 reader into the triangle soup of restir_host.h, as the
// reference's loadScene (src/scene.cpp:105-381, 722-808, on fastgltf) and
// describeScene (scene.cpp:810-834) prepare a model for the BVH:
//
//   - the default scene's nodes depth first, each node's transform the
//     parent's times its own (a matrix, or translation * rotation * scale);
//   - every triangle-list primitive: POSITION, NORMAL (else the area-weighted
//     face normals of its corners), indices (8, 16 or 32 bit, or none),
//     positions through the node's transform, normals through the inverse
//     transpose and normalised ((0, 1, 0) when degenerate);
//   - triangles grouped by material, in material order, each material's in
//     the order its primitives were met (the reference's per-material draws,
//     which are the BVH builder's input order, bvh.cpp:253-290), primitives
//     without a material last with the default (white, rough, metallic);
//   - per material: baseColorFactor, metallicFactor, roughnessFactor,
//     emissiveFactor times KHR_materials_emissive_strength, doubleSided;
//   - the point light in front of the area-weighted emissive centroid, along
//     the emitters' summed vertex normals, 0.15 radii out (describeScene).
//
// Not read: textures (a textured material keeps its factors), COLOR_0,
// tangents, sparse accessors, morph targets and skins. The per-triangle
// shading normal is the normalised sum of the three corner normals. Buffers
// may be external files, base64 data URIs, or the BIN chunk of a .glb.
#include "../../include/restir_gpu.h"
#include "mesh.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <new>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace restir
{
namespace
{

// --- JSON ------------------------------------------------------------------------------------

struct Json
{
	enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
	double number = 0.0;
	bool boolean = false;
	std::string text;
	std::vector<Json> items;
	std::vector<std::pair<std::string, Json>> fields;

	const Json* find(const char* key) const
	{
		if (kind != Object)
		{
			return nullptr;
		}
		for (const auto& f : fields)
		{
			if (f.first == key)
			{
				return &f.second;
			}
		}
		return nullptr;
	}
	double num(const char* key, double fallback) const
	{
		const Json* v = find(key);
		return v != nullptr && v->kind == Number ? v->number : fallback;
	}
	bool flag(const char* key, bool fallback) const
	{
		const Json* v = find(key);
		return v != nullptr && v->kind == Bool ? v->boolean : fallback;
	}
	const Json& at(size_t i) const
	{
		if (kind != Array || i >= items.size())
		{
			throw std::runtime_error("glTF: index out of range");
		}
		return items[i];
	}
};

class JsonParser
{
public:
	explicit JsonParser(const std::string& text) : m_text(text) {}

	Json parse()
	{
		Json v = value();
		space();
		if (m_at != m_text.size())
		{
			throw std::runtime_error("glTF: trailing characters after the JSON document");
		}
		return v;
	}

private:
	void space()
	{
		while (m_at < m_text.size() && (m_text[m_at] == ' ' || m_text[m_at] == '\n' || m_text[m_at] == '\r' || m_text[m_at] == '\t'))
		{
			++m_at;
		}
	}
	char peek()
	{
		space();
		if (m_at >= m_text.size())
		{
			throw std::runtime_error("glTF: unexpected end of the JSON document");
		}
		return m_text[m_at];
	}
	void expect(char c)
	{
		if (peek() != c)
		{
			throw std::runtime_error(std::string("glTF: expected '") + c + "' in the JSON document");
		}
		++m_at;
	}
	bool word(const char* w)
	{
		const size_t n = std::strlen(w);
		if (m_text.compare(m_at, n, w) == 0)
		{
			m_at += n;
			return true;
		}
		return false;
	}
	std::string string()
	{
		expect('"');
		std::string out;
		while (m_at < m_text.size() && m_text[m_at] != '"')
		{
			char c = m_text[m_at++];
			if (c == '\\')
			{
				if (m_at >= m_text.size())
				{
					break;
				}
				const char e = m_text[m_at++];
				switch (e)
				{
				case 'n': out += '\n'; break;
				case 't': out += '\t'; break;
				case 'r': out += '\r'; break;
				case 'b': out += '\b'; break;
				case 'f': out += '\f'; break;
				case 'u':
				{
					// Keep ASCII; other code points are not needed for keys and URIs here.
					const unsigned code = unsigned(std::stoul(m_text.substr(m_at, 4), nullptr, 16));
					m_at += 4;
					out += code < 0x80 ? char(code) : '?';
					break;
				}
				default: out += e; break;
				}
			}
			else
			{
				out += c;
			}
		}
		expect('"');
		return out;
	}
	Json value()
	{
		Json v;
		const char c = peek();
		if (c == '{')
		{
			++m_at;
			v.kind = Json::Object;
			if (peek() == '}')
			{
				++m_at;
				return v;
			}
			for (;;)
			{
				std::string key = string();
				expect(':');
				v.fields.emplace_back(std::move(key), value());
				if (peek() == ',')
				{
					++m_at;
					continue;
				}
				expect('}');
				return v;
			}
		}
		if (c == '[')
		{
			++m_at;
			v.kind = Json::Array;
			if (peek() == ']')
			{
				++m_at;
				return v;
			}
			for (;;)
			{
				v.items.push_back(value());
				if (peek() == ',')
				{
					++m_at;
					continue;
				}
				expect(']');
				return v;
			}
		}
		if (c == '"')
		{
			v.kind = Json::String;
			v.text = string();
			return v;
		}
		if (word("true"))
		{
			v.kind = Json::Bool;
			v.boolean = true;
			return v;
		}
		if (word("false"))
		{
			v.kind = Json::Bool;
			return v;
		}
		if (word("null"))
		{
			return v;
		}
		const char* begin = m_text.c_str() + m_at;
		char* end = nullptr;
		v.number = std::strtod(begin, &end);
		if (end == begin)
		{
			throw std::runtime_error("glTF: invalid JSON value");
		}
		v.kind = Json::Number;
		m_at += size_t(end - begin);
		return v;
	}

	const std::string& m_text;
	size_t m_at = 0;
};

// --- files and buffers ---------------------------------------------------------------------------

std::string readFile(const std::string& path)
{
	std::ifstream in(path, std::ios::binary);
	if (!in)
	{
		throw std::runtime_error("glTF: cannot open '" + path + "'");
	}
	std::ostringstream s;
	s << in.rdbuf();
	return s.str();
}

std::string directoryOf(const std::string& path)
{
	const size_t slash = path.find_last_of("/\\");
	return slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
}

std::string decodeBase64(const std::string& text)
{
	auto value = [](char c) -> int
	{
		if (c >= 'A' && c <= 'Z') return c - 'A';
		if (c >= 'a' && c <= 'z') return c - 'a' + 26;
		if (c >= '0' && c <= '9') return c - '0' + 52;
		if (c == '+' || c == '-') return 62;
		if (c == '/' || c == '_') return 63;
		return -1;
	};
	std::string out;
	uint32_t bits = 0;
	int count = 0;
	for (char c : text)
	{
		const int v = value(c);
		if (v < 0)
		{
			continue; // padding and whitespace
		}
		bits = (bits << 6) | uint32_t(v);
		count += 6;
		if (count >= 8)
		{
			count -= 8;
			out += char((bits >> count) & 0xffu);
		}
	}
	return out;
}

std::string percentDecode(const std::string& uri)
{
	std::string out;
	for (size_t i = 0; i < uri.size(); ++i)
	{
		if (uri[i] == '%' && i + 2 < uri.size())
		{
			out += char(std::stoi(uri.substr(i + 1, 2), nullptr, 16));
			i += 2;
		}
		else
		{
			out += uri[i];
		}
	}
	return out;
}

uint32_t readU32(const std::string& data, size_t at)
{
	uint32_t v;
	std::memcpy(&v, data.data() + at, 4);
	return v;
}

// --- the document ----------------------------------------------------------------------------

struct Mat4
{
	float m[16]; // column-major, as glTF stores matrices

	static Mat4 identity()
	{
		Mat4 r = {};
		r.m[0] = r.m[5] = r.m[10] = r.m[15] = 1.0f;
		return r;
	}
	Mat4 operator*(const Mat4& b) const
	{
		Mat4 r;
		for (int c = 0; c < 4; ++c)
		{
			for (int row = 0; row < 4; ++row)
			{
				float s = 0.0f;
				for (int k = 0; k < 4; ++k)
				{
					s = s + m[k * 4 + row] * b.m[c * 4 + k];
				}
				r.m[c * 4 + row] = s;
			}
		}
		return r;
	}
};

struct Document
{
	Json root;
	std::vector<std::string> buffers;
	std::string directory;

	const Json& list(const char* key) const
	{
		static const Json empty = [] { Json j; j.kind = Json::Array; return j; }();
		const Json* v = root.find(key);
		return v != nullptr && v->kind == Json::Array ? *v : empty;
	}

	// An accessor as rows of `components` values of its component type.
	struct View
	{
		const uint8_t* data = nullptr;
		size_t count = 0, stride = 0;
		int componentType = 0, components = 0;
		bool normalized = false;
	};

	View view(size_t accessorIndex) const
	{
		const Json& a = list("accessors").at(accessorIndex);
		if (a.find("sparse") != nullptr)
		{
			throw std::runtime_error("glTF: sparse accessors are not supported");
		}
		View v;
		v.count = size_t(a.num("count", 0));
		v.componentType = int(a.num("componentType", 0));
		v.normalized = a.flag("normalized", false);
		const Json* type = a.find("type");
		const std::string t = type != nullptr ? type->text : "";
		v.components = t == "SCALAR" ? 1 : t == "VEC2" ? 2 : t == "VEC3" ? 3 : t == "VEC4" ? 4 : 0;
		const int size = v.componentType == 5126 || v.componentType == 5125 ? 4
			: (v.componentType == 5123 || v.componentType == 5122 ? 2 : (v.componentType == 5121 || v.componentType == 5120 ? 1 : 0));
		if (v.components == 0 || size == 0)
		{
			throw std::runtime_error("glTF: unsupported accessor type");
		}
		const Json* viewIndex = a.find("bufferView");
		if (viewIndex == nullptr)
		{
			throw std::runtime_error("glTF: accessors without a buffer view are not supported");
		}
		const Json& bv = list("bufferViews").at(size_t(viewIndex->number));
		const size_t buffer = size_t(bv.num("buffer", 0));
		if (buffer >= buffers.size())
		{
			throw std::runtime_error("glTF: a buffer view names a missing buffer");
		}
		const size_t offset = size_t(bv.num("byteOffset", 0)) + size_t(a.num("byteOffset", 0));
		const size_t element = size_t(size) * size_t(v.components);
		v.stride = bv.find("byteStride") != nullptr ? size_t(bv.num("byteStride", 0)) : element;
		const size_t length = size_t(bv.num("byteLength", 0));
		if (v.count > 0 && (offset + (v.count - 1) * v.stride + element > buffers[buffer].size()
			|| size_t(a.num("byteOffset", 0)) + (v.count - 1) * v.stride + element > length))
		{
			throw std::runtime_error("glTF: an accessor runs past its buffer");
		}
		v.data = reinterpret_cast<const uint8_t*>(buffers[buffer].data()) + offset;
		return v;
	}

	std::vector<float> floats(size_t accessorIndex, int components) const
	{
		const View v = view(accessorIndex);
		if (v.componentType != 5126 || v.components != components)
		{
			throw std::runtime_error("glTF: expected a float accessor of " + std::to_string(components) + " components");
		}
		std::vector<float> out(v.count * size_t(components));
		for (size_t i = 0; i < v.count; ++i)
		{
			std::memcpy(&out[i * components], v.data + i * v.stride, sizeof(float) * components);
		}
		return out;
	}

	std::vector<uint32_t> indices(size_t accessorIndex) const
	{
		const View v = view(accessorIndex);
		if (v.components != 1)
		{
			throw std::runtime_error("glTF: an index accessor is not scalar");
		}
		std::vector<uint32_t> out(v.count);
		for (size_t i = 0; i < v.count; ++i)
		{
			const uint8_t* p = v.data + i * v.stride;
			switch (v.componentType)
			{
			case 5121: out[i] = p[0]; break;
			case 5123: { uint16_t x; std::memcpy(&x, p, 2); out[i] = x; break; }
			case 5125: { uint32_t x; std::memcpy(&x, p, 4); out[i] = x; break; }
			default: throw std::runtime_error("glTF: an index accessor has an invalid component type");
			}
		}
		return out;
	}
};

Mat4 nodeTransform(const Json& node)
{
	Mat4 m = Mat4::identity();
	if (const Json* matrix = node.find("matrix"))
	{
		for (int i = 0; i < 16 && i < int(matrix->items.size()); ++i)
		{
			m.m[i] = float(matrix->items[i].number);
		}
		return m;
	}
	float t[3] = { 0.0f, 0.0f, 0.0f }, r[4] = { 0.0f, 0.0f, 0.0f, 1.0f }, s[3] = { 1.0f, 1.0f, 1.0f };
	if (const Json* v = node.find("translation"))
	{
		for (int i = 0; i < 3; ++i) t[i] = float(v->at(i).number);
	}
	if (const Json* v = node.find("rotation"))
	{
		for (int i = 0; i < 4; ++i) r[i] = float(v->at(i).number);
	}
	if (const Json* v = node.find("scale"))
	{
		for (int i = 0; i < 3; ++i) s[i] = float(v->at(i).number);
	}
	// T * R * S with R from the unit quaternion (x, y, z, w).
	const float x = r[0], y = r[1], z = r[2], w = r[3];
	const float rot[9] = {
		1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w),  // column 0
		2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w),  // column 1
		2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y) }; // column 2
	for (int c = 0; c < 3; ++c)
	{
		for (int row = 0; row < 3; ++row)
		{
			m.m[c * 4 + row] = rot[c * 3 + row] * s[c];
		}
	}
	m.m[12] = t[0];
	m.m[13] = t[1];
	m.m[14] = t[2];
	return m;
}

struct Vec3
{
	float x, y, z;
};

Vec3 sub(Vec3 a, Vec3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
Vec3 add(Vec3 a, Vec3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
Vec3 cross(Vec3 a, Vec3 b) { return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }
float length(Vec3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

struct Loaded
{
	// Per material slot: triangles as 9 positions, 3 normals.
	std::vector<std::vector<float>> positions, normals;
	Vec3 emissiveCentroid = { 0.0f, 0.0f, 0.0f }, emissiveNormal = { 0.0f, 0.0f, 0.0f };
	float emissiveArea = 0.0f;
};

void appendPrimitive(const Document& doc, const Json& primitive, const Mat4& transform, const std::vector<Material>& materials,
	const std::vector<bool>& emissive, Loaded& out)
{
	if (primitive.num("mode", 4) != 4)
	{
		return; // only triangle lists
	}
	const Json* attributes = primitive.find("attributes");
	const Json* position = attributes != nullptr ? attributes->find("POSITION") : nullptr;
	if (position == nullptr)
	{
		throw std::runtime_error("glTF: a primitive has no POSITION attribute");
	}
	const std::vector<float> p = doc.floats(size_t(position->number), 3);
	const size_t vertices = p.size() / 3;
	std::vector<uint32_t> idx;
	if (const Json* indices = primitive.find("indices"))
	{
		idx = doc.indices(size_t(indices->number));
	}
	else
	{
		idx.resize(vertices);
		for (size_t i = 0; i < vertices; ++i)
		{
			idx[i] = uint32_t(i);
		}
	}
	if (idx.empty() || idx.size() % 3 != 0)
	{
		throw std::runtime_error("glTF: a primitive has an invalid triangle index count");
	}
	for (uint32_t i : idx)
	{
		if (i >= vertices)
		{
			throw std::runtime_error("glTF: a primitive contains an out-of-range index");
		}
	}
	std::vector<float> n;
	if (const Json* normal = attributes->find("NORMAL"))
	{
		n = doc.floats(size_t(normal->number), 3);
		if (n.size() != p.size())
		{
			throw std::runtime_error("glTF: a primitive has mismatched POSITION and NORMAL counts");
		}
	}
	else
	{
		n.assign(p.size(), 0.0f);
		for (size_t t = 0; t < idx.size(); t += 3)
		{
			const Vec3 a = { p[idx[t] * 3], p[idx[t] * 3 + 1], p[idx[t] * 3 + 2] };
			const Vec3 b = { p[idx[t + 1] * 3], p[idx[t + 1] * 3 + 1], p[idx[t + 1] * 3 + 2] };
			const Vec3 c = { p[idx[t + 2] * 3], p[idx[t + 2] * 3 + 1], p[idx[t + 2] * 3 + 2] };
			const Vec3 face = cross(sub(b, a), sub(c, a));
			for (int k = 0; k < 3; ++k)
			{
				n[idx[t + k] * 3] += face.x;
				n[idx[t + k] * 3 + 1] += face.y;
				n[idx[t + k] * 3 + 2] += face.z;
			}
		}
	}
	// World positions, and normals through the inverse transpose of the 3x3 part.
	const float* m = transform.m;
	const double a00 = m[0], a10 = m[1], a20 = m[2], a01 = m[4], a11 = m[5], a21 = m[6], a02 = m[8], a12 = m[9], a22 = m[10];
	const double det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
	float nt[9]; // row-major (inverse)^T
	if (det != 0.0)
	{
		nt[0] = float((a11 * a22 - a12 * a21) / det);
		nt[1] = float(-(a10 * a22 - a12 * a20) / det);
		nt[2] = float((a10 * a21 - a11 * a20) / det);
		nt[3] = float(-(a01 * a22 - a02 * a21) / det);
		nt[4] = float((a00 * a22 - a02 * a20) / det);
		nt[5] = float(-(a00 * a21 - a01 * a20) / det);
		nt[6] = float((a01 * a12 - a02 * a11) / det);
		nt[7] = float(-(a00 * a12 - a02 * a10) / det);
		nt[8] = float((a00 * a11 - a01 * a10) / det);
	}
	else
	{
		std::fill(nt, nt + 9, 0.0f);
	}
	std::vector<Vec3> wp(vertices), wn(vertices);
	for (size_t i = 0; i < vertices; ++i)
	{
		const float x = p[i * 3], y = p[i * 3 + 1], z = p[i * 3 + 2];
		wp[i] = { m[0] * x + m[4] * y + m[8] * z + m[12], m[1] * x + m[5] * y + m[9] * z + m[13],
			m[2] * x + m[6] * y + m[10] * z + m[14] };
		const float nx = n[i * 3], ny = n[i * 3 + 1], nz = n[i * 3 + 2];
		const Vec3 tn = { nt[0] * nx + nt[1] * ny + nt[2] * nz, nt[3] * nx + nt[4] * ny + nt[5] * nz,
			nt[6] * nx + nt[7] * ny + nt[8] * nz };
		const float l = length(tn);
		wn[i] = l > 1e-12f ? Vec3{ tn.x / l, tn.y / l, tn.z / l } : Vec3{ 0.0f, 1.0f, 0.0f };
	}
	const Json* materialIndex = primitive.find("material");
	const size_t slot = materialIndex != nullptr ? size_t(materialIndex->number) : materials.size() - 1;
	if (slot >= materials.size())
	{
		throw std::runtime_error("glTF: a primitive names a missing material");
	}
	std::vector<float>& positions = out.positions[slot];
	std::vector<float>& normals = out.normals[slot];
	for (size_t t = 0; t < idx.size(); t += 3)
	{
		const Vec3 a = wp[idx[t]], b = wp[idx[t + 1]], c = wp[idx[t + 2]];
		for (const Vec3& v : { a, b, c })
		{
			positions.insert(positions.end(), { v.x, v.y, v.z });
		}
		const Vec3 sum = add(add(wn[idx[t]], wn[idx[t + 1]]), wn[idx[t + 2]]);
		const float l = length(sum);
		const Vec3 shading = l > 0.0f ? Vec3{ sum.x / l, sum.y / l, sum.z / l } : cross(sub(b, a), sub(c, a));
		normals.insert(normals.end(), { shading.x, shading.y, shading.z });
		if (emissive[slot])
		{
			// describeScene's light placement (scene.cpp:355-378).
			const float area = 0.5f * length(cross(sub(b, a), sub(c, a)));
			const Vec3 centroid = { (a.x + b.x + c.x) * (1.0f / 3.0f), (a.y + b.y + c.y) * (1.0f / 3.0f), (a.z + b.z + c.z) * (1.0f / 3.0f) };
			out.emissiveCentroid = add(out.emissiveCentroid, { centroid.x * area, centroid.y * area, centroid.z * area });
			out.emissiveNormal = add(out.emissiveNormal, { sum.x * area, sum.y * area, sum.z * area });
			out.emissiveArea += area;
		}
	}
}

void visit(const Document& doc, size_t nodeIndex, const Mat4& parent, const std::vector<Material>& materials,
	const std::vector<bool>& emissive, Loaded& out, int depth)
{
	if (depth > 256)
	{
		throw std::runtime_error("glTF: the node hierarchy is too deep (a cycle?)");
	}
	const Json& node = doc.list("nodes").at(nodeIndex);
	const Mat4 transform = parent * nodeTransform(node);
	if (const Json* mesh = node.find("mesh"))
	{
		const Json& m = doc.list("meshes").at(size_t(mesh->number));
		if (const Json* primitives = m.find("primitives"))
		{
			for (const Json& primitive : primitives->items)
			{
				appendPrimitive(doc, primitive, transform, materials, emissive, out);
			}
		}
	}
	if (const Json* children = node.find("children"))
	{
		for (const Json& child : children->items)
		{
			visit(doc, size_t(child.number), transform, materials, emissive, out, depth + 1);
		}
	}
}

} // namespace

// Loads path into mesh; throws std::runtime_error with a readable message.
void loadGltf(const std::string& path, Mesh& mesh)
{
	Document doc;
	doc.directory = directoryOf(path);
	const std::string file = readFile(path);
	std::string json;
	std::string binChunk;
	if (file.size() >= 12 && file.compare(0, 4, "glTF") == 0)
	{
		// .glb: header, a JSON chunk, an optional BIN chunk.
		size_t at = 12;
		while (at + 8 <= file.size())
		{
			const uint32_t length = readU32(file, at), type = readU32(file, at + 4);
			if (at + 8 + length > file.size())
			{
				throw std::runtime_error("glTF: a .glb chunk runs past the file");
			}
			if (type == 0x4E4F534Au)
			{
				json = file.substr(at + 8, length);
			}
			else if (type == 0x004E4942u)
			{
				binChunk = file.substr(at + 8, length);
			}
			at += 8 + length;
		}
	}
	else
	{
		json = file;
	}
	doc.root = JsonParser(json).parse();
	for (const Json& b : doc.list("buffers").items)
	{
		const Json* uri = b.find("uri");
		if (uri == nullptr)
		{
			doc.buffers.push_back(binChunk);
		}
		else if (uri->text.compare(0, 5, "data:") == 0)
		{
			const size_t comma = uri->text.find(',');
			doc.buffers.push_back(decodeBase64(comma == std::string::npos ? std::string() : uri->text.substr(comma + 1)));
		}
		else
		{
			doc.buffers.push_back(readFile(doc.directory + percentDecode(uri->text)));
		}
	}

	// Materials (loadMaterials / appendPrimitive's factors), then the default one.
	std::vector<Material> materials;
	std::vector<bool> emissive;
	std::vector<uint8_t> twoSided;
	for (const Json& m : doc.list("materials").items)
	{
		Material q;
		q.base[0] = q.base[1] = q.base[2] = 1.0f;
		q.roughness = 1.0f;
		q.metallic = 1.0f;
		if (const Json* pbr = m.find("pbrMetallicRoughness"))
		{
			if (const Json* base = pbr->find("baseColorFactor"))
			{
				for (int k = 0; k < 3; ++k)
				{
					q.base[k] = float(base->at(size_t(k)).number);
				}
			}
			q.roughness = float(pbr->num("roughnessFactor", 1.0));
			q.metallic = float(pbr->num("metallicFactor", 1.0));
		}
		float strength = 1.0f;
		if (const Json* extensions = m.find("extensions"))
		{
			if (const Json* s = extensions->find("KHR_materials_emissive_strength"))
			{
				strength = float(s->num("emissiveStrength", 1.0));
			}
		}
		if (const Json* e = m.find("emissiveFactor"))
		{
			for (int k = 0; k < 3; ++k)
			{
				q.emission[k] = float(e->at(size_t(k)).number) * strength;
			}
		}
		const float strongest = std::max(q.emission[0], std::max(q.emission[1], q.emission[2]));
		emissive.push_back(strongest > 0.0f && m.find("emissiveTexture") == nullptr);
		twoSided.push_back(m.flag("doubleSided", false) ? 1 : 0);
		materials.push_back(q);
	}
	Material fallback;
	fallback.base[0] = fallback.base[1] = fallback.base[2] = 1.0f;
	fallback.roughness = 1.0f;
	fallback.metallic = 1.0f;
	materials.push_back(fallback);
	emissive.push_back(false);
	twoSided.push_back(0);

	Loaded loaded;
	loaded.positions.resize(materials.size());
	loaded.normals.resize(materials.size());
	const Json& scenes = doc.list("scenes");
	if (scenes.items.empty())
	{
		throw std::runtime_error("glTF: the file has no scenes");
	}
	const size_t scene = size_t(doc.root.num("scene", 0));
	const Json* roots = scenes.at(scene).find("nodes");
	if (roots != nullptr)
	{
		for (const Json& node : roots->items)
		{
			visit(doc, size_t(node.number), Mat4::identity(), materials, emissive, loaded, 0);
		}
	}

	mesh = Mesh();
	mesh.materials = materials;
	for (size_t slot = 0; slot < materials.size(); ++slot)
	{
		const size_t triangles = loaded.normals[slot].size() / 3;
		mesh.positions.insert(mesh.positions.end(), loaded.positions[slot].begin(), loaded.positions[slot].end());
		mesh.normals.insert(mesh.normals.end(), loaded.normals[slot].begin(), loaded.normals[slot].end());
		mesh.material.insert(mesh.material.end(), triangles, uint32_t(slot));
		mesh.twoSided.insert(mesh.twoSided.end(), triangles, twoSided[slot]);
	}
	if (mesh.material.empty())
	{
		throw std::runtime_error("glTF: the scene contains no drawable triangles");
	}
	mesh.finalize();
	const float offset = 0.15f * mesh.radius;
	const float normalLength = length(loaded.emissiveNormal);
	if (loaded.emissiveArea > 0.0f && normalLength > 0.0f)
	{
		const float inverseArea = 1.0f / loaded.emissiveArea, inverseLength = 1.0f / normalLength;
		mesh.lightPosition[0] = loaded.emissiveCentroid.x * inverseArea + loaded.emissiveNormal.x * inverseLength * offset;
		mesh.lightPosition[1] = loaded.emissiveCentroid.y * inverseArea + loaded.emissiveNormal.y * inverseLength * offset;
		mesh.lightPosition[2] = loaded.emissiveCentroid.z * inverseArea + loaded.emissiveNormal.z * inverseLength * offset;
	}
	else
	{
		mesh.lightPosition[0] = mesh.center[0];
		mesh.lightPosition[1] = mesh.boundsMax[1] - offset;
		mesh.lightPosition[2] = mesh.center[2];
	}
	// The first view of a loaded model (main.cpp:58-83): 3.17 radii out, yaw
	// 0.64, pitch 0.255; the sky on, except for the bundled Cornell box.
	const float distance = 3.17f * mesh.radius, yaw = 0.64f, pitch = 0.255f;
	const float cp = std::cos(pitch);
	const float forward[3] = { -cp * std::sin(yaw), -std::sin(pitch), -cp * std::cos(yaw) };
	for (int k = 0; k < 3; ++k)
	{
		mesh.cameraEye[k] = mesh.center[k] - forward[k] * distance;
	}
	mesh.cameraYaw = yaw;
	mesh.cameraPitch = pitch;
	const std::string cornell = "cornell_box/scene.gltf";
	mesh.sky = !(path.size() >= cornell.size() && path.compare(path.size() - cornell.size(), cornell.size(), cornell) == 0);
}

} // namespace restir

using namespace restir;

extern "C" void* restir_mesh_load_gltf(const char* path, char* error, uint32_t error_capacity)
{
	if (error != nullptr && error_capacity > 0)
	{
		error[0] = '\0';
	}
	if (path == nullptr)
	{
		return nullptr;
	}
	std::unique_ptr<Mesh> mesh(new (std::nothrow) Mesh());
	if (!mesh)
	{
		return nullptr;
	}
	try
	{
		loadGltf(path, *mesh);
	}
	catch (const std::exception& e)
	{
		if (error != nullptr && error_capacity > 0)
		{
			std::strncpy(error, e.what(), error_capacity - 1);
			error[error_capacity - 1] = '\0';
		}
		return nullptr;
	}
	return mesh.release();
}
