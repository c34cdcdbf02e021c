/*
 * ORACLE (test infrastructure): stand-ins for the bgfx declarations that the
 * reference's src/scene.h names (a vertex layout description), so that
 * src/bvh.cpp and src/lights.cpp compile here. Nothing of bgfx runs.
 */
#pragma once
#include <cstdint>

namespace bgfx
{
struct Attrib
{
	enum Enum { Position, Normal, Color0, TexCoord0, TexCoord1, Tangent };
};
struct AttribType
{
	enum Enum { Float };
};
struct VertexLayout
{
	VertexLayout& begin() { return *this; }
	VertexLayout& add(Attrib::Enum, uint8_t, AttribType::Enum) { return *this; }
	void end() {}
};
} // namespace bgfx
