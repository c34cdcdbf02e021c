/*
 * ORACLE (test infrastructure): what the C interface over the reference's
 * shader code (ref_passes.cpp) shares: the dispatchers that run a compute
 * pass's invocations (one after another, or a group's lanes as threads that
 * meet at the shader's barriers) and a fragment pass at every texel centre,
 * and the helpers that bind RestirParams' fields to the shaders' uniforms.
 */
#ifndef ORACLE_REF_COMMON_H
#define ORACLE_REF_COMMON_H

#include "shader_shim.h"

#include "../../include/restir_gpu.h"

#include <cstring>
#include <functional>

namespace refsh
{

// Runs _main for every invocation of a width x height dispatch in groups of
// groupX x groupY lanes, one thread per lane, groups one after another.
void dispatchGroups(uint32_t width, uint32_t height, uint32_t groupX, uint32_t groupY, const std::function<void()>& _main);

// Runs _main for every invocation, one after another in row-major order.
void dispatchSequential(uint32_t width, uint32_t height, const std::function<void()>& _main);

// A fragment pass at every texel centre of a width x height target (gl_FragColor stored in its format).
void dispatchFragments(uint32_t width, uint32_t height, const std::function<void()>& _main, const Texture& _target);

inline Texture image(const void* data, uint32_t width, uint32_t height, TexelFormat format, void* write = nullptr)
{
	Texture t;
	t.data = data;
	t.width = int(width);
	t.height = int(height);
	t.format = format;
	t.write = write;
	return t;
}

inline vec4 vec4At(const float* p) { return vec4(p[0], p[1], p[2], p[3]); }

inline mat4 matrix(const float* p)
{
	mat4 m;
	std::memcpy(m.m, p, sizeof(m.m));
	return m;
}

} // namespace refsh

#endif // ORACLE_REF_COMMON_H
