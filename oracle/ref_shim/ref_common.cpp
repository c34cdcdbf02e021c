/*
 * ORACLE (test infrastructure): the built-ins and dispatchers of the C
 * interface over the reference's shader code (see ref_common.h).
 */
#include "ref_common.h"

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <thread>
#include <vector>

namespace refsh
{
thread_local uvec3 gl_GlobalInvocationID;
thread_local uvec3 gl_LocalInvocationID;
thread_local uvec3 gl_WorkGroupID;
thread_local uint gl_LocalInvocationIndex;
thread_local vec2 v_texcoord0;
thread_local vec4 gl_FragCoord;
thread_local vec4 gl_FragColor;
thread_local vec4 gl_FragData[4];
bool g_originBottomLeft = false;

namespace
{
std::recursive_mutex g_atomics;
} // namespace

void atomicLock() { g_atomics.lock(); }
void atomicUnlock() { g_atomics.unlock(); }

// The lanes of one compute group as threads: the shader's barrier() is a
// barrier of all of them. A barrier that is not met within a minute means a
// lane left the shader early, which the shaders rule out (compute.sh:14-15):
// the process stops with a message instead of hanging.
class LaneBarrier
{
public:
	explicit LaneBarrier(int count) : m_count(count) {}

	void wait()
	{
		std::unique_lock<std::mutex> lock(m_mutex);
		const uint64_t generation = m_generation;
		if (++m_waiting == m_count)
		{
			m_waiting = 0;
			++m_generation;
			m_condition.notify_all();
			return;
		}
		if (!m_condition.wait_for(lock, std::chrono::seconds(60), [&] { return m_generation != generation; }))
		{
			std::fprintf(stderr, "ref_shaders: a compute group's barrier was not met\n");
			std::abort();
		}
	}

private:
	std::mutex m_mutex;
	std::condition_variable m_condition;
	int m_count;
	int m_waiting = 0;
	uint64_t m_generation = 0;
};

thread_local LaneBarrier* t_barrier = nullptr;

// Sequential dispatch meets every barrier already; lanes wait for each other.
void barrier()
{
	if (t_barrier != nullptr)
	{
		t_barrier->wait();
	}
}

void dispatchGroups(uint32_t width, uint32_t height, uint32_t groupX, uint32_t groupY, const std::function<void()>& _main)
{
	const uint32_t lanes = groupX * groupY;
	const uint32_t groupsX = (width + groupX - 1) / groupX;
	const uint32_t groupsY = (height + groupY - 1) / groupY;
	LaneBarrier groupBarrier{int(lanes)};
	std::vector<std::thread> threads;
	for (uint32_t lane = 0; lane < lanes; ++lane)
	{
		threads.emplace_back([&, lane]
		{
			t_barrier = &groupBarrier;
			for (uint32_t gy = 0; gy < groupsY; ++gy)
			{
				for (uint32_t gx = 0; gx < groupsX; ++gx)
				{
					const uint32_t lx = lane % groupX, ly = lane / groupX;
					gl_WorkGroupID = uvec3(gx, gy, 0u);
					gl_LocalInvocationID = uvec3(lx, ly, 0u);
					gl_LocalInvocationIndex = lane;
					gl_GlobalInvocationID = uvec3(gx * groupX + lx, gy * groupY + ly, 0u);
					_main();
					groupBarrier.wait(); // shared memory is free for the next group
				}
			}
			t_barrier = nullptr;
		});
	}
	for (std::thread& t : threads)
	{
		t.join();
	}
}

void dispatchSequential(uint32_t width, uint32_t height, const std::function<void()>& _main)
{
	for (uint32_t y = 0; y < height; ++y)
	{
		for (uint32_t x = 0; x < width; ++x)
		{
			gl_GlobalInvocationID = uvec3(x, y, 0u);
			_main();
		}
	}
}

void dispatchFragments(uint32_t width, uint32_t height, const std::function<void()>& _main, const Texture& _target)
{
	const vec2 texel(1.0f / float(width), 1.0f / float(height));
	for (uint32_t y = 0; y < height; ++y)
	{
		for (uint32_t x = 0; x < width; ++x)
		{
			v_texcoord0 = (vec2(float(x), float(y)) + 0.5f) * texel;
			gl_FragCoord = vec4(float(x) + 0.5f, float(y) + 0.5f, 0.0f, 1.0f);
			gl_FragColor = vec4();
			_main();
			_target.store(int(x), int(y), gl_FragColor);
		}
	}
}


} // namespace refsh
