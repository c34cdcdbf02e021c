/*
 * ORACLE (test infrastructure): the built-ins and dispatchers of the C
 * interface over the reference's shader code (see ref_common.h).
 *
 * A compute group's lanes run as coroutines (ucontext) inside one worker
 * thread: each runs until the shader's barrier(), then the next lane runs;
 * a barrier is met once every lane has reached it, which the shaders
 * guarantee (every thread of a group calls every barrier, compute.sh:14-15).
 * Groups, compute invocations and fragments are spread over
 * ref_set_threads() worker threads (default 1, which keeps every pass's
 * order of atomics fixed: invocations in row-major order).
 */
#include "ref_common.h"

#include <ucontext.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace refsh
{
thread_local int t_lane = 0;
thread_local LaneBuiltins t_builtins[kMaxLanes];
thread_local vec2 v_texcoord0;
thread_local vec4 gl_FragCoord;
thread_local vec4 gl_FragColor;
thread_local vec4 gl_FragData[4];
bool g_originBottomLeft = false;

namespace
{
std::recursive_mutex g_atomics;
int g_threads = 1;

// The coroutines of the group a worker thread is running.
struct LaneContext
{
	ucontext_t context;
	std::unique_ptr<char[]> stack;
	bool done = false;
};

constexpr size_t kLaneStack = 512 * 1024;

struct GroupRunner
{
	ucontext_t scheduler;
	LaneContext lanes[kMaxLanes];
	const std::function<void()>* main = nullptr;
	bool inGroup = false;
};

thread_local std::unique_ptr<GroupRunner> t_runnerOwner; // one per worker thread
thread_local GroupRunner* t_runner = nullptr;

void laneEntry()
{
	GroupRunner* runner = t_runner;
	(*runner->main)();
	runner->lanes[t_lane].done = true;
	// Returns to the scheduler through uc_link.
}

// body(i) for every item in [0, items): on the caller's thread, or on
// g_threads worker threads that take items in order from a shared counter.
void forEach(uint32_t items, const std::function<void(uint32_t)>& body)
{
	const int threads = g_threads > 1 ? g_threads : 1;
	if (threads == 1 || items < 2u)
	{
		for (uint32_t i = 0; i < items; ++i)
		{
			body(i);
		}
		return;
	}
	std::atomic<uint32_t> next(0u);
	std::vector<std::thread> pool;
	for (int t = 0; t < threads; ++t)
	{
		pool.emplace_back([&]
		{
			for (uint32_t i = next++; i < items; i = next++)
			{
				body(i);
			}
		});
	}
	for (std::thread& t : pool)
	{
		t.join();
	}
}

} // namespace

void atomicLock() { g_atomics.lock(); }
void atomicUnlock() { g_atomics.unlock(); }

// Inside a group: back to the scheduler, which runs the other lanes up to
// this barrier before resuming this one. Outside a group (one invocation at
// a time) every barrier is already met.
void barrier()
{
	GroupRunner* runner = t_runner;
	if (runner == nullptr || !runner->inGroup)
	{
		return;
	}
	swapcontext(&runner->lanes[t_lane].context, &runner->scheduler);
}

void dispatchGroups(uint32_t width, uint32_t height, uint32_t groupX, uint32_t groupY, const std::function<void()>& _main)
{
	const uint32_t lanes = groupX * groupY;
	if (lanes == 0u || lanes > uint32_t(kMaxLanes))
	{
		std::fprintf(stderr, "ref_shaders: groups of %u lanes are not supported\n", lanes);
		std::abort();
	}
	const uint32_t groupsX = (width + groupX - 1) / groupX;
	const uint32_t groupsY = (height + groupY - 1) / groupY;
	forEach(groupsX * groupsY, [&](uint32_t group)
	{
		if (t_runner == nullptr)
		{
			t_runnerOwner.reset(new GroupRunner());
			t_runner = t_runnerOwner.get();
			for (LaneContext& lane : t_runner->lanes)
			{
				lane.stack.reset(new char[kLaneStack]);
			}
		}
		GroupRunner& runner = *t_runner;
		runner.main = &_main;
		const uint32_t gx = group % groupsX, gy = group / groupsX;
		for (uint32_t lane = 0; lane < lanes; ++lane)
		{
			LaneContext& c = runner.lanes[lane];
			const uint32_t lx = lane % groupX, ly = lane / groupX;
			t_builtins[lane].groupId = uvec3(gx, gy, 0u);
			t_builtins[lane].localId = uvec3(lx, ly, 0u);
			t_builtins[lane].localIndex = lane;
			t_builtins[lane].globalId = uvec3(gx * groupX + lx, gy * groupY + ly, 0u);
			c.done = false;
			getcontext(&c.context);
			c.context.uc_stack.ss_sp = c.stack.get();
			c.context.uc_stack.ss_size = kLaneStack;
			c.context.uc_link = &runner.scheduler;
			makecontext(&c.context, laneEntry, 0);
		}
		runner.inGroup = true;
		// Round robin: each round runs every lane that is not done up to its
		// next barrier (or its end).
		for (bool running = true; running;)
		{
			running = false;
			for (uint32_t lane = 0; lane < lanes; ++lane)
			{
				if (!runner.lanes[lane].done)
				{
					t_lane = int(lane);
					swapcontext(&runner.scheduler, &runner.lanes[lane].context);
					running = running || !runner.lanes[lane].done;
				}
			}
		}
		runner.inGroup = false;
		t_lane = 0;
	});
}

void dispatchSequential(uint32_t width, uint32_t height, const std::function<void()>& _main)
{
	forEach(height, [&](uint32_t y)
	{
		t_lane = 0;
		for (uint32_t x = 0; x < width; ++x)
		{
			gl_GlobalInvocationID = uvec3(x, y, 0u);
			_main();
		}
	});
}

void dispatchFragments(uint32_t width, uint32_t height, const std::function<void()>& _main, const Texture& _target)
{
	const vec2 texel(1.0f / float(width), 1.0f / float(height));
	forEach(height, [&](uint32_t y)
	{
		t_lane = 0;
		for (uint32_t x = 0; x < width; ++x)
		{
			v_texcoord0 = (vec2(float(x), float(y)) + 0.5f) * texel;
			gl_FragCoord = vec4(float(x) + 0.5f, float(y) + 0.5f, 0.0f, 1.0f);
			gl_FragColor = vec4();
			_main();
			_target.store(int(x), int(y), gl_FragColor);
		}
	});
}

} // namespace refsh

extern "C"
{

/* Worker threads of the passes (1: one invocation at a time, in row-major
 * order, which fixes the order of the grid insert's atomics). */
void ref_set_threads(int threads)
{
	refsh::g_threads = threads > 0 ? threads : int(std::thread::hardware_concurrency());
}

int ref_get_threads(void)
{
	return refsh::g_threads;
}

} // extern "C"
