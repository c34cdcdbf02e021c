/*
 * ORACLE (test infrastructure): a dynamic parallel-for over std::thread
 * (this toolchain has no OpenMP runtime). Work items are handed out in
 * chunks from an atomic counter; f(item, thread) runs on thread in
 * [0, threads()).
 */
#ifndef ORACLE_PARALLEL_H
#define ORACLE_PARALLEL_H

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

namespace oracle
{

int& threadSetting();

inline int threads()
{
	int t = threadSetting();
	if (t <= 0)
	{
		t = int(std::max(1u, std::thread::hardware_concurrency()));
	}
	return t;
}

template<typename F>
void parallelFor(int64_t _count, int64_t _chunk, F&& _f)
{
	const int n = int(std::min<int64_t>(threads(), std::max<int64_t>(1, (_count + _chunk - 1) / _chunk)));
	std::atomic<int64_t> next(0);
	auto worker = [&](int _thread)
	{
		for (;;)
		{
			int64_t begin = next.fetch_add(_chunk);
			if (begin >= _count)
			{
				break;
			}
			int64_t end = std::min(_count, begin + _chunk);
			for (int64_t i = begin; i < end; ++i)
			{
				_f(i, _thread);
			}
		}
	};
	if (n <= 1)
	{
		worker(0);
		return;
	}
	std::vector<std::thread> pool;
	for (int t = 1; t < n; ++t)
	{
		pool.emplace_back(worker, t);
	}
	worker(0);
	for (auto& th : pool)
	{
		th.join();
	}
}

} // namespace oracle

#endif // ORACLE_PARALLEL_H
