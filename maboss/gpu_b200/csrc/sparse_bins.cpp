#include "sparse_bins.h"

#include <algorithm>
#include <exception>
#include <mutex>
#include <thread>

namespace mb {

namespace {

inline int window_of(const uint64_t* k, size_t i) { return (int)(k[2 * i + 1] >> 48) - 1; }

inline unsigned __int128 index_of(const uint64_t* k, size_t i)
{
	return ((unsigned __int128)(k[2 * i + 1] & 0xffffffffffffull) << 64) | k[2 * i];
}

inline bool same_key(const uint64_t* k, size_t a, size_t b) { return k[2 * a] == k[2 * b] && k[2 * a + 1] == k[2 * b + 1]; }

} // namespace

// f(0) .. f(T - 1): chunk 0 on the calling thread, the others on new threads; a chunk whose thread
// cannot be created runs on the calling thread too. Every chunk runs inside a catch: an exception
// (std::bad_alloc from a resize, say) is kept, every started thread is joined, and then the first
// exception is rethrown on the calling thread, so it reaches the C ABI's error translation instead
// of std::terminate.
void parallel_for(int T, const std::function<void(int)>& f)
{
	std::mutex m;
	std::exception_ptr first;
	auto guarded = [&](int t) {
		try
		{
			f(t);
		}
		catch (...)
		{
			std::lock_guard<std::mutex> lock(m);
			if (!first)
				first = std::current_exception();
		}
	};
	std::vector<std::thread> pool;
	int t = 1;
	try
	{
		pool.reserve(T > 1 ? (size_t)(T - 1) : 0);
		for (; t < T; t++)
			pool.emplace_back(guarded, t);
	}
	catch (...)
	{
	}
	for (int u = t; u < T; u++)
		guarded(u);
	guarded(0);
	for (auto& th : pool)
		th.join();
	if (first)
		std::rethrow_exception(first);
}

namespace {

template <typename F>
void parallel(int T, F f)
{
	parallel_for(T, std::function<void(int)>(std::move(f)));
}

} // namespace

void decode_sorted_bins(const uint64_t* keys, const long long* vals, size_t n, int n_windows, int threads,
						bulk_vector<int>& sp_w, bulk_vector<unsigned __int128>& sp_idx,
						bulk_vector<long long>& sp_val, std::vector<size_t>& sp_begin,
						std::vector<unsigned __int128>& fin_idx, std::vector<unsigned>& fin_cnt)
{
	// small inputs stay on the calling thread
	const int T = n < ((size_t)1 << 16) ? 1 : std::max(1, std::min(threads, 64));
	// chunk t covers [start[t], start[t + 1]); a chunk never starts inside a run of equal keys
	std::vector<size_t> start(T + 1, n);
	start[0] = 0;
	for (int t = 1; t < T; t++)
	{
		size_t s = std::max(start[t - 1], n * (size_t)t / (size_t)T);
		while (s > 0 && s < n && same_key(keys, s, s - 1))
			s++;
		start[t] = s;
	}
	// pass 1: distinct window entries and final states per chunk
	std::vector<size_t> nw(T, 0), nf(T, 0);
	parallel(T, [&](int t) {
		size_t a = 0, b = 0;
		for (size_t i = start[t]; i < start[t + 1]; i++)
			if (i == start[t] || !same_key(keys, i, i - 1))
				(window_of(keys, i) < n_windows ? a : b)++;
		nw[t] = a;
		nf[t] = b;
	});
	std::vector<size_t> ow(T + 1, 0), of(T + 1, 0);
	for (int t = 0; t < T; t++)
	{
		ow[t + 1] = ow[t] + nw[t];
		of[t + 1] = of[t] + nf[t];
	}
	// the entry vectors are not initialised (bulk_vector): pass 2 writes every element
	sp_idx.resize(ow[T]);
	sp_val.resize(ow[T]);
	sp_w.resize(ow[T]);
	fin_idx.resize(of[T]);
	fin_cnt.resize(of[T]);
	// pass 2: each chunk writes its entries at its offsets, adding equal adjacent keys
	parallel(T, [&](int t) {
		size_t a = ow[t], b = of[t];
		for (size_t i = start[t]; i < start[t + 1];)
		{
			long long v = 0;
			size_t j = i;
			for (; j < start[t + 1] && same_key(keys, j, i); j++)
				v += vals[j];
			const int w = window_of(keys, i);
			if (w < n_windows)
			{
				sp_w[a] = w;
				sp_idx[a] = index_of(keys, i);
				sp_val[a] = v;
				a++;
			}
			else
			{
				fin_idx[b] = index_of(keys, i);
				fin_cnt[b] = (unsigned)v;
				b++;
			}
			i = j;
		}
	});
	sp_begin.assign((size_t)n_windows + 1, 0);
	for (int w = 0; w <= n_windows; w++)
		sp_begin[w] = (size_t)(std::lower_bound(sp_w.begin(), sp_w.end(), w) - sp_w.begin());
}

void parallel_ranges(size_t n, int threads, const std::function<void(size_t, size_t)>& f)
{
	const int T = n < ((size_t)1 << 16) ? 1 : std::max(1, std::min(threads, 64));
	parallel(T, [&](int t) { f(n * (size_t)t / (size_t)T, n * (size_t)(t + 1) / (size_t)T); });
}

} // namespace mb
