// Host side of the sparse window bins (more than 20 non-internal nodes): the bin table's
// (key, value) pairs, sorted on the device, turned into a result's per-window entries and final
// states. Plain C++ (no CUDA types), so the CPU tests compile and check it directly.
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <new>
#include <type_traits>
#include <utility>
#include <vector>

namespace mb {

// An allocator whose value-less construct() leaves trivially constructible elements uninitialised:
// resize() of a result's sparse vectors (gigabytes on a large job) then neither zero-fills nor
// touches the pages, which are first written by the parallel decode (each host thread faults in
// its own part) instead of by one thread per vector.
template <class T>
struct uninit_allocator : std::allocator<T>
{
	using value_type = T;
	template <class U>
	struct rebind
	{
		using other = uninit_allocator<U>;
	};
	uninit_allocator() = default;
	template <class U>
	uninit_allocator(const uninit_allocator<U>&) noexcept
	{
	}
	template <class U>
	void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value)
	{
		::new (static_cast<void*>(p)) U;
	}
	template <class U, class... A>
	void construct(U* p, A&&... a)
	{
		::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
	}
};
template <class T>
using bulk_vector = std::vector<T, uninit_allocator<T>>;

// keys: two u64 per bin, {index bits 0-63, index bits 64-111 | (window + 1) << 48}, sorted by
// (second, first) word, i.e. by window then index; vals: the bins' sums. Equal adjacent keys are
// added together. Bins of window n_windows are final states (their sums are counts); the others
// become (sp_w, sp_idx, sp_val) entries with sp_begin[w] = the first entry of window w
// (n_windows + 1 values). The work is split over at most `threads` host threads, at key boundaries.
void decode_sorted_bins(const uint64_t* keys, const long long* vals, size_t n, int n_windows, int threads,
						bulk_vector<int>& sp_w, bulk_vector<unsigned __int128>& sp_idx,
						bulk_vector<long long>& sp_val, std::vector<size_t>& sp_begin,
						std::vector<unsigned __int128>& fin_idx, std::vector<unsigned>& fin_cnt);

// f(0) .. f(T - 1), chunk 0 on the calling thread and the others on their own threads (on the
// calling thread when a thread cannot be created). Returns after every chunk has finished; if any
// chunk threw, the first exception is rethrown then (never std::terminate).
void parallel_for(int T, const std::function<void(int)>& f);

// f(begin, end) over [0, n) in contiguous ranges, one per host thread (at most `threads`; one
// range on the calling thread for small n). The ranges cover every index exactly once.
void parallel_ranges(size_t n, int threads, const std::function<void(size_t, size_t)>& f);

} // namespace mb
