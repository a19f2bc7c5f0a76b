// Ordering of the sparse window bins on the device (ahead-of-time compiled for sm_100a): the bins of
// a result must come out sorted by window, then non-internal index, which is the order of their
// 128-bit keys (high word: window + 1 in bits 48-63 above index bits 64-111; low word: index bits
// 0-63). Two stable least-significant-digit radix sorts of a permutation (CUB, from the CUDA toolkit)
// — by the low word, then by the high word — give that order; the keys and values are then gathered.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "runtime.h"

namespace mb {

namespace {

__global__ void mbs_split(unsigned n, const mb_key128* __restrict__ keys, unsigned long long* __restrict__ lo,
						  unsigned* __restrict__ pos)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		lo[i] = keys[i].lo;
		pos[i] = i;
	}
}

__global__ void mbs_gather_hi(unsigned n, const mb_key128* __restrict__ keys, const unsigned* __restrict__ pos,
							  unsigned long long* __restrict__ hi)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		hi[i] = keys[pos[i]].hi;
}

__global__ void mbs_gather(unsigned n, const mb_key128* __restrict__ keys, const long long* __restrict__ vals,
						   const unsigned* __restrict__ pos, mb_key128* __restrict__ out_keys,
						   long long* __restrict__ out_vals)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		out_keys[i] = keys[pos[i]];
		out_vals[i] = vals[pos[i]];
	}
}

} // namespace

void sort_bins(const mb_key128* keys, const long long* vals, unsigned n, mb_key128* out_keys, long long* out_vals,
			   cudaStream_t s)
{
	if (n == 0)
		return;
	dbuf lo((size_t)n * 8), lo_sorted((size_t)n * 8), hi((size_t)n * 8), hi_sorted((size_t)n * 8);
	dbuf pos((size_t)n * 4), pos_a((size_t)n * 4), pos_b((size_t)n * 4);
	const unsigned grid = (n + 255) / 256;
	mbs_split<<<grid, 256, 0, s>>>(n, keys, lo.as<unsigned long long>(), pos.as<unsigned>());
	MB_CUDA(cudaGetLastError());
	size_t tmp_bytes = 0, tmp2 = 0;
	MB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, lo.as<unsigned long long>(),
											lo_sorted.as<unsigned long long>(), pos.as<unsigned>(),
											pos_a.as<unsigned>(), (int)n, 0, 64, s));
	MB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp2, hi.as<unsigned long long>(),
											hi_sorted.as<unsigned long long>(), pos_a.as<unsigned>(),
											pos_b.as<unsigned>(), (int)n, 0, 64, s));
	dbuf tmp(std::max(tmp_bytes, tmp2));
	// by the low word, then (stable) by the high word
	MB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, lo.as<unsigned long long>(),
											lo_sorted.as<unsigned long long>(), pos.as<unsigned>(),
											pos_a.as<unsigned>(), (int)n, 0, 64, s));
	mbs_gather_hi<<<grid, 256, 0, s>>>(n, keys, pos_a.as<unsigned>(), hi.as<unsigned long long>());
	MB_CUDA(cudaGetLastError());
	tmp2 = tmp.bytes;
	MB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp2, hi.as<unsigned long long>(),
											hi_sorted.as<unsigned long long>(), pos_a.as<unsigned>(),
											pos_b.as<unsigned>(), (int)n, 0, 64, s));
	mbs_gather<<<grid, 256, 0, s>>>(n, keys, vals, pos_b.as<unsigned>(), out_keys, out_vals);
	MB_CUDA(cudaGetLastError());
	MB_CUDA(cudaStreamSynchronize(s)); // the scratch buffers are released on return
}

namespace {

// number of non-zero cells (warp-aggregated into one 64-bit counter)
template <typename T>
__global__ void mbs_count_nonzero(const T* __restrict__ v, unsigned long long cells,
								  unsigned long long* __restrict__ count)
{
	unsigned long long local = 0;
	for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < cells;
		 i += (unsigned long long)gridDim.x * blockDim.x)
		local += v[i] != 0 ? 1ull : 0ull;
	for (int o = 16; o > 0; o >>= 1)
		local += __shfl_down_sync(0xffffffffu, local, o);
	if ((threadIdx.x & 31) == 0 && local)
		atomicAdd(count, local);
}

template <typename T>
struct mbs_nonzero
{
	const T* v;
	__host__ __device__ bool operator()(unsigned long long i) const { return v[i] != 0; }
};

template <typename T>
__global__ void mbs_gather_cells(unsigned long long n, const T* __restrict__ v, const unsigned long long* __restrict__ idx,
								 long long* __restrict__ out)
{
	const unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = (long long)v[idx[i]];
}

template <typename T>
long long compact_cells_t(const T* v, unsigned long long cells, unsigned long long max_entries, dbuf& idx_out,
						  dbuf& val_out, int sm_count, cudaStream_t s)
{
	if (cells == 0)
		return 0;
	dbuf counters(2 * sizeof(unsigned long long));
	unsigned long long* count = counters.as<unsigned long long>();
	MB_CUDA(cudaMemsetAsync(count, 0, 2 * sizeof(unsigned long long), s));
	const unsigned grid = (unsigned)std::min<unsigned long long>((cells + 255) / 256, (unsigned long long)sm_count * 8);
	mbs_count_nonzero<T><<<grid, 256, 0, s>>>(v, cells, count);
	MB_CUDA(cudaGetLastError());
	unsigned long long n = 0;
	MB_CUDA(cudaMemcpyAsync(&n, count, sizeof n, cudaMemcpyDeviceToHost, s));
	MB_CUDA(cudaStreamSynchronize(s));
	if (n > max_entries)
		return -1;
	if (idx_out.bytes < n * sizeof(unsigned long long) || idx_out.bytes == 0)
		idx_out.alloc(std::max<unsigned long long>(n, 1) * sizeof(unsigned long long));
	if (val_out.bytes < n * sizeof(long long) || val_out.bytes == 0)
		val_out.alloc(std::max<unsigned long long>(n, 1) * sizeof(long long));
	unsigned long long* idx = idx_out.as<unsigned long long>();
	unsigned long long* selected = count + 1;
	// in index order (window, then state): chunks of at most 2^30 cells for CUB's item count
	const unsigned long long chunk = 1ull << 30;
	unsigned long long written = 0;
	dbuf tmp;
	for (unsigned long long base = 0; base < cells; base += chunk)
	{
		const int items = (int)std::min(chunk, cells - base);
		thrust::counting_iterator<unsigned long long> in(base);
		size_t tmp_bytes = 0;
		MB_CUDA(cub::DeviceSelect::If(nullptr, tmp_bytes, in, idx + written, selected, items, mbs_nonzero<T> { v }, s));
		if (tmp.bytes < tmp_bytes)
			tmp.alloc(tmp_bytes);
		MB_CUDA(cub::DeviceSelect::If(tmp.p, tmp_bytes, in, idx + written, selected, items, mbs_nonzero<T> { v }, s));
		unsigned long long got = 0;
		MB_CUDA(cudaMemcpyAsync(&got, selected, sizeof got, cudaMemcpyDeviceToHost, s));
		MB_CUDA(cudaStreamSynchronize(s));
		written += got;
	}
	if (written != n)
		throw engine_error(MB_ERR_CUDA, "compaction of the window histogram: inconsistent counts");
	if (n)
	{
		mbs_gather_cells<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, v, idx, val_out.as<long long>());
		MB_CUDA(cudaGetLastError());
	}
	MB_CUDA(cudaStreamSynchronize(s)); // the counters and CUB scratch are released on return
	return (long long)n;
}

} // namespace

long long compact_cells(const long long* occ, const unsigned* cnt, unsigned long long cells,
						unsigned long long max_entries, dbuf& idx_out, dbuf& val_out, int sm_count, cudaStream_t s)
{
	return occ ? compact_cells_t<long long>(occ, cells, max_entries, idx_out, val_out, sm_count, s)
			   : compact_cells_t<unsigned>(cnt, cells, max_entries, idx_out, val_out, sm_count, s);
}

} // namespace mb
