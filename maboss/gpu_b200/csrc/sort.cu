// Ordering of the sparse window bins on the device (ahead-of-time compiled for sm_100a): the bins of
// a result must come out sorted by window, then non-internal index, which is the order of their
// 128-bit keys (high word: window + 1 in bits 48-63 above index bits 64-111; low word: index bits
// 0-63). Two stable least-significant-digit radix sorts of a permutation (CUB, from the CUDA toolkit)
// — by the low word, then by the high word — give that order; the keys and values are then gathered.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

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

} // namespace mb
