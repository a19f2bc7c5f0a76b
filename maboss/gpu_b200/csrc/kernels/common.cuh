// Device helpers that do not depend on the model: hashing, fixed-point window accumulation, a
// runtime-width fixed-point hash insert and the Philox initial state. Shared by the NVRTC-compiled
// engine (kernels/engine.cuh) and the ahead-of-time compiled batched kernels (kernels/batched.cuh).
#pragma once
#include <curand_kernel.h>

__device__ __forceinline__ unsigned long long mb_mix64(unsigned long long x)
{
	x ^= x >> 30;
	x *= 0xbf58476d1ce4e5b9ull;
	x ^= x >> 27;
	x *= 0x94d049bb133111ebull;
	x ^= x >> 31;
	return x;
}

// ---------------------------------------------------------------- window accumulation

// The non-internal index: 32 bits for at most 20 non-internal nodes (dense bins, the reference's
// limit), 128 bits beyond (sparse bins, at most 112 nodes; the generated code defines MBG_WIDE_INDEX).
#ifdef MBG_WIDE_INDEX
typedef unsigned __int128 mb_idx_t;
#else
typedef uint32_t mb_idx_t;
#endif

// Adds v to the sparse bin (w, idx): key = (index bits 0-63, index bits 64-111 | (w + 1) << 48);
// open addressing with bounded linear probing; a bin that finds no slot is counted in bin_overflow
// and lost (never waited on).
__device__ inline void mb_bin_add(const mb_stats_params& p, int w, unsigned long long lo, unsigned long long hi,
								  long long v)
{
	const mb_key128 key = { lo, (hi & 0xffffffffffffull) | ((unsigned long long)(w + 1) << 48) };
	const unsigned long long hsh = mb_mix64(key.lo ^ mb_mix64(key.hi));
	for (unsigned probe = 0; probe < 64; probe++)
	{
		const unsigned slot = (unsigned)(hsh + probe) & p.bin_mask;
		mb_key128 cur = p.bin_keys[slot];
		if (cur.lo == 0ull && cur.hi == 0ull)
		{
			const mb_key128 empty = { 0ull, 0ull };
			cur = atomicCAS(p.bin_keys + slot, empty, key);
			if (cur.lo == 0ull && cur.hi == 0ull)
				cur = key;
		}
		if (cur.lo == key.lo && cur.hi == key.hi)
		{
			atomicAdd(reinterpret_cast<unsigned long long*>(p.bin_vals + slot), (unsigned long long)v);
			return;
		}
	}
	atomicAdd(p.bin_overflow, 1u);
}

// Window sum of the continuous occupancy, the discrete count, and the final-state count.
__device__ __forceinline__ void mb_occ_add(const mb_stats_params& p, int w, mb_idx_t idx, long long q)
{
#ifdef MBG_WIDE_INDEX
	mb_bin_add(p, w, (unsigned long long)idx, (unsigned long long)(idx >> 64), q);
#else
	atomicAdd(reinterpret_cast<unsigned long long*>(p.win_occ + (size_t)w * p.n_bins + idx), (unsigned long long)q);
#endif
}

__device__ __forceinline__ void mb_cnt_add(const mb_stats_params& p, int w, mb_idx_t idx)
{
#ifdef MBG_WIDE_INDEX
	mb_bin_add(p, w, (unsigned long long)idx, (unsigned long long)(idx >> 64), 1);
#else
	atomicAdd(p.win_cnt + (size_t)w * p.n_bins + idx, 1u);
#endif
}

__device__ __forceinline__ void mb_final_add(const mb_stats_params& p, mb_idx_t idx)
{
#ifdef MBG_WIDE_INDEX
	mb_bin_add(p, p.n_windows, (unsigned long long)idx, (unsigned long long)(idx >> 64), 1);
#else
	atomicAdd(p.final_cnt + idx, 1u);
#endif
}

// Per-thread run-length accumulator: consecutive slices that fall into the same
// (window, non-internal state) bin are summed in a register before one atomic.
struct mb_win_acc
{
	int ow;
	mb_idx_t oi;
	long long oq;
	int hw;
	long long hq;
};

__device__ __forceinline__ void mb_acc_init(mb_win_acc& a)
{
	a.ow = -1;
	a.oi = 0;
	a.oq = 0;
	a.hw = -1;
	a.hq = 0;
}

__device__ __forceinline__ void mb_add_h(long long* hsink, int w, long long v)
{
	if (v != 0)
		atomicAdd(reinterpret_cast<unsigned long long*>(hsink + w), (unsigned long long)v);
}

__device__ __forceinline__ void mb_acc_flush(mb_win_acc& a, const mb_stats_params& p, long long* hsink)
{
	if (a.ow >= 0 && a.oq != 0)
		mb_occ_add(p, a.ow, a.oi, a.oq);
	if (a.hw >= 0)
		mb_add_h(hsink, a.hw, a.hq);
	mb_acc_init(a);
}

// Continuous time: the state `idx` occupies (t0, t1]; split it over windows exactly like
// window_average_small.cu:66-92 and add each slice (and h * slice) to its window.
__device__ __forceinline__ void mb_record_cont(mb_win_acc& a, const mb_stats_params& p, long long* hsink,
											   mb_idx_t idx, float t0, float t1, float h)
{
	float sb = t0;
	int w = (int)floorf(sb / p.win_tick);
	for (int guard = 0; t1 > sb && guard <= p.n_windows + 2; guard++)
	{
		const float we = (float)(w + 1) * p.win_tick;
		const float se = fminf(t1, we);
		const float sl = se - sb;
		if (w >= 0 && w < p.n_windows)
		{
			const long long q = __double2ll_rn((double)sl * p.fx);
			if (w == a.ow && idx == a.oi)
				a.oq += q;
			else
			{
				if (a.ow >= 0 && a.oq != 0)
					mb_occ_add(p, a.ow, a.oi, a.oq);
				a.ow = w;
				a.oi = idx;
				a.oq = q;
			}
			const long long hq = __double2ll_rn((double)__fmul_rn(h, sl) * p.fx_h);
			if (w == a.hw)
				a.hq += hq;
			else
			{
				if (a.hw >= 0)
					mb_add_h(hsink, a.hw, a.hq);
				a.hw = w;
				a.hq = hq;
			}
		}
		w++;
		sb = se;
	}
}

// Discrete time: count the state at window lround(t0 / tick) (window_average_small.cu:117-130).
__device__ __forceinline__ void mb_record_disc(const mb_stats_params& p, long long* hsink, mb_idx_t idx, float t0,
											   float h)
{
	const int w = (int)lroundf(t0 / p.win_tick);
	if (w >= 0 && w < p.n_windows)
	{
		mb_cnt_add(p, w, idx);
		mb_add_h(hsink, w, __double2ll_rn((double)h * p.fx_h));
	}
}

// Fixed-point hash insert for a state of `words` words (runtime width; same keys and probing as
// mb_fixed_insert of the engine, so both produce the same table layout).
__device__ inline void mb_fixed_insert_rt(const mb_stats_params& p, const unsigned* st, int words)
{
	mb_key128 k;
	if (words <= 3)
	{
		k.lo = (unsigned long long)st[0] | (words > 1 ? (unsigned long long)st[1] << 32 : 0ull);
		k.hi = (words > 2 ? (unsigned long long)st[2] : 0ull) | (1ull << 63);
	}
	else
	{
		unsigned long long a = 0x243f6a8885a308d3ull, b = 0x13198a2e03707344ull;
		for (int w = 0; w < words; w++)
		{
			a = mb_mix64(a ^ ((unsigned long long)st[w] + 0x9e3779b97f4a7c15ull * (w + 1)));
			b = mb_mix64(b + ((unsigned long long)st[w] ^ (0xc2b2ae3d27d4eb4full * (w + 7))));
		}
		k.lo = a;
		k.hi = b | (1ull << 63);
	}
	const unsigned h = (unsigned)mb_mix64(k.lo ^ mb_mix64(k.hi));
	mb_key128 empty;
	empty.lo = 0;
	empty.hi = 0;
	for (unsigned probe = 0; probe <= p.fp_mask; probe++)
	{
		const unsigned slot = (h + probe) & p.fp_mask;
		const mb_key128 prev = atomicCAS(p.fp_keys + slot, empty, k);
		if (prev.lo == 0ull && prev.hi == 0ull)
		{
			for (int w = 0; w < words; w++)
				p.fp_states[(size_t)slot * words + w] = st[w];
			atomicAdd(p.fp_counts + slot, 1u);
			return;
		}
		if (prev.lo == k.lo && prev.hi == k.hi)
		{
			atomicAdd(p.fp_counts + slot, 1u);
			return;
		}
	}
	atomicAdd(p.fp_overflow, 1u);
}

// ---------------------------------------------------------------- Philox initial state

// The initial state of one trajectory, drawn by a whole warp (fast and batched kernels): node i is
// on when the uniform that curand_init(seed, stream, i) followed by curand_uniform gives is at most
// istate[i]. That uniform is output i % 4 of the stream's Philox block i / 4, so one block serves
// four nodes: lane L draws block 32c + L (nodes 128c + 4L .. 4L + 3) with curand_uniform4, and the
// lanes of the four words of that chunk take their node's uniform from it by shuffles (one block
// per lane per 128 nodes instead of one per node; the same states). set_word(w, bits) receives
// each state word (the same value on every lane).
template <class SET_WORD>
__device__ __forceinline__ void mb_philox_initial_state(unsigned long long seed, unsigned long long stream,
														int n_nodes, const float* __restrict__ istate,
														SET_WORD set_word)
{
	const int lane = threadIdx.x & 31;
	const int n_words = (n_nodes + 31) >> 5;
	for (int c = 0; 4 * c < n_words; c++)
	{
		float4 u4 = make_float4(1.f, 1.f, 1.f, 1.f);
		const int b = 32 * c + lane;
		if (4 * b < n_nodes)
		{
			curandStatePhilox4_32_10_t r;
			curand_init(seed, stream, 4ull * (unsigned long long)b, &r);
			u4 = curand_uniform4(&r);
		}
		for (int ww = 0; ww < 4 && 4 * c + ww < n_words; ww++)
		{
			const int w = 4 * c + ww, i = 32 * w + lane;
			const int src = 8 * ww + (lane >> 2);
			const float ux = __shfl_sync(0xffffffffu, u4.x, src);
			const float uy = __shfl_sync(0xffffffffu, u4.y, src);
			const float uz = __shfl_sync(0xffffffffu, u4.z, src);
			const float uw = __shfl_sync(0xffffffffu, u4.w, src);
			const int k = lane & 3;
			const float u = k == 0 ? ux : k == 1 ? uy : k == 2 ? uz : uw;
			const bool on = i < n_nodes && u <= __ldg(istate + i);
			set_word(w, __ballot_sync(0xffffffffu, on));
		}
	}
}
