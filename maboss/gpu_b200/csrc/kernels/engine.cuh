// B200 trajectory engine: hand-written device code, compiled by NVRTC for sm_100a in one
// translation unit after the generated model code (which defines state_size, state_words,
// discrete_time, max_time, time_tick, the per-node rate functions, get_non_internal_index
// and the mbg_* helpers).
//
// Two execution shapes share the same per-step semantics (src/jit_kernels/simulation.cu:77-164):
//  * fused persistent kernel: one thread runs whole trajectories taken from a work counter and
//    accumulates window occupancy, transition entropy, final states and fixed points in place,
//    so no trajectory buffer is written;
//  * buffered epoch kernels: the reference's simulate -> stats -> partition/refill epochs over
//    SoA buffers [slot][word][trajectory], for the stats-plugin API.
// Window sums are int64 fixed point (value * 2^e, round to nearest even): integer atomics make
// every sum independent of thread order, so results are reproducible bit for bit.
#include <curand_kernel.h>

enum class trajectory_status : uint8_t
{
	CONTINUE,
	FINISHED,
	FIXED_POINT
};

// ---------------------------------------------------------------- small helpers

__device__ __forceinline__ void mb_flip(state_word_t* st, int f)
{
	const int fw = f >> 5;
	const uint32_t m = 1u << (f & 31);
#pragma unroll
	for (int w = 0; w < state_words; w++)
		st[w] ^= (w == fw) ? m : 0u;
}

// Initial state: bit i set iff uniform_i <= istate[i], uniforms drawn in node order
// (simulation.cu:34-71).
template <typename RNG>
__device__ __forceinline__ void mb_init_state(state_word_t* st, RNG& rng, const float* __restrict__ istate)
{
#pragma unroll
	for (int w = 0; w < state_words; w++)
	{
		uint32_t s = 0;
		const int nb = (w == state_words - 1) ? state_size - 32 * w : 32;
		for (int b = 0; b < nb; b++)
			if (curand_uniform(&rng) <= __ldg(istate + 32 * w + b))
				s |= 1u << b;
		st[w] = s;
	}
}

// 128-bit fixed-point key: the state itself when it fits in 96 bits, else two independent
// 64-bit hashes. The top bit is always set so that 0 marks an empty slot.
__device__ __forceinline__ mb_key128 mb_state_key(const state_word_t* st)
{
	mb_key128 k;
	if (state_words <= 3)
	{
		k.lo = (unsigned long long)st[0] | (state_words > 1 ? ((unsigned long long)st[state_words > 1 ? 1 : 0] << 32) : 0ull);
		k.hi = (state_words > 2 ? (unsigned long long)st[state_words > 2 ? 2 : 0] : 0ull) | (1ull << 63);
	}
	else
	{
		unsigned long long a = 0x243f6a8885a308d3ull, b = 0x13198a2e03707344ull;
#pragma unroll
		for (int w = 0; w < state_words; w++)
		{
			a = mb_mix64(a ^ ((unsigned long long)st[w] + 0x9e3779b97f4a7c15ull * (w + 1)));
			b = mb_mix64(b + ((unsigned long long)st[w] ^ (0xc2b2ae3d27d4eb4full * (w + 7))));
		}
		k.lo = a;
		k.hi = b | (1ull << 63);
	}
	return k;
}

// Open-addressing insert of a fixed point (bounded probing; overflow is counted, never waited on).
__device__ void mb_fixed_insert(const mb_stats_params& p, const state_word_t* st)
{
	const mb_key128 key = mb_state_key(st);
	const unsigned h = (unsigned)mb_mix64(key.lo ^ mb_mix64(key.hi));
	mb_key128 empty;
	empty.lo = 0;
	empty.hi = 0;
	for (unsigned probe = 0; probe <= p.fp_mask; probe++)
	{
		const unsigned slot = (h + probe) & p.fp_mask;
		const mb_key128 prev = atomicCAS(p.fp_keys + slot, empty, key);
		if (prev.lo == 0ull && prev.hi == 0ull)
		{
#pragma unroll
			for (int w = 0; w < state_words; w++)
				p.fp_states[(size_t)slot * state_words + w] = st[w];
			atomicAdd(p.fp_counts + slot, 1u);
			return;
		}
		if (prev.lo == key.lo && prev.hi == key.hi)
		{
			atomicAdd(p.fp_counts + slot, 1u);
			return;
		}
	}
	atomicAdd(p.fp_overflow, 1u);
}

__device__ __forceinline__ void mb_record(mb_win_acc& a, const mb_stats_params& p, long long* hsink,
										  const state_word_t* st, float t0, float t1, float h)
{
	if (t1 == 0.f) // zero-time slots are empty (window_average_small.cu:68)
		return;
	const mb_idx_t idx = get_non_internal_index(st);
	if (discrete_time)
		mb_record_disc(p, hsink, idx, t0, h);
	else
		mb_record_cont(a, p, hsink, idx, t0, t1, h);
}

// ---------------------------------------------------------------- fused persistent kernel

// One whole trajectory. EXACT reproduces the reference bit for bit: XORWOW streams seeded by
// curand_init(seed, trajectory id, 0), the reference's fp32 operation order, and the 100-slot
// epoch boundary at which the reference stops without flipping and redraws the waiting time
// of the same state in the next epoch (simulation.cu:137-147 with simulation_runner.cu:104-162).
template <bool EXACT, typename RNG>
__device__ __forceinline__ void mb_trajectory(const mb_fused_params& P, RNG& rng, long long* hsink,
											  unsigned long long& trans, mb_win_acc& acc)
{
	state_word_t st[state_words];
	mb_init_state(st, rng, P.istate);
	float time = 0.f;
	int slot = 1;
	bool fixed = false;
	for (;;)
	{
		const float total = mbg_total_rate(st);
		float h = 0.f, tn;
		if (isinf(total))
		{
			// an infinite total rate gives zero waiting times forever: stop this trajectory
			atomicAdd(P.errors, 1u);
			break;
		}
		if (total == 0.f)
		{
			fixed = true;
			tn = max_time;
		}
		else
		{
			if (discrete_time)
			{
				tn = time + time_tick;
				tn = max_time - time_tick < tn ? max_time : tn;
			}
			else
				tn = time + -logf(curand_uniform(&rng)) / total;
			tn = fminf(tn, max_time);
			h = EXACT ? mbg_entropy(st) : mbg_entropy_fast(st);
		}
		trans += (tn != 0.f) ? 1ull : 0ull;
		mb_record(acc, P.st, hsink, st, time, tn, h);
		time = tn;
		if (time >= max_time)
			break;
		if (EXACT && P.traj_len > 1)
		{
			if (++slot >= P.traj_len)
			{
				slot = 1;
				continue;
			}
		}
		const float r = curand_uniform(&rng) * total;
		mb_flip(st, mbg_select_flip(st, r));
	}
	mb_final_add(P.st, get_non_internal_index(st));
	if (fixed)
		mb_fixed_insert(P.st, st);
}

template <bool EXACT>
__device__ __forceinline__ void mb_fused_body(const mb_fused_params& P)
{
	extern __shared__ long long mb_smem_h[];
	long long* hsink = P.st.win_h;
	if (P.st.h_in_smem)
	{
		for (int i = threadIdx.x; i < P.st.n_windows; i += blockDim.x)
			mb_smem_h[i] = 0;
		__syncthreads();
		hsink = mb_smem_h;
	}

	unsigned long long trans = 0;
	mb_win_acc acc;
	mb_acc_init(acc);
	for (;;)
	{
		const unsigned long long t = atomicAdd(P.next_traj, 1ull);
		if (t >= P.n_traj)
			break;
		const unsigned long long id = P.first_traj + t;
		if (EXACT)
		{
			curandState rng;
			if (P.rands)
				rng = static_cast<const curandState*>(P.rands)[t];
			else
				curand_init(P.seed, id, 0ull, &rng);
			mb_trajectory<true>(P, rng, hsink, trans, acc);
		}
		else
		{
			curandStatePhilox4_32_10_t rng;
			curand_init(P.seed, id, 0ull, &rng);
			mb_trajectory<false>(P, rng, hsink, trans, acc);
		}
	}
	mb_acc_flush(acc, P.st, hsink);

#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		trans += __shfl_down_sync(0xffffffffu, trans, o);
	if ((threadIdx.x & 31) == 0 && trans)
		atomicAdd(P.transitions, trans);

	if (P.st.h_in_smem)
	{
		__syncthreads();
		for (int i = threadIdx.x; i < P.st.n_windows; i += blockDim.x)
			if (mb_smem_h[i] != 0)
				atomicAdd(reinterpret_cast<unsigned long long*>(P.st.win_h + i), (unsigned long long)mb_smem_h[i]);
	}
}


#ifdef MBG_INCREMENTAL
// ---------------------------------------------------------------- incremental fast kernel
// Fast mode for models whose rates all have the form `@logic ? U : 0` / `@logic ? 0 : D`.
// A node is unstable when its bit differs from its logic; only unstable nodes have a rate
// (U when off, D when on). Per trajectory, in shared memory: the state words, the unstable
// masks and the integer rate sum of every state word (rates in fixed point 2^-shift); in
// registers: group sums over MB_WPG words and the total. After a flip only the flipped node
// and the nodes whose logic reads it are re-evaluated (truth tables over their inputs), so a
// step costs O(dependents + W/MB_WPG + MB_WPG + 32) instead of O(N) rate evaluations. The flip
// is drawn exactly in proportion to the integer rates with a 64-bit uniform; waiting times and
// window slices are computed as in the other kernels. Statistically equivalent to the
// reference; not bit-exact (different random streams and rate rounding below 2^-shift).
constexpr int MB_WPG = state_words <= 2 ? 1 : (state_words <= 8 ? 2 : 8);
constexpr int MB_GROUPS = (state_words + MB_WPG - 1) / MB_WPG;
constexpr int MB_STEPS_PER_PASS = 4;

// OR of a non-internal index contribution over the warp (128-bit indices as four 32-bit parts).
__device__ __forceinline__ mb_idx_t mb_or_all(mb_idx_t v)
{
#ifdef MBG_WIDE_INDEX
	mb_idx_t r = 0;
#pragma unroll
	for (int q = 0; q < 4; q++)
		r |= (mb_idx_t)__reduce_or_sync(0xffffffffu, (unsigned)(v >> (32 * q))) << (32 * q);
	return r;
#else
	return __reduce_or_sync(0xffffffffu, v);
#endif
}

struct mb_incr_view
{
	uint32_t* st; // [w * blockDim + t]
	uint32_t* un;
	uint32_t* ws;
	int stride;
	__device__ __forceinline__ uint32_t& S(int w) const { return st[w * stride]; }
	__device__ __forceinline__ uint32_t& U(int w) const { return un[w * stride]; }
	__device__ __forceinline__ uint32_t& Q(int w) const { return ws[w * stride]; }
};

// Logic value of the node of dependent record `hdr`/`in` in the state held by view `v`.
__device__ __forceinline__ bool mb_incr_logic(const mb_incr_view& v, int r, const uint4& rec)
{
	const int m = (rec.x >> 16) & 31;
	const unsigned ins[2] = { rec.z, rec.w };
	unsigned p = 0;
#pragma unroll
	for (int t = 0; t < 4; t++)
	{
		if (t < m)
		{
			const unsigned node = (ins[t >> 1] >> ((t & 1) * 16)) & 0xffffu;
			p |= ((v.S(node >> 5) >> (node & 31)) & 1u) << t;
		}
	}
	if (m > 4)
	{
		const uint4 ext = __ldg(mbg_inc_cext + r);
		const unsigned ins2[4] = { ext.x, ext.y, ext.z, ext.w };
#pragma unroll
		for (int t = 4; t < 12; t++)
		{
			if (t < m)
			{
				const unsigned node = (ins2[(t - 4) >> 1] >> ((t & 1) * 16)) & 0xffffu;
				p |= ((v.S(node >> 5) >> (node & 31)) & 1u) << t;
			}
		}
	}
	const unsigned ttw = m <= 5 ? rec.y : __ldg(mbg_inc_tt + rec.y + (p >> 5));
	return (ttw >> (p & 31)) & 1u;
}

// gs[i] is the rate sum of groups 0..i (inclusive prefix sums); a change d in group g moves every
// prefix from g on
__device__ __forceinline__ void mb_group_add(unsigned long long (&gs)[MB_GROUPS], int g, long long d)
{
#pragma unroll
	for (int i = 0; i < MB_GROUPS; i++)
		gs[i] += (i >= g) ? (unsigned long long)d : 0ull;
}

// entropy of the non-internal rates, h = log2(S) - sum(r log2 r) / S
__device__ __forceinline__ float mb_incr_entropy(const mb_incr_view& v)
{
	// the sums over the non-internal nodes in their order, straight-line (generated code)
	float t = 0.f, tl = 0.f;
	mbg_ni_rate_sums(v, t, tl);
	if (!(t > 0.f))
		return 0.f;
	const float h = log2f(t) - tl / t;
	return h > 0.f ? h : 0.f;
}

// Warp-cooperative start of trajectory `t` for the lane whose shared-memory column is `col`:
// lane l draws the initial bit of node 32w + l (Philox is counter based, so the uniform of node
// i is output i of the trajectory's stream, as in a sequential draw), evaluates its logic and
// rate, and the words, unstable masks and word sums are assembled with warp votes/reductions.
// Returns (through the references, valid in every lane) the group sums, total and the index of
// the non-internal state.
__device__ __forceinline__ void mb_incr_start(const mb_fused_params& P, const mb_incr_view& v0, int col,
											  unsigned long long t, unsigned long long (&gs)[MB_GROUPS],
											  unsigned long long& total, mb_idx_t& idx)
{
	const int lane = threadIdx.x & 31;
	mb_incr_view v = v0;
	v.st = v0.st - (threadIdx.x - col);
	v.un = v0.un - (threadIdx.x - col);
	v.ws = v0.ws - (threadIdx.x - col);
	mb_philox_initial_state(P.seed, P.first_traj + t, state_size, P.istate, [&](int w, uint32_t word) {
		if (lane == 0)
			v.S(w) = word;
	});
	__syncwarp();
#pragma unroll
	for (int g = 0; g < MB_GROUPS; g++)
		gs[g] = 0;
	total = 0;
	idx = 0;
	for (int w = 0; w < state_words; w++)
	{
		const int i = 32 * w + lane;
		const uint32_t sw = v.S(w);
		const bool on = (sw >> lane) & 1u;
		bool unstable = false;
		uint32_t q = 0;
		mb_idx_t nibit = 0;
		if (i < state_size)
		{
			const int r = __ldg(mbg_inc_self + i);
			const uint4 rec = __ldg(mbg_inc_crec + r);
			unstable = on != mb_incr_logic(v, r, rec);
			const uint2 qi = __ldg(reinterpret_cast<const uint2*>(mbg_inc_q) + i);
			q = unstable ? (on ? qi.y : qi.x) : 0u;
			const int pos = (int)((rec.x >> 21) & 127u) - 1;
			nibit = (pos >= 0 && on) ? ((mb_idx_t)1 << pos) : (mb_idx_t)0;
		}
		const uint32_t um = __ballot_sync(0xffffffffu, unstable);
		const uint32_t qw = __reduce_add_sync(0xffffffffu, q);
		idx |= mb_or_all(nibit);
		if (lane == 0)
		{
			v.U(w) = um;
			v.Q(w) = qw;
		}
		mb_group_add(gs, w / MB_WPG, qw);
		total += qw;
	}
	__syncwarp();
}

#endif // MBG_INCREMENTAL

#if defined(MBG_INCREMENTAL) && (defined(MB_FAMILY_EXACT) || (defined(MB_FAMILY_EPOCH) && !defined(MB_EPOCH_DENSE)))
// ---- the exact algorithm on incremental unstable sets (models whose rates all have the @logic form)
//
// Bit-identical to the reference algorithm (XORWOW streams, draw order, fp32 operation order),
// without evaluating all N rate functions per step: a stable node's rate is exactly 0 and
// x + 0.0f == x, so the reference's sequential fp32 sum over all nodes equals the sequential sum over
// the unstable nodes in node order, and its prefix-count flip selection always stops at an unstable
// node (simulation.cu:9-21: the first prefix sum reaching r belongs to a node with a non-zero rate).
// Unstable masks are kept incrementally as in the fast kernel; rates are the float values of the
// generated code (mbg_inc_rate). The running sum at the end of every state word is kept in shared
// memory (view slot Q): after a flip only the words from the lowest changed one are re-summed (the
// running sum up to an unchanged prefix is the same fp32 value), and the flip is found by a binary
// search over the word-end sums (non-decreasing, all rates being >= 0) and a scan of one word from
// the previous word-end sum, which reproduces the reference's running comparisons exactly.

// Running fp32 sum over the unstable nodes of state word w, in node order, starting from `run`,
// four nodes per iteration: their rate loads and bit arithmetic are independent of the chain of
// adds (+9.8 % on the 1000-node network over two per iteration; adds of 0.f for the missing nodes
// of a group of four leave a non-negative sum unchanged, so the sums are the same).
__device__ __forceinline__ float mb_exact_word_sum(float run, uint32_t um, uint32_t sw, int w)
{
	while (um)
	{
		const int b0 = __ffs(um) - 1;
		um &= um - 1u;
		const int b1 = __ffs(um) - 1;
		um &= um - 1u;
		const int b2 = __ffs(um) - 1;
		um &= um - 1u;
		const int b3 = __ffs(um) - 1;
		um &= um - 1u;
		const float r0 = __ldg(mbg_inc_rate + 2 * (32 * w + b0) + ((sw >> b0) & 1u));
		const float r1 = b1 >= 0 ? __ldg(mbg_inc_rate + 2 * (32 * w + b1) + ((sw >> b1) & 1u)) : 0.f;
		const float r2 = b2 >= 0 ? __ldg(mbg_inc_rate + 2 * (32 * w + b2) + ((sw >> b2) & 1u)) : 0.f;
		const float r3 = b3 >= 0 ? __ldg(mbg_inc_rate + 2 * (32 * w + b3) + ((sw >> b3) & 1u)) : 0.f;
		run += r0;
		run += r1;
		run += r2;
		run += r3;
	}
	return run;
}

// Unstable masks of the states held by the lanes in `lanes`, computed by the whole warp (all 32 lanes
// call it): one node per lane, one state word at a time. Returns the calling lane's non-internal
// index when the lane is in `lanes`, else `idx`.
__device__ __forceinline__ mb_idx_t mb_exact_masks(const mb_incr_view& v, unsigned lanes, mb_idx_t idx)
{
	const int lane = threadIdx.x & 31;
	while (lanes)
	{
		const int src = __ffs(lanes) - 1;
		lanes &= lanes - 1u;
		mb_incr_view c = v;
		c.st = v.st - (lane - src);
		c.un = v.un - (lane - src);
		mb_idx_t ix = 0;
		for (int w = 0; w < state_words; w++)
		{
			const int i = 32 * w + lane;
			const bool on = (c.S(w) >> lane) & 1u;
			bool unstable = false;
			mb_idx_t nibit = 0;
			if (i < state_size)
			{
				const int r = __ldg(mbg_inc_self + i);
				const uint4 hdr = __ldg(mbg_inc_crec + r);
				unstable = on != mb_incr_logic(c, r, hdr);
				const int pos = (int)((hdr.x >> 21) & 127u) - 1;
				nibit = (pos >= 0 && on) ? ((mb_idx_t)1 << pos) : (mb_idx_t)0;
			}
			const uint32_t um = __ballot_sync(0xffffffffu, unstable);
			ix |= mb_or_all(nibit);
			if (lane == 0)
				c.U(w) = um;
		}
		__syncwarp();
		if (lane == src)
			idx = ix;
	}
	return idx;
}

// compute_transition_rates: the total rate, re-summing the word-end sums from word `lo` on.
__device__ __forceinline__ float mb_exact_total(const mb_incr_view& v, int lo)
{
	float total = lo > 0 ? __uint_as_float(v.Q(lo - 1)) : 0.f;
	for (int w = lo; w < state_words; w++)
	{
		total = mb_exact_word_sum(total, v.U(w), v.S(w), w);
		v.Q(w) = __float_as_uint(total);
	}
	return total;
}

// compute_transition_entropy over the non-internal rates (generator.cpp:146-175).
__device__ __forceinline__ float mb_exact_entropy(const mb_incr_view& v)
{
	float ni_total = 0.f;
	for (int k = 0; k < mbg_noninternal_count; k++)
	{
		const int i = __ldg(mbg_inc_ni_node + k);
		const uint32_t bit = 1u << (i & 31);
		if (v.U(i >> 5) & bit)
			ni_total += __ldg(mbg_inc_rate + 2 * i + ((v.S(i >> 5) & bit) ? 1 : 0));
	}
	if (ni_total == 0.f)
		return 0.f;
	float entropy = 0.f;
	for (int k = 0; k < mbg_noninternal_count; k++)
	{
		const int i = __ldg(mbg_inc_ni_node + k);
		const uint32_t bit = 1u << (i & 31);
		const float r = (v.U(i >> 5) & bit) ? __ldg(mbg_inc_rate + 2 * i + ((v.S(i >> 5) & bit) ? 1 : 0)) : 0.f;
		const float tmp_prob = r / ni_total;
		entropy -= (tmp_prob == 0.f) ? 0.f : log2f(tmp_prob) * tmp_prob;
	}
	return entropy;
}

// select_flip_bit: the first node whose running fp32 sum reaches r; its word is the first whose
// word-end sum reaches r (r <= total = the last word-end sum).
__device__ __forceinline__ int mb_exact_select(const mb_incr_view& v, float r)
{
	int wl = 0, wh = state_words - 1;
	while (wl < wh)
	{
		const int mid = (wl + wh) >> 1;
		if (__uint_as_float(v.Q(mid)) < r)
			wl = mid + 1;
		else
			wh = mid;
	}
	float sum = wl > 0 ? __uint_as_float(v.Q(wl - 1)) : 0.f;
	uint32_t um = v.U(wl);
	const uint32_t sw = v.S(wl);
	int j = -1;
	while (um)
	{
		const int b = __ffs(um) - 1;
		um &= um - 1u;
		j = 32 * wl + b;
		sum += __ldg(mbg_inc_rate + 2 * j + ((sw >> b) & 1u));
		if (!(sum < r))
			break;
	}
	return j;
}

// Flips node j, re-evaluates it and the nodes whose logic reads it, updates the non-internal index;
// returns the lowest state word whose rates changed, and sets ni_changed when the rate of a
// non-internal node may have changed (the transition entropy depends on nothing else).
__device__ __forceinline__ int mb_exact_flip(const mb_incr_view& v, int j, mb_idx_t& idx, bool& ni_changed)
{
	v.S(j >> 5) ^= 1u << (j & 31);
	int lo = j >> 5;
	const uint2 nj = __ldg(reinterpret_cast<const uint2*>(mbg_inc_dep) + j);
	const int pj = (int)(nj.y >> 16) - 1;
	if (pj >= 0)
		idx ^= (mb_idx_t)1 << pj;
	ni_changed |= pj >= 0;
	const int d0 = (int)nj.x, d1 = d0 + (int)(nj.y & 0xffffu);
	// the dependents two at a time, both records' loads in flight (+1 % on the 1000-node network)
	auto dependent = [&](int d, const uint4& hdr) {
		const int k = (int)(hdr.x & 0xffffu);
		const uint32_t bk = 1u << (k & 31);
		const bool on = (v.S(k >> 5) & bk) != 0;
		const bool unstable = on != mb_incr_logic(v, d, hdr);
		const uint32_t uw = v.U(k >> 5);
		if (unstable != ((uw & bk) != 0))
		{
			v.U(k >> 5) = uw ^ bk;
			lo = min(lo, k >> 5);
			ni_changed |= ((hdr.x >> 21) & 127u) != 0u;
		}
	};
	for (int d = d0; d < d1; d += 2)
	{
		const bool two = d + 1 < d1;
		const uint4 h0 = __ldg(mbg_inc_crec + d);
		const uint4 h1 = two ? __ldg(mbg_inc_crec + d + 1) : make_uint4(0u, 0u, 0u, 0u);
		dependent(d, h0);
		if (two)
			dependent(d + 1, h1);
	}
	return lo;
}

// The per-thread shared-memory view of the exact kernels: state words, unstable masks and word-end
// running sums, [3 * state_words][blockDim] u32.
__device__ __forceinline__ mb_incr_view mb_exact_view(uint32_t* smem)
{
	const int B = blockDim.x;
	mb_incr_view v;
	v.stride = B;
	v.st = smem + threadIdx.x;
	v.un = smem + (size_t)state_words * B + threadIdx.x;
	v.ws = smem + (size_t)2 * state_words * B + threadIdx.x;
	return v;
}
#endif

#ifdef MB_FAMILY_EXACT
#ifndef MBG_INCREMENTAL
extern "C" __global__ void __launch_bounds__(256) mb_fused_exact(mb_fused_params P) { mb_fused_body<true>(P); }
#else
// Exact mode: persistent, one thread = one trajectory at a time, with the reference's 100-slot epoch
// boundary (every traj_len - 1 steps the same state is re-evaluated with a fresh draw).
extern "C" __global__ void __launch_bounds__(128) mb_fused_exact(mb_fused_params P)
{
	extern __shared__ uint32_t mb_smem_u32[];
	const int B = blockDim.x;
	const int lane = threadIdx.x & 31;
	const mb_incr_view v = mb_exact_view(mb_smem_u32);
	long long* hsink = P.st.win_h;
	long long* smem_h = reinterpret_cast<long long*>(mb_smem_u32 + (size_t)3 * state_words * B);
	if (P.st.h_in_smem)
	{
		for (int i = threadIdx.x; i < P.st.n_windows; i += B)
			smem_h[i] = 0;
		__syncthreads();
		hsink = smem_h;
	}

	unsigned long long trans = 0;
	mb_win_acc acc;
	mb_acc_init(acc);
	bool working = true, running = false;
	mb_idx_t idx = 0;
	float time = 0.f;
	int slot = 1;
	int lo = 0;				// lowest state word changed since the word-end sums were computed
	bool h_stale = true;	// the transition entropy must be recomputed
	float h_cache = 0.f;
	curandState rng;

	while (__any_sync(0xffffffffu, working || running))
	{
		bool starting = false;
		if (working && !running)
		{
			const unsigned long long t = atomicAdd(P.next_traj, 1ull);
			if (t < P.n_traj)
			{
				starting = true;
				// curand_init's skip-ahead is long and a lane starting a trajectory would run it while
				// the rest of its warp waits: the states come from a parallel init launch when given
				if (P.rands)
					rng = static_cast<const curandState*>(P.rands)[t];
				else
					curand_init(P.seed, P.first_traj + t, 0ull, &rng);
				// initial state: one uniform per node in node order (simulation.cu:51-53)
				for (int w = 0; w < state_words; w++)
				{
					uint32_t sw = 0;
					const int nb = (w == state_words - 1) ? state_size - 32 * w : 32;
					for (int b = 0; b < nb; b++)
						if (curand_uniform(&rng) <= __ldg(P.istate + 32 * w + b))
							sw |= 1u << b;
					v.S(w) = sw;
				}
			}
			else
				working = false;
		}
		__syncwarp();
		idx = mb_exact_masks(v, __ballot_sync(0xffffffffu, starting), idx);
		if (starting)
		{
			time = 0.f;
			slot = 1;
			lo = 0;
			h_stale = true;
			running = true;
		}

		// up to MB_STEPS_PER_PASS steps of a running trajectory per pass of the work-fetch loop
		// (+1.6 % on the 1000-node network; as in the fast kernel)
		for (int step = 0; step < MB_STEPS_PER_PASS && running; step++)
		{
		float total = 0.f, h = 0.f, tn = 0.f;
		if (running)
		{
			total = mb_exact_total(v, lo);
			lo = state_words;
			if (isinf(total))
			{
				// an infinite total rate gives zero waiting times forever: stop this trajectory
				atomicAdd(P.errors, 1u);
				running = false;
				mb_final_add(P.st, idx);
			}
			else if (total == 0.f)
				tn = max_time;
			else
			{
				if (discrete_time)
				{
					tn = time + time_tick;
					tn = max_time - time_tick < tn ? max_time : tn;
				}
				else
					tn = time + -logf(curand_uniform(&rng)) / total;
				tn = fminf(tn, max_time);
				if (h_stale)
					h_cache = mb_exact_entropy(v);
				h_stale = false;
				h = h_cache;
			}
		}
		if (running)
		{
			trans += (tn != 0.f) ? 1ull : 0ull;
			if (tn != 0.f)
			{
				if (discrete_time)
					mb_record_disc(P.st, hsink, idx, time, h);
				else
					mb_record_cont(acc, P.st, hsink, idx, time, tn, h);
			}
			time = tn;
			if (time >= max_time)
			{
				running = false;
				mb_final_add(P.st, idx);
				if (total == 0.f)
				{
					state_word_t st[state_words];
#pragma unroll
					for (int w = 0; w < state_words; w++)
						st[w] = v.S(w);
					mb_fixed_insert(P.st, st);
				}
			}
			else if (P.traj_len > 1 && ++slot >= P.traj_len)
				slot = 1; // epoch boundary: the next epoch re-evaluates the same state
			else
				lo = mb_exact_flip(v, mb_exact_select(v, curand_uniform(&rng) * total), idx, h_stale);
		}
		}
		__syncwarp();
	}
	mb_acc_flush(acc, P.st, hsink);

#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		trans += __shfl_down_sync(0xffffffffu, trans, o);
	if (lane == 0 && trans)
		atomicAdd(P.transitions, trans);

	if (P.st.h_in_smem)
	{
		__syncthreads();
		for (int i = threadIdx.x; i < P.st.n_windows; i += B)
			if (smem_h[i] != 0)
				atomicAdd(reinterpret_cast<unsigned long long*>(P.st.win_h + i), (unsigned long long)smem_h[i]);
	}
}
#endif // MBG_INCREMENTAL
#endif // MB_FAMILY_EXACT

#ifdef MB_FAMILY_FAST
#if !defined(MBG_INCREMENTAL) || !defined(MBG_INTEGER_RATES)
// dense fast kernel: models outside the @logic rate form, and @logic models whose rates the
// integer fixed point cannot hold to 2^-21 (rates spanning more than about 2^12 within a word sum)
extern "C" __global__ void __launch_bounds__(256) mb_fused_fast(mb_fused_params P) { mb_fused_body<false>(P); }
#else
// at least 5 resident blocks of 128: 89 registers on the 1000-node network, no spills. Measured
// (autotuned shapes): the 1000-node network runs equally at 4 and 5 (shared memory limits it to 3
// or 4 blocks), the 50-node network 5.6 % faster at 5; at 6 the 1000-node network loses 11 %.
extern "C" __global__ void __launch_bounds__(128, 5) mb_fused_fast(mb_fused_params P)
{
	extern __shared__ uint32_t mb_smem_u32[];
	const int B = blockDim.x;
	const int lane = threadIdx.x & 31;
	mb_incr_view v;
	v.stride = B;
	v.st = mb_smem_u32 + threadIdx.x;
	v.un = mb_smem_u32 + (size_t)state_words * B + threadIdx.x;
	v.ws = mb_smem_u32 + (size_t)2 * state_words * B + threadIdx.x;
	long long* hsink = P.st.win_h;
	long long* smem_h = reinterpret_cast<long long*>(mb_smem_u32 + (size_t)3 * state_words * B);
	if (P.st.h_in_smem)
	{
		for (int i = threadIdx.x; i < P.st.n_windows; i += B)
			smem_h[i] = 0;
		__syncthreads();
		hsink = smem_h;
	}
	const float inv_scale = 1.0f / (float)(1u << mbg_inc_rate_shift);

	unsigned long long trans = 0;
	mb_win_acc acc;
	mb_acc_init(acc);

	// per-lane trajectory registers
	bool working = true;  // the work counter is not exhausted for this lane
	bool running = false; // the lane holds a trajectory
	unsigned long long gs[MB_GROUPS]; // inclusive prefix sums of the groups' rate sums
	unsigned long long total = 0;
	mb_idx_t idx = 0;
	float time = 0.f, h = 0.f;
	curandStatePhilox4_32_10_t rng;

	// The warp stays converged at the top of every iteration: lanes that need a trajectory take
	// one from the work counter and the whole warp initialises them together; then every lane
	// with a trajectory performs one Gillespie step.
	while (__any_sync(0xffffffffu, working || running))
	{
		unsigned long long t = 0;
		bool starting = false;
		if (working && !running)
		{
			t = atomicAdd(P.next_traj, 1ull);
			if (t < P.n_traj)
				starting = true;
			else
				working = false;
		}
		unsigned pending = __ballot_sync(0xffffffffu, starting);
		while (pending)
		{
			const int src = __ffs(pending) - 1;
			pending &= pending - 1u;
			const unsigned long long ts = __shfl_sync(0xffffffffu, t, src);
			unsigned long long gsx[MB_GROUPS];
			unsigned long long tot;
			mb_idx_t ix;
			mb_incr_start(P, v, (threadIdx.x & ~31) + src, ts, gsx, tot, ix);
			if (lane == src)
			{
#pragma unroll
				for (int g = 0; g < MB_GROUPS; g++)
					gs[g] = gsx[g];
				total = tot;
				idx = ix;
			}
		}
		if (starting)
		{
			// after the N initial-state uniforms, every step uses one whole Philox block (4 x 32 bits)
			curand_init(P.seed, P.first_traj + t, (unsigned long long)((state_size + 3) & ~3), &rng);
			h = mb_incr_entropy(v);
			time = 0.f;
			running = true;
		}

		// up to MB_STEPS_PER_PASS steps of a running trajectory per pass of the work-fetch loop (its
		// votes and branches once per four steps: +2.4 % on the 1000-node network, +2.9 % on the
		// 50-node one; a lane whose trajectory ends idles for the rest of the pass)
		for (int step = 0; step < MB_STEPS_PER_PASS && running; step++)
		{
			const uint4 rb = curand4(&rng); // x: waiting time, (y, z): flip
			float tn;
			if (total == 0)
				tn = max_time;
			else
			{
				if (discrete_time)
				{
					tn = time + time_tick;
					tn = max_time - time_tick < tn ? max_time : tn;
				}
				else
				{
					// uniform in (0, 1]: the top 24 bits plus one, times 2^-24
					const float u = (float)((rb.x >> 8) + 1u) * 5.9604644775390625e-8f;
					tn = time + -logf(u) / ((float)total * inv_scale);
				}
				tn = fminf(tn, max_time);
			}
			trans += (tn != 0.f) ? 1ull : 0ull;
			if (tn != 0.f)
			{
				if (discrete_time)
					mb_record_disc(P.st, hsink, idx, time, total == 0 ? 0.f : h);
				else
					mb_record_cont(acc, P.st, hsink, idx, time, tn, total == 0 ? 0.f : h);
			}
			time = tn;
			if (time >= max_time)
			{
				// end of the trajectory: final state, fixed point
				running = false;
				mb_final_add(P.st, idx);
				if (total == 0)
				{
					state_word_t st[state_words];
#pragma unroll
					for (int w = 0; w < state_words; w++)
						st[w] = v.S(w);
					mb_fixed_insert(P.st, st);
				}
			}
			else
			{
				// draw the flip: r uniform in [0, total), then group -> word -> node
				const unsigned long long r = __umul64hi(((unsigned long long)rb.y << 32) | rb.z, total);
				// gs holds inclusive prefix sums over the groups: the flip's group is the number of
				// prefixes <= r, counted with independent comparisons (a chain of additions before:
				// +2.4 % on the 1000-node network, same selection)
				unsigned long long cum = 0;
				int g = 0;
#pragma unroll
				for (int i = 0; i < MB_GROUPS - 1; i++)
				{
					const bool le = gs[i] <= r;
					g += le ? 1 : 0;
					cum = le ? gs[i] : cum;
				}
				// the group's word sums are loaded together (independent shared-memory loads), their
				// prefix sums formed as a tree (3 levels for 8 words) and the chosen word counted with
				// independent comparisons (+1.5 % on the 1000-node network over a compare-and-add chain,
				// which was +2.3 % over a load-compare loop; same selection)
				int word = g * MB_WPG;
				{
					unsigned long long pq[MB_WPG];
#pragma unroll
					for (int i = 0; i < MB_WPG; i++)
					{
						const int w = g * MB_WPG + i;
						pq[i] = w < state_words ? (unsigned long long)v.Q(w) : 0ull;
					}
#pragma unroll
					for (int d = 1; d < MB_WPG; d <<= 1)
#pragma unroll
						for (int i = MB_WPG - 1; i >= d; i--)
							pq[i] += pq[i - d];
					const unsigned long long rr = r - cum;
					int k = 0;
					unsigned long long c = 0;
#pragma unroll
					for (int i = 0; i < MB_WPG - 1; i++)
					{
						const bool le = pq[i] <= rr && g * MB_WPG + i + 1 < state_words;
						k += le ? 1 : 0;
						c = le ? pq[i] : c;
					}
					word = g * MB_WPG + k;
					cum += c;
				}
				const uint32_t sw = v.S(word);
				uint32_t um = v.U(word);
				int j = 32 * word + 31 - __clz(um | 1u);
				const uint2* q2 = reinterpret_cast<const uint2*>(mbg_inc_q);
				// the chosen word's unstable nodes two at a time: both rate loads are issued before
				// the first comparison (+1.9 % on the 1000-node network over one load per step)
				while (um)
				{
					const int b0 = __ffs(um) - 1;
					const uint32_t um1 = um & (um - 1u);
					const int b1 = um1 ? __ffs(um1) - 1 : b0;
					const uint2 qq0 = __ldg(q2 + 32 * word + b0);
					const uint2 qq1 = __ldg(q2 + 32 * word + b1);
					const uint32_t qa = ((sw >> b0) & 1u) ? qq0.y : qq0.x;
					j = 32 * word + b0;
					if (r < cum + qa)
						break;
					cum += qa;
					if (!um1)
						break;
					const uint32_t qb = ((sw >> b1) & 1u) ? qq1.y : qq1.x;
					j = 32 * word + b1;
					if (r < cum + qb)
						break;
					cum += qb;
					um = um1 & (um1 - 1u);
				}
				const uint2 nj = __ldg(reinterpret_cast<const uint2*>(mbg_inc_dep) + j);

				// flip j and re-evaluate it and the nodes whose logic reads it
				v.S(j >> 5) ^= 1u << (j & 31);
				const int pj = (int)(nj.y >> 16) - 1;
				if (pj >= 0)
					idx ^= (mb_idx_t)1 << pj;
				bool ni_changed = pj >= 0;
				const int d0 = (int)nj.x, d1 = d0 + (int)(nj.y & 0xffffu);
				// the dependents of one flip are distinct nodes: their records are evaluated
				// independently, two at a time so that both records' loads are in flight together
				auto dependent = [&](int d, const uint4& rec) {
					const int k = (int)(rec.x & 0xffffu);
					const uint2 qk = __ldg(q2 + k);
					const int wk = k >> 5;
					const uint32_t bk = 1u << (k & 31);
					const bool on = (v.S(wk) & bk) != 0;
					const bool was_on = (k == j) ? !on : on;
					const uint32_t uw = v.U(wk);
					const bool was_unstable = (uw & bk) != 0;
					const bool unstable = on != mb_incr_logic(v, d, rec);
					const uint32_t qo = was_unstable ? (was_on ? qk.y : qk.x) : 0u;
					const uint32_t qn = unstable ? (on ? qk.y : qk.x) : 0u;
					if (unstable != was_unstable)
						v.U(wk) = uw ^ bk;
					if (qn != qo)
					{
						const long long dq = (long long)qn - (long long)qo;
						v.Q(wk) += (uint32_t)dq;
						mb_group_add(gs, wk / MB_WPG, dq);
						total += (unsigned long long)dq;
					}
					if (qn != qo || unstable != was_unstable)
						ni_changed |= ((rec.x >> 21) & 127u) != 0u;
				};
				for (int d = d0; d < d1; d += 2)
				{
					const bool two = d + 1 < d1;
					const uint4 rec0 = __ldg(mbg_inc_crec + d);
					const uint4 rec1 = two ? __ldg(mbg_inc_crec + d + 1) : make_uint4(0u, 0u, 0u, 0u);
					dependent(d, rec0);
					if (two)
						dependent(d + 1, rec1);
				}
				if (ni_changed)
					h = mb_incr_entropy(v);
			}
		}
		__syncwarp();
	}
	mb_acc_flush(acc, P.st, hsink);

#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		trans += __shfl_down_sync(0xffffffffu, trans, o);
	if (lane == 0 && trans)
		atomicAdd(P.transitions, trans);

	if (P.st.h_in_smem)
	{
		__syncthreads();
		for (int i = threadIdx.x; i < P.st.n_windows; i += B)
			if (smem_h[i] != 0)
				atomicAdd(reinterpret_cast<unsigned long long*>(P.st.win_h + i), (unsigned long long)smem_h[i]);
	}
}
#endif // MBG_INCREMENTAL && MBG_INTEGER_RATES
#endif // MB_FAMILY_FAST

// ---------------------------------------------------------------- buffered epoch kernels (SoA)
// Layouts (stride = batch capacity B):
//   last_states[w * B + i], last_times[i], rands[i] (curandState), statuses[i]
//   traj_states[(s * W + w) * B + i], traj_times[s * B + i], traj_h[s * B + i]

#if defined(MB_FAMILY_EXACT) || defined(MB_FAMILY_EPOCH)
// (kept out of the fast family: curand_init's XORWOW skip-ahead tables are megabytes of code)
// The state of trajectory i is curand_init(seed, first + i, 0) (simulation.cu:23-32). A thread
// initialises `per` consecutive trajectories: curand_init for the first, then one subsequence jump
// each (skipahead_sequence(1)), one matrix product instead of the one per digit of the trajectory
// number that curand_init applies; the states are the same. The host takes per > 1 only when the
// threads still fill the GPU (the initialisation is latency bound below that).
extern "C" __global__ void mb_initialize_random(int n, unsigned long long seed, unsigned long long first,
												 curandState* __restrict__ rands, int per)
{
	const long long id0 = (long long)(blockIdx.x * blockDim.x + threadIdx.x) * per;
	if (id0 >= n)
		return;
	curandState st;
	curand_init(seed, first + (unsigned long long)id0, 0ull, &st);
	rands[id0] = st;
	for (int k = 1; k < per && id0 + k < n; k++)
	{
		skipahead_sequence(1ull, &st);
		rands[id0 + k] = st;
	}
}
#endif

extern "C" __global__ void mb_initialize_initial_state(int n, int stride, const float* __restrict__ istate,
														uint32_t* __restrict__ states, float* __restrict__ times,
														curandState* __restrict__ rands)
{
	const int id = blockIdx.x * blockDim.x + threadIdx.x;
	if (id >= n)
		return;
	curandState r = rands[id];
	state_word_t st[state_words];
	mb_init_state(st, r, istate);
#pragma unroll
	for (int w = 0; w < state_words; w++)
		states[(size_t)w * stride + id] = st[w];
	times[id] = 0.f;
	rands[id] = r;
}

#ifdef MB_FAMILY_EPOCH
#if defined(MBG_INCREMENTAL) && !defined(MB_EPOCH_DENSE)
// One epoch of at most L-1 recorded steps per trajectory (simulation.cu:77-164) for models whose
// rates all have the @logic form: the exact algorithm on incremental unstable sets (the same
// results as the dense per-step evaluation below), each step written to the SoA trajectory buffer
// (a warp stores 128 contiguous bytes per slot and word). Shared memory: [3 * state_words][blockDim].
extern "C" __global__ void __launch_bounds__(128)
	mb_simulate_epoch(int n, int stride, int L, uint32_t* __restrict__ last_states, float* __restrict__ last_times,
					  curandState* __restrict__ rands, uint32_t* __restrict__ traj_states,
					  float* __restrict__ traj_times, float* __restrict__ traj_h, uint8_t* __restrict__ statuses,
					  unsigned long long* __restrict__ transitions)
{
	extern __shared__ uint32_t mb_smem_u32[];
	const int id = blockIdx.x * blockDim.x + threadIdx.x;
	const bool active = id < n;
	const mb_incr_view v = mb_exact_view(mb_smem_u32);
	for (int w = 0; w < state_words; w++)
		v.S(w) = active ? last_states[(size_t)w * stride + id] : 0u;
	__syncwarp();
	mb_idx_t idx = mb_exact_masks(v, __ballot_sync(0xffffffffu, active), 0u);
	unsigned long long trans = 0;
	if (active)
	{
		curandState rng = rands[id];
		float time = last_times[id];
		trajectory_status status = trajectory_status::CONTINUE;
		int step = 0;
		traj_times[(size_t)step * stride + id] = time;
		step++;
		int lo = 0;
		bool h_stale = true;
		float h_cache = 0.f;
		for (;;)
		{
			const float total = mb_exact_total(v, lo);
			lo = state_words;
			float h = 0.f;
			if (isinf(total))
			{
				// an infinite total rate gives zero waiting times forever: end the trajectory
				time = max_time;
				break;
			}
			if (total == 0.f)
			{
				status = trajectory_status::FIXED_POINT;
				time = max_time;
			}
			else
			{
				if (discrete_time)
				{
					time += time_tick;
					time = max_time - time_tick < time ? max_time : time;
				}
				else
					time += -logf(curand_uniform(&rng)) / total;
				time = fminf(time, max_time);
				if (h_stale)
					h_cache = mb_exact_entropy(v);
				h_stale = false;
				h = h_cache;
			}
			for (int w = 0; w < state_words; w++)
				traj_states[((size_t)step * state_words + w) * stride + id] = v.S(w);
			traj_times[(size_t)step * stride + id] = time;
			traj_h[(size_t)step * stride + id] = h;
			trans += (time != 0.f) ? 1ull : 0ull;
			step++;
			if (time >= max_time || step >= L)
				break;
			lo = mb_exact_flip(v, mb_exact_select(v, curand_uniform(&rng) * total), idx, h_stale);
		}
		for (int s = step; s < L; s++) // empty slots carry the zero-time sentinel
			traj_times[(size_t)s * stride + id] = 0.f;
		for (int w = 0; w < state_words; w++)
			last_states[(size_t)w * stride + id] = v.S(w);
		rands[id] = rng;
		last_times[id] = time;
		if (status != trajectory_status::FIXED_POINT)
			status = (time >= max_time) ? trajectory_status::FINISHED : trajectory_status::CONTINUE;
		statuses[id] = (uint8_t)status;
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		trans += __shfl_down_sync(0xffffffffu, trans, o);
	if ((threadIdx.x & 31) == 0 && trans)
		atomicAdd(transitions, trans);
}
#else
// One epoch of at most L-1 recorded steps per trajectory (simulation.cu:77-164): the reference's
// per-step algorithm, every node's generated rate function evaluated at every step.
extern "C" __global__ void __launch_bounds__(256)
	mb_simulate_epoch(int n, int stride, int L, uint32_t* __restrict__ last_states, float* __restrict__ last_times,
					  curandState* __restrict__ rands, uint32_t* __restrict__ traj_states,
					  float* __restrict__ traj_times, float* __restrict__ traj_h, uint8_t* __restrict__ statuses,
					  unsigned long long* __restrict__ transitions)
{
	const int id = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long trans = 0;
	if (id < n)
	{
		state_word_t st[state_words];
#pragma unroll
		for (int w = 0; w < state_words; w++)
			st[w] = last_states[(size_t)w * stride + id];
		curandState rng = rands[id];
		float time = last_times[id];
		trajectory_status status = trajectory_status::CONTINUE;
		int step = 0;
		traj_times[(size_t)step * stride + id] = time;
		step++;
		for (;;)
		{
			const float total = mbg_total_rate(st);
			float h = 0.f;
			if (isinf(total))
			{
				// an infinite total rate gives zero waiting times forever: end the trajectory
				time = max_time;
				break;
			}
			if (total == 0.f)
			{
				status = trajectory_status::FIXED_POINT;
				time = max_time;
			}
			else
			{
				if (discrete_time)
				{
					time += time_tick;
					time = max_time - time_tick < time ? max_time : time;
				}
				else
					time += -logf(curand_uniform(&rng)) / total;
				time = fminf(time, max_time);
				h = mbg_entropy(st);
			}
#pragma unroll
			for (int w = 0; w < state_words; w++)
				traj_states[((size_t)step * state_words + w) * stride + id] = st[w];
			traj_times[(size_t)step * stride + id] = time;
			traj_h[(size_t)step * stride + id] = h;
			trans += (time != 0.f) ? 1ull : 0ull;
			step++;
			if (time >= max_time || step >= L)
				break;
			const float r = curand_uniform(&rng) * total;
			mb_flip(st, mbg_select_flip(st, r));
		}
		for (int s = step; s < L; s++) // empty slots carry the zero-time sentinel
			traj_times[(size_t)s * stride + id] = 0.f;
#pragma unroll
		for (int w = 0; w < state_words; w++)
			last_states[(size_t)w * stride + id] = st[w];
		rands[id] = rng;
		last_times[id] = time;
		if (status != trajectory_status::FIXED_POINT)
			status = (time >= max_time) ? trajectory_status::FINISHED : trajectory_status::CONTINUE;
		statuses[id] = (uint8_t)status;
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		trans += __shfl_down_sync(0xffffffffu, trans, o);
	if ((threadIdx.x & 31) == 0 && trans)
		atomicAdd(transitions, trans);
}
#endif // MBG_INCREMENTAL && !MB_EPOCH_DENSE

#endif // MB_FAMILY_EPOCH

// Window statistics over one epoch's buffer (window_average_small.cu:50-136 over the SoA buffer):
// one thread per trajectory walking its slots, coalesced across threads for every slot, consecutive
// slices of the same (window, state) summed in registers before one 64-bit atomic. The next slot's
// time, entropy and state words are loaded before the current slot is recorded (the loads would
// otherwise wait behind the atomics of the slot before). Measured and rejected: grouping the lanes
// that flush to the same cell with __match_any_sync and adding once per group (one epoch step of
// the 10-node network 5.3 ms -> 27.9 ms, whose state changes at almost every slot so that almost
// every slot flushes; the 1000-node network -1 %).
extern "C" __global__ void __launch_bounds__(256)
	mb_window_epoch(int n, int stride, int L, const uint32_t* __restrict__ traj_states,
					const float* __restrict__ traj_times, const float* __restrict__ traj_h, mb_stats_params p)
{
	extern __shared__ long long mb_smem_h[];
	long long* hsink = p.win_h;
	if (p.h_in_smem)
	{
		for (int i = threadIdx.x; i < p.n_windows; i += blockDim.x)
			mb_smem_h[i] = 0;
		__syncthreads();
		hsink = mb_smem_h;
	}
	const int id = blockIdx.x * blockDim.x + threadIdx.x;
	if (id < n)
	{
		mb_win_acc acc;
		mb_acc_init(acc);
		float t0 = traj_times[id];
		// slot s + 1 is loaded while slot s is recorded
		float t_next = L > 1 ? traj_times[(size_t)stride + id] : 0.f;
		float h_next = L > 1 ? traj_h[(size_t)stride + id] : 0.f;
		state_word_t st_next[state_words];
#pragma unroll
		for (int w = 0; w < state_words; w++)
			st_next[w] = L > 1 ? traj_states[((size_t)state_words + w) * stride + id] : 0u;
		for (int s = 1; s < L; s++)
		{
			const float t1 = t_next, hh = h_next;
			state_word_t st[state_words];
#pragma unroll
			for (int w = 0; w < state_words; w++)
				st[w] = st_next[w];
			if (s + 1 < L)
			{
				t_next = traj_times[(size_t)(s + 1) * stride + id];
				h_next = traj_h[(size_t)(s + 1) * stride + id];
#pragma unroll
				for (int w = 0; w < state_words; w++)
					st_next[w] = traj_states[((size_t)(s + 1) * state_words + w) * stride + id];
			}
			mb_record(acc, p, hsink, st, t0, t1, hh);
			t0 = t1;
		}
		mb_acc_flush(acc, p, hsink);
	}
	if (p.h_in_smem)
	{
		__syncthreads();
		for (int i = threadIdx.x; i < p.n_windows; i += blockDim.x)
			if (mb_smem_h[i] != 0)
				atomicAdd(reinterpret_cast<unsigned long long*>(p.win_h + i), (unsigned long long)mb_smem_h[i]);
	}
}

// Final states of FINISHED / FIXED_POINT trajectories (final_states.cu:9-21).
extern "C" __global__ void mb_final_epoch(int n, int stride, const uint32_t* __restrict__ last_states,
										   const uint8_t* __restrict__ statuses, mb_stats_params p)
{
	const int id = blockIdx.x * blockDim.x + threadIdx.x;
	if (id >= n)
		return;
	const uint8_t s = statuses[id];
	if (s == (uint8_t)trajectory_status::FINISHED || s == (uint8_t)trajectory_status::FIXED_POINT)
	{
		state_word_t st[state_words];
#pragma unroll
		for (int w = 0; w < state_words; w++)
			st[w] = last_states[(size_t)w * stride + id];
		mb_final_add(p, get_non_internal_index(st));
	}
}

// Compaction of the occupied sparse bins into (key, value) records.
extern "C" __global__ void mb_bins_extract(unsigned cap, const mb_key128* __restrict__ keys,
										   const long long* __restrict__ vals, unsigned* __restrict__ out_n,
										   mb_key128* __restrict__ out_keys, long long* __restrict__ out_vals)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= cap)
		return;
	const mb_key128 k = keys[i];
	if (k.lo == 0ull && k.hi == 0ull)
		return;
	const unsigned o = atomicAdd(out_n, 1u);
	out_keys[o] = k;
	out_vals[o] = vals[i];
}

// Fixed points of one epoch (replaces the CUB select/sort/run-length pipeline of
// fixed_states.cu:84-125 with a device hash table).
extern "C" __global__ void mb_fixed_epoch(int n, int stride, const uint32_t* __restrict__ last_states,
										   const uint8_t* __restrict__ statuses, mb_stats_params p)
{
	const int id = blockIdx.x * blockDim.x + threadIdx.x;
	if (id >= n)
		return;
	if (statuses[id] == (uint8_t)trajectory_status::FIXED_POINT)
	{
		state_word_t st[state_words];
#pragma unroll
		for (int w = 0; w < state_words; w++)
			st[w] = last_states[(size_t)w * stride + id];
		mb_fixed_insert(p, st);
	}
}

// ---- stable partition of CONTINUE trajectories to the front (simulation_runner.cu:129-137)
constexpr int MB_SCAN_BLOCK = 1024;

extern "C" __global__ void __launch_bounds__(MB_SCAN_BLOCK)
	mb_compact_count(int n, const uint8_t* __restrict__ statuses, unsigned* __restrict__ block_counts)
{
	const int id = blockIdx.x * MB_SCAN_BLOCK + threadIdx.x;
	const bool keep = id < n && statuses[id] == (uint8_t)trajectory_status::CONTINUE;
	const int c = __syncthreads_count(keep);
	if (threadIdx.x == 0)
		block_counts[blockIdx.x] = (unsigned)c;
}

// Exclusive scan of up to 1024 * 1024 block counts in one block; writes the total last.
extern "C" __global__ void __launch_bounds__(MB_SCAN_BLOCK)
	mb_compact_scan(int nblocks, const unsigned* __restrict__ block_counts, unsigned* __restrict__ block_offsets)
{
	__shared__ unsigned part[MB_SCAN_BLOCK];
	const int per = (nblocks + MB_SCAN_BLOCK - 1) / MB_SCAN_BLOCK;
	const int b0 = threadIdx.x * per;
	unsigned s = 0;
	for (int i = 0; i < per; i++)
		if (b0 + i < nblocks)
			s += block_counts[b0 + i];
	part[threadIdx.x] = s;
	__syncthreads();
	for (int o = 1; o < MB_SCAN_BLOCK; o <<= 1)
	{
		unsigned v = threadIdx.x >= o ? part[threadIdx.x - o] : 0u;
		__syncthreads();
		part[threadIdx.x] += v;
		__syncthreads();
	}
	unsigned run = part[threadIdx.x] - s;
	for (int i = 0; i < per; i++)
		if (b0 + i < nblocks)
		{
			block_offsets[b0 + i] = run;
			run += block_counts[b0 + i];
		}
	if (threadIdx.x == MB_SCAN_BLOCK - 1)
		block_offsets[nblocks] = part[MB_SCAN_BLOCK - 1];
}

extern "C" __global__ void __launch_bounds__(MB_SCAN_BLOCK)
	mb_compact_scatter(int n, int stride, const uint8_t* __restrict__ statuses,
					   const unsigned* __restrict__ block_offsets, const uint32_t* __restrict__ src_states,
					   const float* __restrict__ src_times, const curandState* __restrict__ src_rands,
					   uint32_t* __restrict__ dst_states, float* __restrict__ dst_times, curandState* __restrict__ dst_rands,
					   int rejected_rands)
{
	__shared__ unsigned warp_sums[MB_SCAN_BLOCK / 32];
	const int id = blockIdx.x * MB_SCAN_BLOCK + threadIdx.x;
	const bool keep = id < n && statuses[id] == (uint8_t)trajectory_status::CONTINUE;
	const unsigned ballot = __ballot_sync(0xffffffffu, keep);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0)
		warp_sums[warp] = __popc(ballot);
	__syncthreads();
	if (warp == 0)
	{
		unsigned v = warp_sums[lane];
		unsigned inc = v;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1)
		{
			unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
			if (lane >= o)
				inc += t;
		}
		warp_sums[lane] = inc - v;
	}
	__syncthreads();
	const unsigned kept_before = block_offsets[blockIdx.x] + warp_sums[warp] + __popc(ballot & ((1u << lane) - 1u));
	if (keep)
	{
		const unsigned dst = kept_before;
#pragma unroll
		for (int w = 0; w < state_words; w++)
			dst_states[(size_t)w * stride + dst] = src_states[(size_t)w * stride + id];
		dst_times[dst] = src_times[id];
		dst_rands[dst] = src_rands[id];
	}
	else if (rejected_rands && id < n)
	{
		// the finished trajectories' random states behind the kept ones, last first: where
		// thrust::partition (simulation_runner.cu:133-137) leaves them for the refill to continue
		dst_rands[n - 1 - (id - kept_before)] = src_rands[id];
	}
}


// ---- compaction of the fixed-point table into (state, count) records
extern "C" __global__ void mb_fixed_extract(unsigned cap, const mb_key128* __restrict__ keys,
											 const unsigned* __restrict__ counts, const uint32_t* __restrict__ states,
											 unsigned* __restrict__ out_n, uint32_t* __restrict__ out_states,
											 unsigned* __restrict__ out_counts)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= cap)
		return;
	const mb_key128 k = keys[i];
	if (k.lo == 0ull && k.hi == 0ull)
		return;
	const unsigned o = atomicAdd(out_n, 1u);
#pragma unroll
	for (int w = 0; w < state_words; w++)
		out_states[(size_t)o * state_words + w] = states[(size_t)i * state_words + w];
	out_counts[o] = counts[i];
}
