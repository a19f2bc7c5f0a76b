// Batched incremental kernel: one persistent launch over many (network, parameter variant,
// trajectory) work items, with optional score-function (likelihood-ratio) gradients.
//
// It runs the same algorithm as the incremental fast kernel of kernels/engine.cuh (integer rates
// 2^-shift, one Philox block per step, flips drawn with a 64-bit uniform walking groups -> words ->
// unstable bits, warp-cooperative trajectory start), but nothing is compiled into it: network
// sizes, dependency records, truth tables and rates are runtime data. Networks of different sizes
// and any number of rate variants therefore share one launch, and rates change without
// recompilation. With equal rates and seeds it reproduces the NVRTC-compiled fast kernel.
//
// Gradients. For a path with jumps of rates a_j and total rate a_0, the score up to time t is
//   S(t) = sum_{jumps <= t} d log a_j / d theta  -  int_0^t d a_0 / d theta ds,
// and d E[int_window 1{x(t) = s} dt] / d theta = E[int_window 1{x(t) = s} S(t) dt] (the path after t
// does not change the occupancy at t). Given a cotangent c[w][s] (the gradient of a loss with
// respect to the window probabilities), each trajectory adds to grad[p]
//   sum over recorded slices [u, v] of state s in window w:  c[w][s] * int_u^v S_p(t) dt,
// i.e. the vector-Jacobian product. S_p is kept lazily: S_p(t) = S_p - D_p (t - tp_p), where
// D_p = d a_0 / d theta_p of the current state and tp_p the time D_p last changed; jumps add
// (d rate / d theta_p) / rate. Discrete time uses the step score sum (d log a_j - d a_0 / a_0).

struct mb_net
{
	int N, W, k, discrete;
	int wpg_shift; // log2 of the state words per register group sum: 2^wpg_shift >= ceil(W / MBB_GROUPS)
	float max_time, tick; // simulation constants (as the generated code of the network has them)
	const uint2* dep;	  // per node: {first record, dependents | (ni_pos + 1) << 16}
	const uint4* rec;	  // {k | m << 16 | (ni_pos + 1) << 21, truth table or offset, inputs 0-1, inputs 2-3}
	const uint4* ext;	  // inputs 4-11 of records with more than 4 inputs
	const unsigned* tt;
	const int* self;
	const int* ni_node; // [k]
};

struct mb_variant
{
	int net;
	int rate_shift;
	const uint2* q;		  // [N] (q_up, q_down) integer rates
	const float* rate;	  // [2N] (up, down) float rates
	const float* rlog;	  // [2N] r * log2(r) of those rates (fp64 log2 rounded to fp32, as the NVRTC tables)
	const float* istate;  // [N]
	unsigned long long begin; // first global work index of this variant
	unsigned long long first_traj; // random stream of the variant's trajectory 0
	unsigned n_traj;
	mb_stats_params st;	  // this variant's accumulators (entropy sums in global memory)
	unsigned long long* transitions;
	// gradient (cot == nullptr: off)
	const double* cot;	  // [T * S]
	const int* g_ptr;	  // [2N + 1] CSR of (parameter, d rate / d parameter) per node direction
	const int* g_p;
	const float* g_d;
	double* grad;		  // [P]
};

struct mb_batch_params
{
	const mb_net* nets;
	const mb_variant* vars;
	int n_vars;
	int max_W;			  // shared memory rows per lane
	int P;				  // gradient parameters (rows of gradient scratch), 0 = none
	unsigned long long total;
	unsigned long long seed;
	unsigned long long* next;
	unsigned* errors;
	double* gmem;		  // gradient runs: per-lane global scratch [P][gstride] of partial products R_p,
	unsigned gstride;	  // gstride = the launch's thread count
};

// The number of register group sums; words per group = ceil(W / 8). Measured on C5 (256 variants, 1 to 16 words):
// 8 groups 7.26e9 transitions/s, 4 groups 6.70e9, 16 groups 6.34e9 (predicated updates of every
// group register at each rate change cost more than the longer word walk saves)
constexpr int MBB_GROUPS = 8;

// Network access of the kernel body. mbb_net_rt reads a network's descriptor (every network of a
// batch is runtime data: one launch covers networks of different sizes); the NVRTC build of a
// single network's batch (MB_FAMILY_BATCH, below) instead gives the same quantities as compile-time
// constants and tables of that network's generated code, so that loops over its words unroll and
// no descriptor is read. The variant data (rates, derivatives, accumulators) stays runtime in both.

struct mbb_net_rt
{
	const mb_net& n;
	__device__ __forceinline__ mbb_net_rt(const mb_batch_params& B, const mb_variant& v) : n(B.nets[v.net]) {}
	__device__ __forceinline__ int N() const { return n.N; }
	__device__ __forceinline__ int W() const { return n.W; }
	__device__ __forceinline__ int k() const { return n.k; }
	__device__ __forceinline__ bool discrete() const { return n.discrete != 0; }
	__device__ __forceinline__ float max_time() const { return n.max_time; }
	__device__ __forceinline__ float tick() const { return n.tick; }
	__device__ __forceinline__ int wpg_shift() const { return n.wpg_shift; }
	// the register groups the kernel keeps: all of them (a runtime bound on the group loops cost
	// more than the updates of empty groups, whose prefixes then stay equal to the total)
	__device__ __forceinline__ static constexpr int groups() { return MBB_GROUPS; }
	__device__ __forceinline__ static constexpr int steps_per_pass() { return 1; }
	__device__ __forceinline__ const uint2* dep() const { return n.dep; }
	__device__ __forceinline__ const uint4* rec() const { return n.rec; }
	__device__ __forceinline__ const uint4* ext() const { return n.ext; }
	__device__ __forceinline__ const unsigned* tt() const { return n.tt; }
	__device__ __forceinline__ const int* self() const { return n.self; }
	__device__ __forceinline__ const int* ni_node() const { return n.ni_node; }
	// rate sums of the unstable non-internal nodes, in their order
	template <class V>
	__device__ __forceinline__ void ni_rate_sums(const V& v, const mb_variant& var, float& t, float& tl) const
	{
		for (int kk = 0; kk < n.k; kk++)
		{
			const int i = __ldg(n.ni_node + kk);
			const uint32_t bit = 1u << (i & 31);
			if (v.U(i >> 5) & bit)
			{
				const int e = 2 * i + ((v.S(i >> 5) & bit) ? 1 : 0);
				t += __ldg(var.rate + e);
				tl += __ldg(var.rlog + e);
			}
		}
	}
};


struct mbb_lane
{
	uint32_t* st;
	uint32_t* un;
	uint32_t* ws;
	// per gradient parameter p (continuous time: the score is S_p(t) = A_p - D_p t between changes);
	// A_p and D_p in shared memory, R_p in the lane's global scratch
	float* gS;	 // [P] A_p (continuous) or the score S_p (discrete)
	float* gD;	 // [P] D_p = d a0 / d theta_p of the current state
	double* gR;	 // [P] continuous: sum over p's changes of dD * C2 - dA * C1; discrete: sum of c * S_p;
				 // accumulates the lane's trajectories of one variant
	int stride;		  // shared-memory rows (block size)
	unsigned gstride; // global-scratch rows (threads of the launch)
	__device__ __forceinline__ uint32_t& S(int w) const { return st[w * stride]; }
	__device__ __forceinline__ uint32_t& U(int w) const { return un[w * stride]; }
	__device__ __forceinline__ uint32_t& Q(int w) const { return ws[w * stride]; }
	__device__ __forceinline__ float& GS(int p) const { return gS[p * stride]; }
	__device__ __forceinline__ float& GD(int p) const { return gD[p * stride]; }
	__device__ __forceinline__ double* GR(int p) const { return gR + (size_t)p * gstride; }
};

template <class NET>
__device__ __forceinline__ bool mbb_logic(const NET& net, const mbb_lane& v, int r, const uint4& rec)
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
		const uint4 ext = __ldg(net.ext() + r);
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
	const unsigned ttw = m <= 5 ? rec.y : __ldg(net.tt() + rec.y + (p >> 5));
	return (ttw >> (p & 31)) & 1u;
}

// gs[i] is the rate sum of groups 0..i (inclusive prefix sums; groups past the network's last are
// empty); a change d in group g moves every kept prefix from g on (ng = NET::groups(): the
// network's groups in the specialised kernels, all MBB_GROUPS in the ahead-of-time ones)
__device__ __forceinline__ void mbb_group_add(unsigned long long (&gs)[MBB_GROUPS], int g, long long d, int ng)
{
#pragma unroll
	for (int i = 0; i < MBB_GROUPS; i++)
		if (i < ng)
			gs[i] += (i >= g) ? (unsigned long long)d : 0ull;
}

template <class NET>
__device__ __forceinline__ float mbb_entropy(const NET& net, const mb_variant& var, const mbb_lane& v)
{
	float t = 0.f, tl = 0.f;
	net.ni_rate_sums(v, var, t, tl);
	if (!(t > 0.f))
		return 0.f;
	const float h = log2f(t) - tl / t;
	return h > 0.f ? h : 0.f;
}

// R_p lives in the lane's own global scratch: it is only ever added to, with a reduction that
// does not return the old value (red), so the lane does not wait for an L2 round trip per change;
// the lane reads it back once, with an atomic exchange (ordered after its own reductions).
__device__ __forceinline__ void mbb_red_add(double* a, double v)
{
	asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(a), "d"(v) : "memory");
}

// Continuous time, summed by parts: with the running sums C1 = sum c * length and
// C2 = sum c * length * midpoint over the trajectory's slices, and A_p, D_p piecewise constant,
//   sum over slices of c * int (A_p - D_p t) dt = A_p C1 - D_p C2 - sum over p's changes (dA C1 - dD C2),
// each change's term taken at the sums of its time; a change costs one update of R_p and a slice O(1).

// D_p of the parameters of node k's rate in direction dir changes by sign * d rate / d theta_p at
// time `now`; continuous time keeps S_p(now) (A_p absorbs the change).
__device__ __forceinline__ void mbb_grad_active(const mb_variant& var, const mbb_lane& v, int k, int dir, float sign,
												float now, bool discrete, double C1, double C2)
{
	const int a = __ldg(var.g_ptr + 2 * k + dir), b = __ldg(var.g_ptr + 2 * k + dir + 1);
	for (int e = a; e < b; e++)
	{
		const int p = __ldg(var.g_p + e);
		const float dd = sign * __ldg(var.g_d + e);
		if (!discrete)
		{
			const float dA = dd * now;
			mbb_red_add(v.GR(p), (double)dd * C2 - (double)dA * C1);
			v.GS(p) += dA;
		}
		v.GD(p) += dd;
	}
}

// the lane's trajectory ends: its products join R_p (which then holds the sum over the lane's
// trajectories) and the score restarts
__device__ __forceinline__ void mbb_grad_end(const mbb_lane& v, int P, bool discrete, double C1, double C2)
{
	for (int p = 0; p < P; p++)
	{
		if (!discrete)
			mbb_red_add(v.GR(p), (double)v.GS(p) * C1 - (double)v.GD(p) * C2);
		v.GS(p) = 0.f;
		v.GD(p) = 0.f;
	}
}

// R_p of the lane's trajectories of variant `var` into the variant's gradient
__device__ __forceinline__ void mbb_grad_emit(const mb_variant& var, const mbb_lane& v, int P)
{
	for (int p = 0; p < P; p++)
	{
		const double g = __longlong_as_double(
			(long long)atomicExch(reinterpret_cast<unsigned long long*>(v.GR(p)), 0ull));
		if (g != 0.0)
			atomicAdd(var.grad + p, g);
	}
}

// The cotangent of the lane's last (window, state) cell: consecutive slices mostly stay in one
// cell, so the load is repeated only when the window or the non-internal state changes (gradient on
// the 50-node network 28.4 -> 27.6 ms; the lane resets it when it moves to another variant)
struct mbb_cot_cache
{
	int w = -1;
	unsigned idx = 0;
	double c = 0.0;
};

// the slice [u, w1] of window `w` in state `idx` contributes c * int S dt (continuous: into the
// trajectory's running sums C1, C2) or c * S (discrete)

__device__ __forceinline__ void mbb_grad_slice(const mb_variant& var, const mbb_lane& v, int P, int w, unsigned idx,
											   float u, float w1, bool discrete, double& C1, double& C2,
											   mbb_cot_cache& cc)
{
	if (w != cc.w || idx != cc.idx)
	{
		cc.w = w;
		cc.idx = idx;
		cc.c = __ldg(var.cot + (size_t)w * var.st.n_bins + idx);
	}
	const double c = cc.c;
	if (c == 0.0)
		return;
	if (discrete)
	{
		const float cf = (float)c;
		for (int p = 0; p < P; p++)
			mbb_red_add(v.GR(p), (double)(cf * v.GS(p)));
		return;
	}
	const double len = (double)w1 - (double)u;
	C1 += c * len;
	C2 += c * len * 0.5 * ((double)u + (double)w1);
}

template <bool GRAD>
__device__ __forceinline__ void mbb_record(const mb_variant& var, const mbb_lane& v, int P, mb_win_acc& acc,
										   unsigned idx, float t0, float t1, float h, bool discrete, float tick,
										   double& C1, double& C2, mbb_cot_cache& cc)
{
	if (t1 == 0.f)
		return;
	if (discrete)
	{
		mb_record_disc(var.st, var.st.win_h, idx, t0, h);
		if (GRAD)
		{
			const int w = (int)lroundf(t0 / tick);
			if (w >= 0 && w < var.st.n_windows)
				mbb_grad_slice(var, v, P, w, idx, t0, t1, true, C1, C2, cc);
		}
		return;
	}
	mb_record_cont(acc, var.st, var.st.win_h, idx, t0, t1, h);
	if (GRAD)
	{
		// the same window slices as mb_record_cont
		float sb = t0;
		int w = (int)floorf(sb / tick);
		for (int guard = 0; t1 > sb && guard <= var.st.n_windows + 2; guard++)
		{
			const float we = (float)(w + 1) * tick;
			const float se = fminf(t1, we);
			if (w >= 0 && w < var.st.n_windows)
				mbb_grad_slice(var, v, P, w, idx, sb, se, false, C1, C2, cc);
			w++;
			sb = se;
		}
	}
}

template <bool GRAD, class NET>
__device__ void mbb_body(const mb_batch_params& B)
{
	extern __shared__ uint32_t mbb_smem[];
	const int bs = blockDim.x, lane = threadIdx.x & 31;
	const int MW = B.max_W, P = GRAD ? B.P : 0;
	mbb_lane v;
	v.stride = bs;
	v.st = mbb_smem + threadIdx.x;
	v.un = mbb_smem + (size_t)MW * bs + threadIdx.x;
	v.ws = mbb_smem + (size_t)2 * MW * bs + threadIdx.x;
	float* gbase = reinterpret_cast<float*>(mbb_smem + (size_t)3 * MW * bs);
	v.gS = gbase + threadIdx.x;
	v.gD = gbase + (size_t)P * bs + threadIdx.x;
	v.gstride = B.gstride;
	v.gR = GRAD ? B.gmem + blockIdx.x * bs + threadIdx.x : nullptr;
	double C1 = 0.0, C2 = 0.0; // continuous-time gradient running sums of the lane's trajectory
	for (int p = 0; p < P; p++)
	{
		v.GS(p) = 0.f;
		v.GD(p) = 0.f;
		*v.GR(p) = 0.0;
	}

	mb_win_acc acc;
	mb_acc_init(acc);
	int acc_var = -1; // variant whose accumulators `acc` refers to
	mbb_cot_cache cc;

	bool working = true, running = false;
	int vi = 0; // current variant of this lane
	unsigned long long gs[MBB_GROUPS];
	unsigned long long total = 0;
	uint32_t idx = 0;
	float time = 0.f, h = 0.f;
	unsigned long long trans = 0;
	curandStatePhilox4_32_10_t rng;

	while (__any_sync(0xffffffffu, working || running))
	{
		unsigned long long t = 0;
		int tv = 0;
		bool starting = false;
		if (working && !running)
		{
			t = atomicAdd(B.next, 1ull);
			if (t < B.total)
			{
				// variant of work item t (variants are laid out back to back)
				int lo = 0, hi = B.n_vars - 1;
				while (lo < hi)
				{
					const int mid = (lo + hi + 1) >> 1;
					if (B.vars[mid].begin <= t)
						lo = mid;
					else
						hi = mid - 1;
				}
				tv = lo;
				starting = true;
			}
			else
				working = false;
		}
		unsigned pending = __ballot_sync(0xffffffffu, starting);
		while (pending)
		{
			const int src = __ffs(pending) - 1;
			pending &= pending - 1u;
			const unsigned long long ts = __shfl_sync(0xffffffffu, t, src);
			const int vs = __shfl_sync(0xffffffffu, tv, src);
			const mb_variant& var = B.vars[vs];
			const NET net(B, var);
			const unsigned long long stream = var.first_traj + (ts - var.begin);
			mbb_lane c = v;
			const int off = (int)threadIdx.x - ((threadIdx.x & ~31) + src);
			c.st = v.st - off;
			c.un = v.un - off;
			c.ws = v.ws - off;
			mb_philox_initial_state(B.seed, stream, net.N(), var.istate, [&](int w, uint32_t word) {
				if (lane == 0)
					c.S(w) = word;
			});
			__syncwarp();
			unsigned long long gsx[MBB_GROUPS];
#pragma unroll
			for (int g = 0; g < MBB_GROUPS; g++)
				gsx[g] = 0;
			unsigned long long tot = 0;
			uint32_t ix = 0;
			const int wsh = net.wpg_shift(), ng = net.groups();
			for (int w = 0; w < net.W(); w++)
			{
				const int i = 32 * w + lane;
				const bool on = (c.S(w) >> lane) & 1u;
				bool unstable = false;
				uint32_t q = 0, nibit = 0;
				if (i < net.N())
				{
					const int r = __ldg(net.self() + i);
					const uint4 rec = __ldg(net.rec() + r);
					unstable = on != mbb_logic(net, c, r, rec);
					const uint2 qq = __ldg(var.q + i);
					q = unstable ? (on ? qq.y : qq.x) : 0u;
					const int pos = (int)((rec.x >> 21) & 31u) - 1;
					nibit = (pos >= 0 && on) ? (1u << pos) : 0u;
				}
				const uint32_t um = __ballot_sync(0xffffffffu, unstable);
				const uint32_t qw = __reduce_add_sync(0xffffffffu, q);
				ix |= __reduce_or_sync(0xffffffffu, nibit);
				if (lane == 0)
				{
					c.U(w) = um;
					c.Q(w) = qw;
				}
				mbb_group_add(gsx, w >> wsh, qw, ng);
				tot += qw;
			}
			__syncwarp();
			if (lane == src)
			{
#pragma unroll
				for (int g = 0; g < MBB_GROUPS; g++)
					gs[g] = gsx[g];
				total = tot;
				idx = ix;
			}
		}
		if (starting)
		{
			vi = tv;
			const mb_variant& var = B.vars[vi];
			const NET net(B, var);
			const unsigned long long stream = var.first_traj + (t - var.begin);
			curand_init(B.seed, stream, (unsigned long long)((net.N() + 3) & ~3), &rng);
			h = mbb_entropy(net, var, v);
			time = 0.f;
			running = true;
			if (acc_var != vi)
			{
				if (acc_var >= 0)
				{
					mb_acc_flush(acc, B.vars[acc_var].st, B.vars[acc_var].st.win_h);
					if (GRAD)
						mbb_grad_emit(B.vars[acc_var], v, P);
				}
				acc_var = vi;
				cc.w = -1;
			}
			if (GRAD)
			{
				C1 = C2 = 0.0;
				// d a0 / d theta of the initial state: every unstable node's active-direction derivatives
				for (int w = 0; w < net.W(); w++)
				{
					uint32_t um = v.U(w);
					const uint32_t sw = v.S(w);
					while (um)
					{
						const int b = __ffs(um) - 1;
						um &= um - 1u;
						mbb_grad_active(var, v, 32 * w + b, (sw >> b) & 1u, 1.f, 0.f, net.discrete(), C1, C2);
					}
				}
			}
		}

		// steps per pass of the work-fetch loop: several (as in the fast kernel) only in the
		// specialised gradient kernel (the gradient on the 50-node network 21.5 -> 20.6 ms); the
		// specialised forward kernel lost 3.5 % with them, and the ahead-of-time kernels spilled 62
		// bytes and halved the throughput of the 256-variant sweep
		for (int step = 0; step < (GRAD ? NET::steps_per_pass() : 1) && running; step++)
		{
			const mb_variant& var = B.vars[vi];
			const NET net(B, var);
			const bool discrete = net.discrete();
			const float max_time = net.max_time(), tick = net.tick();
			const uint4 rb = curand4(&rng);
			float tn;
			if (total == 0)
				tn = max_time;
			else
			{
				if (discrete)
				{
					tn = time + tick;
					tn = max_time - tick < tn ? max_time : tn;
				}
				else
				{
					const float u = (float)((rb.x >> 8) + 1u) * 5.9604644775390625e-8f;
					tn = time + -logf(u) / ((float)total * (1.0f / (float)(1u << var.rate_shift)));
				}
				tn = fminf(tn, max_time);
			}
			trans += (tn != 0.f) ? 1ull : 0ull;
			mbb_record<GRAD>(var, v, P, acc, idx, time, tn, total == 0 ? 0.f : h, discrete, var.st.win_tick, C1, C2, cc);
			time = tn;
			if (time >= max_time)
			{
				running = false;
				atomicAdd(var.st.final_cnt + idx, 1u);
				if (total == 0)
				{
					unsigned st[64];
					const int W = net.W() < 64 ? net.W() : 64;
					for (int w = 0; w < W; w++)
						st[w] = v.S(w);
					mb_fixed_insert_rt(var.st, st, W);
				}
				if (GRAD)
					mbb_grad_end(v, P, discrete, C1, C2);
				atomicAdd(var.transitions, trans);
				trans = 0;
			}
			else
			{
				const unsigned long long r = __umul64hi(((unsigned long long)rb.y << 32) | rb.z, total);
				const int wsh = net.wpg_shift(), wpg = 1 << wsh, ng = net.groups();
				// the first group whose prefix sum exceeds r: the number of the kept prefixes <= r
				// (r < total, the last kept prefix)
				unsigned long long cum = 0;
				int g = 0;
#pragma unroll
				for (int i = 0; i < MBB_GROUPS - 1; i++)
				{
					if (i + 1 >= ng)
						break;
					const bool le = gs[i] <= r;
					g += le ? 1 : 0;
					cum = le ? gs[i] : cum;
				}
				int word = g * wpg;
				for (int i = 0; i < wpg; i++)
				{
					const int w = g * wpg + i;
					if (w >= net.W())
						break;
					word = w;
					const uint32_t q = v.Q(w);
					if (r < cum + q)
						break;
					cum += q;
				}
				const uint32_t sw = v.S(word);
				uint32_t um = v.U(word);
				int j = 32 * word + 31 - __clz(um | 1u);
				while (um)
				{
					const int b = __ffs(um) - 1;
					const int i = 32 * word + b;
					const uint2 qq = __ldg(var.q + i);
					const uint32_t q = ((sw >> b) & 1u) ? qq.y : qq.x;
					j = i;
					if (r < cum + q)
						break;
					cum += q;
					um &= um - 1u;
				}
				const int jdir = (sw >> (j & 31)) & 1u; // 0: j switches on (up rate), 1: off (down rate)
				if (GRAD)
				{
					const float rj = __ldg(var.rate + 2 * j + jdir);
					const int a = __ldg(var.g_ptr + 2 * j + jdir), b = __ldg(var.g_ptr + 2 * j + jdir + 1);
					for (int e = a; e < b; e++)
					{
						const int p = __ldg(var.g_p + e);
						const float dA = __ldg(var.g_d + e) / rj;
						if (!discrete)
							mbb_red_add(v.GR(p), -(double)dA * C1);
						v.GS(p) += dA;
					}
					if (discrete)
					{
						const float a0 = (float)total * (1.0f / (float)(1u << var.rate_shift));
						for (int p = 0; p < P; p++)
							v.GS(p) -= v.GD(p) / a0;
					}
				}

				// flip j and re-evaluate it and the nodes whose logic reads it
				v.S(j >> 5) ^= 1u << (j & 31);
				const uint2 nj = __ldg(net.dep() + j);
				const int pj = (int)(nj.y >> 16) - 1;
				if (pj >= 0)
					idx ^= 1u << pj;
				bool ni_changed = pj >= 0;
				const int d0 = (int)nj.x, d1 = d0 + (int)(nj.y & 0xffffu);
				for (int d = d0; d < d1; d++)
				{
					const uint4 rec = __ldg(net.rec() + d);
					const int k = (int)(rec.x & 0xffffu);
					const int wk = k >> 5;
					const uint32_t bk = 1u << (k & 31);
					const bool on = (v.S(wk) & bk) != 0;
					const bool was_on = (k == j) ? !on : on;
					const uint32_t uw = v.U(wk);
					const bool was_unstable = (uw & bk) != 0;
					const bool unstable = on != mbb_logic(net, v, d, rec);
					const uint2 qq = __ldg(var.q + k);
					const uint32_t qo = was_unstable ? (was_on ? qq.y : qq.x) : 0u;
					const uint32_t qn = unstable ? (on ? qq.y : qq.x) : 0u;
					if (unstable != was_unstable)
						v.U(wk) = uw ^ bk;
					if (qn != qo)
					{
						const long long dq = (long long)qn - (long long)qo;
						v.Q(wk) += (uint32_t)dq;
						mbb_group_add(gs, wk >> wsh, dq, ng);
						total += (unsigned long long)dq;
					}
					if (GRAD && (unstable != was_unstable || on != was_on))
					{
						if (was_unstable)
							mbb_grad_active(var, v, k, was_on ? 1 : 0, -1.f, time, discrete, C1, C2);
						if (unstable)
							mbb_grad_active(var, v, k, on ? 1 : 0, 1.f, time, discrete, C1, C2);
					}
					if (qn != qo || unstable != was_unstable)
						ni_changed |= ((rec.x >> 21) & 31u) != 0u;
				}
				if (ni_changed)
					h = mbb_entropy(net, var, v);
			}
		}
		__syncwarp();
	}
	if (acc_var >= 0)
	{
		mb_acc_flush(acc, B.vars[acc_var].st, B.vars[acc_var].st.win_h);
		if (GRAD)
			mbb_grad_emit(B.vars[acc_var], v, P);
	}
}

#ifndef MB_FAMILY_BATCH
extern "C" __global__ void __launch_bounds__(128, 5) mb_batched_fast(mb_batch_params B) { mbb_body<false, mbb_net_rt>(B); }
extern "C" __global__ void __launch_bounds__(128, 5) mb_batched_grad(mb_batch_params B) { mbb_body<true, mbb_net_rt>(B); }
#else
// NVRTC build for a batch of one network (compiled together with that network's generated code):
// its structure is compile-time, its rates stay the variants' runtime tables.
struct mbb_net_static
{
	__device__ __forceinline__ mbb_net_static(const mb_batch_params&, const mb_variant&) {}
	__device__ __forceinline__ static constexpr int N() { return state_size; }
	__device__ __forceinline__ static constexpr int W() { return state_words; }
	__device__ __forceinline__ static constexpr int k() { return mbg_noninternal_count; }
	__device__ __forceinline__ static constexpr bool discrete() { return discrete_time; }
	__device__ __forceinline__ static constexpr float max_time() { return ::max_time; }
	__device__ __forceinline__ static constexpr float tick() { return time_tick; }
	__device__ __forceinline__ static constexpr int wpg_shift()
	{
		return state_words <= MBB_GROUPS ? 0 : state_words <= 2 * MBB_GROUPS ? 1 : state_words <= 4 * MBB_GROUPS ? 2 : 3;
	}
	// the register groups the kernel keeps: the network's own (compile-time loop bounds)
	__device__ __forceinline__ static constexpr int groups() { return (state_words + (1 << wpg_shift()) - 1) >> wpg_shift(); }
	__device__ __forceinline__ static constexpr int steps_per_pass() { return 4; }
	__device__ __forceinline__ static const uint2* dep() { return reinterpret_cast<const uint2*>(mbg_inc_dep); }
	__device__ __forceinline__ static const uint4* rec() { return mbg_inc_crec; }
	__device__ __forceinline__ static const uint4* ext() { return mbg_inc_cext; }
	__device__ __forceinline__ static const unsigned* tt() { return mbg_inc_tt; }
	__device__ __forceinline__ static const int* self() { return mbg_inc_self; }
	__device__ __forceinline__ static const int* ni_node() { return mbg_inc_ni_node; }
	// the same sums straight-line (generated code: constant node words and masks)
	template <class V>
	__device__ __forceinline__ static void ni_rate_sums(const V& v, const mb_variant& var, float& t, float& tl)
	{
		mbg_ni_rate_sums_var(v, var.rate, var.rlog, t, tl);
	}
};
extern "C" __global__ void __launch_bounds__(128, 5) mb_batched_fast_static(mb_batch_params B)
{
	mbb_body<false, mbb_net_static>(B);
}
extern "C" __global__ void __launch_bounds__(128, 5) mb_batched_grad_static(mb_batch_params B)
{
	mbb_body<true, mbb_net_static>(B);
}
#endif
