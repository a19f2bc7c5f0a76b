// Batched runs and score-function gradients (host side + ahead-of-time sm_100a kernels).
//
// A batch holds networks (parsed models whose rates have the @logic form) and parameter variants of
// them (variable values, trajectory count, random stream of trajectory 0). One persistent launch
// of mb_batched_fast / mb_batched_grad (kernels/batched.cuh) simulates every trajectory of every
// variant; each variant has its own window / final-state / fixed-point accumulators.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "batch.h"
#include "kernels/params.cuh"
#include "kernels/common.cuh"
#include "kernels/batched.cuh"

namespace mb {

namespace {

// compaction of one variant's fixed-point table into (state, count) records
__global__ void mbb_fixed_extract(unsigned cap, int words, const mb_key128* __restrict__ keys,
								  const unsigned* __restrict__ counts, const unsigned* __restrict__ states,
								  unsigned* __restrict__ out_n, unsigned* __restrict__ out_states,
								  unsigned* __restrict__ out_counts)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= cap)
		return;
	const mb_key128 k = keys[i];
	if (k.lo == 0ull && k.hi == 0ull)
		return;
	const unsigned o = atomicAdd(out_n, 1u);
	for (int w = 0; w < words; w++)
		out_states[(size_t)o * words + w] = states[(size_t)i * words + w];
	out_counts[o] = counts[i];
}

template <typename T>
void upload(dbuf& b, const std::vector<T>& v, cudaStream_t s)
{
	b.alloc(std::max<size_t>(1, v.size()) * sizeof(T));
	if (!v.empty())
		MB_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

float print6(float v)
{
	return (float)std::strtod(print_float(v).c_str(), nullptr);
}

} // namespace

batch_engine::batch_engine(context& c) : ctx(&c) {}
batch_engine::~batch_engine() = default;

int batch_engine::add_model(const model_t& m)
{
	auto net = std::make_unique<network>();
	net->model = m;
	net->L = analyze_model(m);
	const model_layout& L = net->L;
	if (!L.all_fast_path || !L.incremental_ok)
		throw engine_error(MB_ERR_INVALID, "batched runs need every rate in the form rate_up = @logic ? U : 0; "
										   "rate_down = @logic ? 0 : D with at most 12 logic inputs per node");
	if (L.state_words > 64)
		throw engine_error(MB_ERR_LIMIT, "batched runs support networks of at most 2048 nodes");
	if (L.noninternal_nodes.size() > 20)
		throw engine_error(MB_ERR_LIMIT, "more than 20 non-internal nodes");
	MB_CUDA(cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	const incremental_tables t = build_incremental_tables(L, L.up, L.down);
	upload(net->node, t.node, s);
	upload(net->hdr, t.hdr, s);
	upload(net->in1, t.in1, s);
	upload(net->in2, t.in2, s);
	upload(net->tt, t.tt, s);
	upload(net->self, t.self, s);
	upload(net->ni_node, L.noninternal_nodes, s);
	MB_CUDA(cudaStreamSynchronize(s));
	nets.push_back(std::move(net));
	return (int)nets.size() - 1;
}

int batch_engine::add_variant(int net, const std::map<std::string, float>& overrides, long long n_traj,
							  unsigned long long first_traj, const std::vector<std::string>& grad_params)
{
	if (net < 0 || net >= (int)nets.size())
		throw engine_error(MB_ERR_INVALID, "bad network index");
	if (n_traj < 0 || n_traj > 0xffffffffLL)
		throw engine_error(MB_ERR_LIMIT, "trajectories per variant must be in [0, 2^32)");
	network& N = *nets[net];
	auto var = std::make_unique<variant>();
	var->net = net;
	var->n_traj = n_traj;
	var->first_traj = first_traj;
	var->grad_params = grad_params;
	std::map<std::string, float> vars = N.model.variables;
	for (auto& kv : overrides)
	{
		if (!vars.count(kv.first))
			throw engine_error(MB_ERR_INVALID, "unknown variable " + kv.first);
		vars[kv.first] = kv.second;
	}
	const model_layout& L = N.L;
	if (overrides.empty() && grad_params.empty())
	{
		// the model's own values, exactly as the compiled single-model kernels see them
		var->rates.up = L.up;
		var->rates.down = L.down;
		var->rates.grad_ptr.assign(2 * L.state_size + 1, 0);
	}
	else
		var->rates = fast_rates(N.model, vars, grad_params);
	const incremental_tables t = build_incremental_tables(L, var->rates.up, var->rates.down);
	if (!t.ok)
		throw engine_error(MB_ERR_INVALID, "rates must be finite, non-negative, and positive rates within 2^20 of "
										   "the largest one");
	var->rate_shift = t.rate_shift;
	var->q = t.q;
	vars_.push_back(std::move(var));
	return (int)vars_.size() - 1;
}

void batch_engine::run(unsigned long long seed, const std::vector<std::vector<double>>* cotangents)
{
	MB_CUDA(cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	const bool grad = cotangents != nullptr;
	int max_W = 1, P = 0;
	std::vector<mb_net> hnets(nets.size());
	for (size_t i = 0; i < nets.size(); i++)
	{
		network& N = *nets[i];
		const model_layout& L = N.L;
		mb_net& d = hnets[i];
		d.N = L.state_size;
		d.W = L.state_words;
		d.k = (int)L.noninternal_nodes.size();
		d.discrete = L.discrete_time ? 1 : 0;
		d.max_time = print6(L.max_time); // the generated code's 6-digit constants
		d.tick = print6(L.time_tick);
		d.node = N.node.as<uint4>();
		d.hdr = N.hdr.as<uint4>();
		d.in1 = N.in1.as<uint4>();
		d.in2 = N.in2.as<uint4>();
		d.tt = N.tt.as<unsigned>();
		d.self = N.self.as<int>();
		d.ni_node = N.ni_node.as<int>();
		max_W = std::max(max_W, d.W);
	}
	std::vector<mb_variant> hvars(vars_.size());
	unsigned long long begin = 0;
	for (size_t i = 0; i < vars_.size(); i++)
	{
		variant& V = *vars_[i];
		const model_layout& L = nets[V.net]->L;
		if (grad)
		{
			if ((*cotangents)[i].size() != (size_t)L.windows() << L.noninternal_nodes.size())
				throw engine_error(MB_ERR_INVALID, "cotangent must have windows * 2^k entries");
			P = std::max(P, (int)V.grad_params.size());
		}
		V.st.init_plain(L.state_words, L.time_tick, L.max_time, L.discrete_time, L.noninternal_nodes, V.n_traj, s);
		std::vector<uint2> q2(L.state_size);
		for (int n = 0; n < L.state_size; n++)
			q2[n] = make_uint2(V.q[2 * n], V.q[2 * n + 1]);
		std::vector<float> rate(2 * L.state_size);
		for (int n = 0; n < L.state_size; n++)
		{
			rate[2 * n] = V.rates.up[n];
			rate[2 * n + 1] = V.rates.down[n];
		}
		upload(V.d_q, q2, s);
		upload(V.d_rate, rate, s);
		upload(V.d_istate, L.istate, s);
		upload(V.d_gptr, V.rates.grad_ptr, s);
		upload(V.d_gp, V.rates.grad_p, s);
		upload(V.d_gd, V.rates.grad_d, s);
		V.d_counters.alloc(16);
		MB_CUDA(cudaMemsetAsync(V.d_counters.p, 0, 16, s));
		V.d_grad.alloc(std::max<size_t>(1, V.grad_params.size()) * sizeof(double));
		MB_CUDA(cudaMemsetAsync(V.d_grad.p, 0, V.d_grad.bytes, s));
		if (grad)
			upload(V.d_cot, (*cotangents)[i], s);
		mb_variant& d = hvars[i];
		d.net = V.net;
		d.rate_shift = V.rate_shift;
		d.q = V.d_q.as<uint2>();
		d.rate = V.d_rate.as<float>();
		d.istate = V.d_istate.as<float>();
		d.begin = begin;
		d.first_traj = V.first_traj;
		d.n_traj = (unsigned)V.n_traj;
		d.st = V.st.p;
		d.transitions = V.d_counters.as<unsigned long long>();
		d.cot = grad ? V.d_cot.as<double>() : nullptr;
		d.g_ptr = V.d_gptr.as<int>();
		d.g_p = V.d_gp.as<int>();
		d.g_d = V.d_gd.as<float>();
		d.grad = V.d_grad.as<double>();
		begin += (unsigned long long)V.n_traj;
	}
	upload(d_nets, hnets, s);
	upload(d_vars, hvars, s);
	dbuf counters(64);
	MB_CUDA(cudaMemsetAsync(counters.p, 0, 64, s));

	mb_batch_params B{};
	B.nets = d_nets.as<mb_net>();
	B.vars = d_vars.as<mb_variant>();
	B.n_vars = (int)hvars.size();
	B.max_W = max_W;
	B.P = P;
	B.total = begin;
	B.seed = seed;
	B.next = counters.as<unsigned long long>();
	B.errors = counters.as<unsigned>() + 4;
	const void* fn = grad ? (const void*)mb_batched_grad : (const void*)mb_batched_fast;
	int block = 128;
	auto smem_of = [&](int b) { return (size_t)b * (3 * (size_t)max_W + (grad ? 4 * (size_t)P : 0)) * 4; };
	constexpr size_t max_smem = 227 * 1024;
	while (block > 32 && smem_of(block) > max_smem)
		block -= 32;
	if (smem_of(block) > max_smem)
		throw engine_error(MB_ERR_LIMIT, "batch too large for shared memory (state words, gradient parameters)");
	const size_t smem = smem_of(block);
	if (smem > 48 * 1024)
		MB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	int per_sm = 0;
	MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem));
	per_sm = std::max(per_sm, 1);
	const unsigned long long needed = (begin + block - 1) / block;
	const unsigned grid = (unsigned)std::max<unsigned long long>(
		1ull, std::min<unsigned long long>(needed, (unsigned long long)per_sm * ctx->sm_count));
	cudaEvent_t e0, e1;
	MB_CUDA(cudaEventCreate(&e0));
	MB_CUDA(cudaEventCreate(&e1));
	MB_CUDA(cudaEventRecord(e0, s));
	if (begin > 0)
	{
		void* args[] = { &B };
		MB_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(block), args, smem, s));
	}
	MB_CUDA(cudaEventRecord(e1, s));
	MB_CUDA(cudaEventSynchronize(e1));
	MB_CUDA(cudaEventElapsedTime(&kernel_ms, e0, e1));
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	last_block = block;
	last_grid = grid;

	// results
	for (size_t i = 0; i < vars_.size(); i++)
	{
		variant& V = *vars_[i];
		const network& N = *nets[V.net];
		V.res = V.st.finalize_plain(V.n_traj, N.L.state_size, s);
		unsigned long long trans = 0;
		MB_CUDA(cudaMemcpy(&trans, V.d_counters.p, sizeof trans, cudaMemcpyDeviceToHost));
		V.res->transitions = trans;
		V.res->kernel_ms = kernel_ms;
		V.grad.assign(V.grad_params.size(), 0.0);
		if (grad && !V.grad_params.empty())
		{
			MB_CUDA(cudaMemcpy(V.grad.data(), V.d_grad.p, V.grad.size() * sizeof(double), cudaMemcpyDeviceToHost));
			// probabilities are occupancy / (n * tick) (continuous) or count / n (discrete)
			const double scale = 1.0 / ((double)std::max(1LL, V.n_traj) *
										(N.L.discrete_time ? 1.0 : (double)N.L.time_tick));
			for (double& g : V.grad)
				g *= scale;
		}
	}
}

// ---- per-variant accumulators (same layout and fixed-point scales as stats_state)

void plain_stats::init_plain(int words, float tick, float tmax, bool discrete, const std::vector<int>& noninternal,
							 long long n, cudaStream_t s)
{
	W = words;
	const int k = (int)noninternal.size();
	const float q = tmax / tick;
	n_windows = (int)std::ceil((double)q);
	n_bins = 1u << k;
	discrete_time = discrete;
	time_tick = tick;
	max_time = tmax;
	noninternal_nodes = noninternal;
	fx = std::ldexp(1.0, occupancy_exponent(n, tick, discrete));
	fx_h = std::ldexp(1.0, entropy_exponent(n, tick, discrete));
	const size_t cells = (size_t)n_windows * n_bins;
	occ.alloc(discrete ? 8 : cells * sizeof(long long));
	cnt.alloc(discrete ? cells * sizeof(unsigned) : 4);
	h.alloc(n_windows * sizeof(long long));
	fin.alloc(n_bins * sizeof(unsigned));
	unsigned cap = 1024;
	while (cap < 2 * std::min<long long>(std::max(n, 1LL), 1LL << 22))
		cap <<= 1;
	fp_cap = cap;
	fp_keys.alloc((size_t)cap * sizeof(mb_key128));
	fp_counts.alloc((size_t)cap * sizeof(unsigned));
	fp_states.alloc((size_t)cap * W * sizeof(unsigned));
	counters.alloc(64);
	MB_CUDA(cudaMemsetAsync(occ.p, 0, occ.bytes, s));
	MB_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
	MB_CUDA(cudaMemsetAsync(h.p, 0, h.bytes, s));
	MB_CUDA(cudaMemsetAsync(fin.p, 0, fin.bytes, s));
	MB_CUDA(cudaMemsetAsync(fp_keys.p, 0, fp_keys.bytes, s));
	MB_CUDA(cudaMemsetAsync(fp_counts.p, 0, fp_counts.bytes, s));
	MB_CUDA(cudaMemsetAsync(counters.p, 0, counters.bytes, s));
	p = mb_stats_params{};
	p.n_windows = n_windows;
	p.n_bins = n_bins;
	p.win_tick = tick;
	p.h_in_smem = 0;
	p.fx = fx;
	p.fx_h = fx_h;
	p.win_occ = occ.as<long long>();
	p.win_cnt = cnt.as<unsigned>();
	p.win_h = h.as<long long>();
	p.final_cnt = fin.as<unsigned>();
	p.fp_keys = fp_keys.as<mb_key128>();
	p.fp_counts = fp_counts.as<unsigned>();
	p.fp_states = fp_states.as<unsigned>();
	p.fp_mask = cap - 1;
	p.fp_overflow = counters.as<unsigned>();
}

std::unique_ptr<result> plain_stats::finalize_plain(long long n, int state_size, cudaStream_t s)
{
	auto r = std::make_unique<result>();
	r->state_size = state_size;
	r->state_words = W;
	r->n_windows = n_windows;
	r->n_bins = n_bins;
	r->n_traj = n;
	r->discrete_time = discrete_time;
	r->time_tick = time_tick;
	r->max_time = max_time;
	r->noninternal_nodes = noninternal_nodes;
	r->fx = fx;
	r->fx_h = fx_h;
	const size_t cells = (size_t)n_windows * n_bins;
	if (discrete_time)
	{
		r->win_cnt.resize(cells);
		MB_CUDA(cudaMemcpyAsync(r->win_cnt.data(), cnt.p, cells * 4, cudaMemcpyDeviceToHost, s));
	}
	else
	{
		r->win_occ.resize(cells);
		MB_CUDA(cudaMemcpyAsync(r->win_occ.data(), occ.p, cells * 8, cudaMemcpyDeviceToHost, s));
	}
	r->win_h.resize(n_windows);
	MB_CUDA(cudaMemcpyAsync(r->win_h.data(), h.p, n_windows * 8, cudaMemcpyDeviceToHost, s));
	r->final_cnt.resize(n_bins);
	MB_CUDA(cudaMemcpyAsync(r->final_cnt.data(), fin.p, n_bins * 4, cudaMemcpyDeviceToHost, s));
	dbuf on((size_t)fp_cap * W * 4), oc((size_t)fp_cap * 4);
	unsigned* out_n = counters.as<unsigned>() + 1;
	mbb_fixed_extract<<<(fp_cap + 255) / 256, 256, 0, s>>>(fp_cap, W, p.fp_keys, p.fp_counts, p.fp_states, out_n,
														  on.as<unsigned>(), oc.as<unsigned>());
	MB_CUDA(cudaGetLastError());
	unsigned ctr[2] = { 0, 0 };
	MB_CUDA(cudaMemcpyAsync(ctr, counters.p, sizeof ctr, cudaMemcpyDeviceToHost, s));
	MB_CUDA(cudaStreamSynchronize(s));
	r->fixed_overflow = ctr[0];
	const unsigned nfp = ctr[1];
	std::vector<unsigned> st((size_t)nfp * W), cn(nfp);
	if (nfp)
	{
		MB_CUDA(cudaMemcpy(st.data(), on.p, st.size() * 4, cudaMemcpyDeviceToHost));
		MB_CUDA(cudaMemcpy(cn.data(), oc.p, cn.size() * 4, cudaMemcpyDeviceToHost));
	}
	std::vector<unsigned> order(nfp);
	std::iota(order.begin(), order.end(), 0u);
	std::sort(order.begin(), order.end(), [&](unsigned a, unsigned b) {
		for (int w = W - 1; w >= 0; w--)
		{
			const unsigned x = st[(size_t)a * W + w], y = st[(size_t)b * W + w];
			if (x != y)
				return x < y;
		}
		return false;
	});
	r->fixed_states.resize((size_t)nfp * W);
	r->fixed_counts.resize(nfp);
	for (unsigned i = 0; i < nfp; i++)
	{
		std::copy(st.begin() + (size_t)order[i] * W, st.begin() + (size_t)(order[i] + 1) * W,
				  r->fixed_states.begin() + (size_t)i * W);
		r->fixed_counts[i] = cn[order[i]];
	}
	return r;
}

} // namespace mb
