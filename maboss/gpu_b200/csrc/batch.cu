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
#include <cstring>
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
	// a buffer that is large enough is kept: descriptors and captured graphs hold its address
	const size_t need = std::max<size_t>(1, v.size()) * sizeof(T);
	if (b.bytes < need)
		b.alloc(need);
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
	std::vector<unsigned> dep;
	for (size_t i = 0; i + 3 < t.node.size(); i += 4)
	{
		dep.push_back(t.node[i + 2]);
		dep.push_back(t.node[i + 3]);
	}
	upload(net->dep, dep, s);
	upload(net->rec, t.crec, s);
	upload(net->ext, t.cext, s);
	upload(net->tt, t.tt, s);
	upload(net->self, t.self, s);
	upload(net->ni_node, L.noninternal_nodes, s);
	MB_CUDA(cudaStreamSynchronize(s));
	invalidate();
	nets.push_back(std::move(net));
	return (int)nets.size() - 1;
}

int batch_engine::add_variant(int net, const std::map<std::string, float>& overrides, long long n_traj,
							  unsigned long long first_traj, const std::vector<std::string>& grad_params,
							  const std::map<std::string, bool>& mutants)
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
	for (auto& kv : overrides)
		if (!N.model.variables.count(kv.first))
			throw engine_error(MB_ERR_INVALID, "unknown variable " + kv.first);
	var->overrides = overrides;
	for (auto& [name, on] : mutants)
	{
		const int i = N.model.node_index(name);
		if (i < 0)
			throw engine_error(MB_ERR_INVALID, "unknown node " + name);
		var->mutants[i] = on;
	}
	var->istate = N.L.istate;
	for (auto& [i, on] : var->mutants)
		var->istate[i] = on ? 1.f : 0.f;
	compute_rates(*var);
	invalidate();
	vars_.push_back(std::move(var));
	return (int)vars_.size() - 1;
}

// Rates, their derivatives and the integer rate tables of a variant from its variable values.
void batch_engine::compute_rates(variant& V) const
{
	const network& N = *nets[V.net];
	const model_layout& L = N.L;
	if (V.overrides.empty() && V.grad_params.empty())
	{
		// the model's own values, exactly as the compiled single-model kernels see them
		V.rates = rate_set{};
		V.rates.up = L.up;
		V.rates.down = L.down;
		V.rates.grad_ptr.assign(2 * L.state_size + 1, 0);
	}
	else
	{
		std::map<std::string, float> vars = N.model.variables;
		for (auto& kv : V.overrides)
			vars[kv.first] = kv.second;
		V.rates = fast_rates(N.model, vars, V.grad_params);
	}
	if (!V.mutants.empty())
	{
		// a mutant node never changes (forced by its initial state): both rates 0, no derivatives
		for (auto& [i, on] : V.mutants)
			V.rates.up[i] = V.rates.down[i] = 0.f;
		rate_set r = V.rates;
		r.grad_ptr.assign(1, 0);
		r.grad_p.clear();
		r.grad_d.clear();
		for (int e = 0; e < 2 * L.state_size; e++)
		{
			if (!V.mutants.count(e / 2))
				for (int k = V.rates.grad_ptr[e]; k < V.rates.grad_ptr[e + 1]; k++)
				{
					r.grad_p.push_back(V.rates.grad_p[k]);
					r.grad_d.push_back(V.rates.grad_d[k]);
				}
			r.grad_ptr.push_back((int)r.grad_p.size());
		}
		V.rates = std::move(r);
	}
	const incremental_tables t = build_incremental_tables(L, V.rates.up, V.rates.down);
	if (!t.ok)
		throw engine_error(MB_ERR_INVALID, "rates must be finite and non-negative, with every positive rate at least "
										   "2^20 units of the fixed point in which each state word's rate sum stays "
										   "below 2^32 (rates within a factor of about 4096 of a word's rate sum)");
	V.rate_shift = t.rate_shift;
	V.q = t.q;
}

// The parameter-dependent device tables of a variant (integer rates, float rates, r log2 r, rate
// derivatives), into its buffers (kept when large enough).
void batch_engine::upload_tables(variant& V, cudaStream_t s)
{
	const model_layout& L = nets[V.net]->L;
	std::vector<uint2> q2(L.state_size);
	for (int n = 0; n < L.state_size; n++)
		q2[n] = make_uint2(V.q[2 * n], V.q[2 * n + 1]);
	std::vector<float> rate(2 * L.state_size), rlog(2 * L.state_size);
	for (int n = 0; n < L.state_size; n++)
	{
		rate[2 * n] = V.rates.up[n];
		rate[2 * n + 1] = V.rates.down[n];
	}
	// r log2 r of the entropy, as the generated tables of the NVRTC kernels compute it
	for (int e = 0; e < 2 * L.state_size; e++)
	{
		const double r = rate[e];
		rlog[e] = r > 0 ? (float)(r * std::log2(r)) : 0.f;
	}
	upload(V.d_q, q2, s);
	upload(V.d_rate, rate, s);
	upload(V.d_rlog, rlog, s);
	upload(V.d_gptr, V.rates.grad_ptr, s);
	upload(V.d_gp, V.rates.grad_p, s);
	upload(V.d_gd, V.rates.grad_d, s);
}

void batch_engine::set_variables(int v, const std::map<std::string, float>& values)
{
	if (v < 0 || v >= (int)vars_.size())
		throw engine_error(MB_ERR_INVALID, "bad variant index");
	variant& V = *vars_[v];
	const network& N = *nets[V.net];
	for (auto& kv : values)
		if (!N.model.variables.count(kv.first))
			throw engine_error(MB_ERR_INVALID, "unknown variable " + kv.first);
	const std::map<std::string, float> before = V.overrides;
	for (auto& kv : values)
		V.overrides[kv.first] = kv.second;
	try
	{
		compute_rates(V);
	}
	catch (...)
	{
		V.overrides = before;
		compute_rates(V);
		throw;
	}
	if (!V.ready)
		return; // uploaded by the first prepare
	MB_CUDA(cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	upload_tables(V, s);
	for (auto& ps : prep)
		if (ps)
		{
			mb_variant& d = ps->hvars[v];
			d.rate_shift = V.rate_shift;
			d.q = V.d_q.as<uint2>();
			d.rate = V.d_rate.as<float>();
			d.rlog = V.d_rlog.as<float>();
			d.g_ptr = V.d_gptr.as<int>();
			d.g_p = V.d_gp.as<int>();
			d.g_d = V.d_gd.as<float>();
			upload(ps->d_vars, ps->hvars, s); // same size: same address, so graphs stay valid
		}
	MB_CUDA(cudaStreamSynchronize(s));
}

void batch_engine::invalidate()
{
	for (auto& ps : prep)
		ps.reset();
}

batch_engine::prepared::~prepared()
{
	if (exec)
		cudaGraphExecDestroy(exec);
	if (graph)
		cudaGraphDestroy(graph);
	if (e0)
		cudaEventDestroy(e0);
	if (e1)
		cudaEventDestroy(e1);
	if (host)
		cudaFreeHost(host);
}

// Device descriptors, per-variant accumulators, extraction buffers and the pinned host arena of one
// kind of run (forward or gradient); built once and reused until the batch changes.
batch_engine::prepared& batch_engine::prepare(bool grad)
{
	std::unique_ptr<prepared>& slot = prep[grad ? 1 : 0];
	if (slot)
		return *slot;
	MB_CUDA(cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	auto ps = std::make_unique<prepared>();
	ps->grad = grad;
	int max_W = 1, P = 0;
	std::vector<mb_net> hnets(nets.size());
	for (size_t i = 0; i < nets.size(); i++)
	{
		network& N = *nets[i];
		const model_layout& L = N.L;
		mb_net& d = hnets[i];
		d.N = L.state_size;
		d.W = L.state_words;
		// words per register group sum: the smallest power of two >= ceil(W / MBB_GROUPS), so that
		// the kernel finds a word's group with a shift
		d.wpg_shift = 0;
		while ((1 << d.wpg_shift) * MBB_GROUPS < d.W)
			d.wpg_shift++;
		d.k = (int)L.noninternal_nodes.size();
		d.discrete = L.discrete_time ? 1 : 0;
		d.max_time = print6(L.max_time); // the generated code's 6-digit constants
		d.tick = print6(L.time_tick);
		d.dep = N.dep.as<uint2>();
		d.rec = N.rec.as<uint4>();
		d.ext = N.ext.as<uint4>();
		d.tt = N.tt.as<unsigned>();
		d.self = N.self.as<int>();
		d.ni_node = N.ni_node.as<int>();
		max_W = std::max(max_W, d.W);
	}
	std::vector<mb_variant> hvars(vars_.size());
	unsigned long long begin = 0;
	size_t host_bytes = 0;
	ps->host_off.resize(vars_.size());
	for (size_t i = 0; i < vars_.size(); i++)
	{
		variant& V = *vars_[i];
		const model_layout& L = nets[V.net]->L;
		if (grad)
			P = std::max(P, (int)V.grad_params.size());
		if (!V.ready)
		{
			// created once: the other kind of run (forward / gradient) shares these buffers
			V.st.init_plain(L.state_words, L.time_tick, L.max_time, L.discrete_time, L.noninternal_nodes, V.n_traj,
							s);
			upload(V.d_istate, V.istate, s);
			V.d_counters.alloc(16);
			V.d_grad.alloc(std::max<size_t>(1, V.grad_params.size()) * sizeof(double));
			V.d_cot.alloc((size_t)L.windows() * ((size_t)1 << L.noninternal_nodes.size()) * sizeof(double));
			V.out_states.alloc((size_t)V.st.fp_cap * L.state_words * 4);
			V.out_counts.alloc((size_t)V.st.fp_cap * 4);
			upload_tables(V, s);
			V.ready = true;
		}
		mb_variant& d = hvars[i];
		d.net = V.net;
		d.rate_shift = V.rate_shift;
		d.q = V.d_q.as<uint2>();
		d.rate = V.d_rate.as<float>();
		d.rlog = V.d_rlog.as<float>();
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
		// pinned host arena: windows, entropy sums, final counts, stats counters, transitions, gradient
		host_off_t& o = ps->host_off[i];
		o.win = host_bytes;
		host_bytes += V.st.occ.bytes > 8 ? V.st.occ.bytes : V.st.cnt.bytes;
		o.h = host_bytes;
		host_bytes += V.st.h.bytes;
		o.fin = host_bytes;
		host_bytes += (V.st.fin.bytes + 7) / 8 * 8;
		o.ctr = host_bytes;
		host_bytes += 8;
		o.trans = host_bytes;
		host_bytes += 8;
		o.grad = host_bytes;
		host_bytes += V.d_grad.bytes;
	}
	upload(ps->d_nets, hnets, s);
	upload(ps->d_vars, hvars, s);
	ps->hvars = hvars;
	ps->counters.alloc(64);
	MB_CUDA(cudaHostAlloc(&ps->host, std::max<size_t>(host_bytes, 8), cudaHostAllocDefault));
	MB_CUDA(cudaEventCreate(&ps->e0));
	MB_CUDA(cudaEventCreate(&ps->e1));
	ps->B = std::make_unique<mb_batch_params>();
	mb_batch_params& B = *ps->B;
	B.nets = ps->d_nets.as<mb_net>();
	B.vars = ps->d_vars.as<mb_variant>();
	B.n_vars = (int)hvars.size();
	B.max_W = max_W;
	B.P = P;
	B.total = begin;
	B.next = ps->counters.as<unsigned long long>();
	B.errors = ps->counters.as<unsigned>() + 4;
	ps->fn = grad ? (const void*)mb_batched_grad : (const void*)mb_batched_fast;
	if (specialize && nets.size() == 1)
	{
		network& N = *nets[0];
		if (!N.mod)
			N.mod = compile_batch_module(*ctx, generate_code(N.model));
		N.mod->ensure(FAMILY_BATCH);
		ps->fn = grad ? N.mod->batched_grad_static : N.mod->batched_fast_static;
	}
	ps->smem_per_thread = (3 * (size_t)max_W + (grad ? 2 * (size_t)P : 0)) * 4;
	MB_CUDA(cudaStreamSynchronize(s));
	slot = std::move(ps);
	return *slot;
}

// Blocks per SM that fit a launch shape, and the shared memory of a block.
int batch_engine::fit(prepared& ps, int block, size_t& smem) const
{
	constexpr size_t max_smem = 227 * 1024;
	smem = (size_t)block * ps.smem_per_thread;
	if (smem > max_smem)
		return 0;
	if (smem > 48 * 1024)
		MB_CUDA(cudaFuncSetAttribute(ps.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	MB_CUDA(cudaFuncSetAttribute(ps.fn, cudaFuncAttributePreferredSharedMemoryCarveout, -1));
	int per_sm = 0;
	MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ps.fn, block, smem));
	return per_sm;
}

void batch_engine::set_shape(prepared& ps, int block, int per_sm)
{
	size_t smem = 0;
	const int max_per_sm = fit(ps, block, smem);
	if (max_per_sm < 1)
		throw engine_error(MB_ERR_LIMIT, "batch too large for shared memory (state words, gradient parameters)");
	per_sm = per_sm > 0 ? std::min(per_sm, max_per_sm) : max_per_sm;
	// fewer blocks than fit leave the rest of the SM's L1/shared memory to L1 (the network tables)
	const int carve = per_sm < max_per_sm ? std::min(100, (int)((per_sm * (smem + 1024) * 100 + 228 * 1024 - 1) /
																 (228 * 1024)))
										  : -1;
	MB_CUDA(cudaFuncSetAttribute(ps.fn, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
	const unsigned long long needed = (ps.B->total + block - 1) / block;
	ps.block = block;
	ps.per_sm = per_sm;
	ps.smem = smem;
	ps.grid = (unsigned)std::max<unsigned long long>(
		1ull, std::min<unsigned long long>(needed, (unsigned long long)per_sm * ctx->sm_count));
	// gradient runs: the lanes' global scratch (partial products R_p, P doubles each)
	ps.B->gstride = ps.grid * (unsigned)block;
	const size_t gbytes = ps.grad ? (size_t)ps.B->P * ps.B->gstride * sizeof(double) : 0;
	if (ps.gscratch.bytes < gbytes)
		ps.gscratch.alloc(gbytes);
	ps.B->gmem = ps.gscratch.as<double>();
	if (ps.exec)
	{
		cudaGraphExecDestroy(ps.exec);
		ps.exec = nullptr;
	}
	if (ps.graph)
	{
		cudaGraphDestroy(ps.graph);
		ps.graph = nullptr;
	}
}

// Everything one run does on the device, in stream order: clear the accumulators, the persistent
// kernel between the two timing events, per-variant compaction of the fixed points, copies of every
// statistic into the pinned arena. Capturable as one CUDA graph (no allocation, no host sync).
void batch_engine::enqueue(prepared& ps, cudaStream_t s, bool capturing)
{
	// inside a capture the timing events must become event-record nodes of the graph
	auto record = [&](cudaEvent_t e) {
		if (capturing)
			MB_CUDA(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal));
		else
			MB_CUDA(cudaEventRecord(e, s));
	};
	for (auto& vp : vars_)
	{
		variant& V = *vp;
		V.st.zero(s);
		MB_CUDA(cudaMemsetAsync(V.d_counters.p, 0, V.d_counters.bytes, s));
		MB_CUDA(cudaMemsetAsync(V.d_grad.p, 0, V.d_grad.bytes, s));
	}
	MB_CUDA(cudaMemsetAsync(ps.counters.p, 0, ps.counters.bytes, s));
	record(ps.e0);
	if (ps.B->total > 0)
	{
		void* args[] = { ps.B.get() };
		MB_CUDA(cudaLaunchKernel(ps.fn, dim3(ps.grid), dim3(ps.block), args, ps.smem, s));
		if (capturing)
		{
			// the node just captured is the kernel's: later runs update its parameter block (the
			// seed) in the instantiated graph. Taken from the capture itself, because
			// cudaGraphKernelNodeGetParams does not describe nodes of library kernels (cudaKernel_t).
			cudaStreamCaptureStatus st;
			const cudaGraphNode_t* deps = nullptr;
			size_t ndeps = 0;
			MB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, nullptr, &deps, &ndeps));
			ps.kernel = ndeps == 1 ? deps[0] : nullptr;
		}
	}
	record(ps.e1);
	char* host = static_cast<char*>(ps.host);
	for (size_t i = 0; i < vars_.size(); i++)
	{
		variant& V = *vars_[i];
		const host_off_t& o = ps.host_off[i];
		V.st.extract(s, V.out_states.as<unsigned>(), V.out_counts.as<unsigned>());
		dbuf& win = V.st.occ.bytes > 8 ? V.st.occ : V.st.cnt;
		MB_CUDA(cudaMemcpyAsync(host + o.win, win.p, win.bytes, cudaMemcpyDeviceToHost, s));
		MB_CUDA(cudaMemcpyAsync(host + o.h, V.st.h.p, V.st.h.bytes, cudaMemcpyDeviceToHost, s));
		MB_CUDA(cudaMemcpyAsync(host + o.fin, V.st.fin.p, V.st.fin.bytes, cudaMemcpyDeviceToHost, s));
		MB_CUDA(cudaMemcpyAsync(host + o.ctr, V.st.counters.p, 8, cudaMemcpyDeviceToHost, s));
		MB_CUDA(cudaMemcpyAsync(host + o.trans, V.d_counters.p, 8, cudaMemcpyDeviceToHost, s));
		MB_CUDA(cudaMemcpyAsync(host + o.grad, V.d_grad.p, V.d_grad.bytes, cudaMemcpyDeviceToHost, s));
	}
}

// Times the candidate launch shapes on the batch itself (one run each after a warm-up run) and keeps
// the fastest: block sizes of 128, 96 and 64 threads, each with the most resident blocks per SM that
// fit and with one block fewer (which leaves more L1 to the network tables).
void batch_engine::tune(prepared& ps, cudaStream_t s)
{
	std::vector<std::pair<int, int>> cands;
	for (int block : { 128, 96, 64 })
	{
		size_t smem = 0;
		const int per_sm = fit(ps, block, smem);
		if (per_sm >= 1)
			cands.push_back({ block, per_sm });
		if (per_sm >= 2)
			cands.push_back({ block, per_sm - 1 });
	}
	if (cands.empty())
		throw engine_error(MB_ERR_LIMIT, "batch too large for shared memory (state words, gradient parameters)");
	float best = 0.f;
	std::pair<int, int> pick = cands[0];
	for (size_t c = 0; c < cands.size(); c++)
	{
		set_shape(ps, cands[c].first, cands[c].second);
		if (c == 0)
		{
			enqueue(ps, s, false); // warm-up (first-launch costs)
			MB_CUDA(cudaStreamSynchronize(s));
		}
		enqueue(ps, s, false);
		MB_CUDA(cudaStreamSynchronize(s));
		float ms = 0.f;
		MB_CUDA(cudaEventElapsedTime(&ms, ps.e0, ps.e1));
		tuning.push_back({ ps.grad, cands[c].first, cands[c].second, ms });
		if (c == 0 || ms < best)
		{
			best = ms;
			pick = cands[c];
		}
	}
	set_shape(ps, pick.first, pick.second);
}

void batch_engine::run(unsigned long long seed, const std::vector<std::vector<double>>* cotangents)
{
	MB_CUDA(cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	const bool grad = cotangents != nullptr;
	prepared& ps = prepare(grad);
	if (grad)
		for (size_t i = 0; i < vars_.size(); i++)
		{
			variant& V = *vars_[i];
			const model_layout& L = nets[V.net]->L;
			if ((*cotangents)[i].size() != (size_t)L.windows() << L.noninternal_nodes.size())
				throw engine_error(MB_ERR_INVALID, "cotangent must have windows * 2^k entries");
			MB_CUDA(cudaMemcpyAsync(V.d_cot.p, (*cotangents)[i].data(), V.d_cot.bytes, cudaMemcpyHostToDevice, s));
		}
	ps.B->seed = seed;
	if (ps.block == 0)
	{
		if (autotune && ps.B->total > 0)
			tune(ps, s);
		else
			set_shape(ps, 128, 0);
	}
	if (use_graph)
	{
		if (!ps.exec)
		{
			cudaGraph_t g = nullptr;
			MB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
			enqueue(ps, s, true);
			MB_CUDA(cudaStreamEndCapture(s, &g));
			ps.graph = g;
			MB_CUDA(cudaGraphInstantiate(&ps.exec, g, 0));
			size_t n_nodes = 0;
			MB_CUDA(cudaGraphGetNodes(g, nullptr, &n_nodes));
			graph_nodes = (unsigned)n_nodes;
			if (!ps.kernel && ps.B->total > 0)
				throw engine_error(MB_ERR_CUDA, "batch graph: the kernel node was not found in the capture");
		}
		if (ps.kernel)
		{
			// this run's seed: the kernel node's parameter block
			cudaKernelNodeParams kp{};
			void* args[] = { ps.B.get() };
			kp.func = const_cast<void*>(ps.fn);
			kp.gridDim = dim3(ps.grid);
			kp.blockDim = dim3(ps.block);
			kp.sharedMemBytes = (unsigned)ps.smem;
			kp.kernelParams = args;
			MB_CUDA(cudaGraphExecKernelNodeSetParams(ps.exec, ps.kernel, &kp));
		}
		MB_CUDA(cudaGraphLaunch(ps.exec, s));
	}
	else
		enqueue(ps, s, false);
	MB_CUDA(cudaStreamSynchronize(s));
	MB_CUDA(cudaEventElapsedTime(&kernel_ms, ps.e0, ps.e1));
	last_block = ps.block;
	last_grid = ps.grid;
	last_per_sm = ps.per_sm;

	// results from the pinned arena (fixed-point records: one copy of the occupied ones)
	const char* host = static_cast<const char*>(ps.host);
	for (size_t i = 0; i < vars_.size(); i++)
	{
		variant& V = *vars_[i];
		const network& N = *nets[V.net];
		const host_off_t& o = ps.host_off[i];
		V.res = V.st.result_from(host + o.win, host + o.h, host + o.fin, host + o.ctr, V.out_states.as<unsigned>(),
								 V.out_counts.as<unsigned>(), V.n_traj, N.L.state_size);
		unsigned long long trans = 0;
		std::memcpy(&trans, host + o.trans, sizeof trans);
		V.res->transitions = trans;
		V.res->kernel_ms = kernel_ms;
		V.grad.assign(V.grad_params.size(), 0.0);
		if (grad && !V.grad_params.empty())
		{
			std::memcpy(V.grad.data(), host + o.grad, V.grad.size() * sizeof(double));
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
	zero(s);
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

void plain_stats::zero(cudaStream_t s)
{
	for (dbuf* b : { &occ, &cnt, &h, &fin, &fp_keys, &fp_counts, &counters })
		MB_CUDA(cudaMemsetAsync(b->p, 0, b->bytes, s));
}

void plain_stats::extract(cudaStream_t s, unsigned* out_states, unsigned* out_counts)
{
	unsigned* out_n = counters.as<unsigned>() + 1;
	mbb_fixed_extract<<<(fp_cap + 255) / 256, 256, 0, s>>>(fp_cap, W, p.fp_keys, p.fp_counts, p.fp_states, out_n,
														  out_states, out_counts);
	MB_CUDA(cudaGetLastError());
}

std::unique_ptr<result> plain_stats::result_from(const void* win, const void* hs, const void* fins, const void* ctrs,
												 const unsigned* out_states, const unsigned* out_counts, long long n,
												 int state_size)
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
		std::memcpy(r->win_cnt.data(), win, cells * 4);
	}
	else
	{
		r->win_occ.resize(cells);
		std::memcpy(r->win_occ.data(), win, cells * 8);
	}
	r->win_h.resize(n_windows);
	std::memcpy(r->win_h.data(), hs, n_windows * 8);
	r->final_cnt.resize(n_bins);
	std::memcpy(r->final_cnt.data(), fins, n_bins * 4);
	unsigned ctr[2];
	std::memcpy(ctr, ctrs, sizeof ctr);
	r->fixed_overflow = ctr[0];
	const unsigned nfp = ctr[1];
	std::vector<unsigned> st((size_t)nfp * W), cn(nfp);
	if (nfp)
	{
		MB_CUDA(cudaMemcpy(st.data(), out_states, st.size() * 4, cudaMemcpyDeviceToHost));
		MB_CUDA(cudaMemcpy(cn.data(), out_counts, cn.size() * 4, cudaMemcpyDeviceToHost));
	}
	set_fixed_sorted(*r, st, cn);
	return r;
}

} // namespace mb
