// Batched runs over parameter variants and networks, and score-function gradients (see batch.cu).
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "codegen.h"
#include "model.h"
#include "runtime.h"

struct mb_batch_params; // kernels/batched.cuh
struct mb_variant;

namespace mb {

// Accumulators of one variant (the layout and fixed-point scales of stats_state, without a
// compiled module).
struct plain_stats
{
	dbuf occ, cnt, h, fin, fp_keys, fp_counts, fp_states, counters;
	unsigned fp_cap = 0;
	int W = 1, n_windows = 0;
	unsigned n_bins = 0;
	bool discrete_time = false;
	float time_tick = 0, max_time = 0;
	double fx = 1, fx_h = 1;
	std::vector<int> noninternal_nodes;
	mb_stats_params p{};
	void init_plain(int words, float tick, float tmax, bool discrete, const std::vector<int>& noninternal, long long n,
					cudaStream_t s);
	void zero(cudaStream_t s); // clear every accumulator (asynchronous, capturable)
	// compact the fixed-point table into (state, count) records; their number goes to counters[1]
	void extract(cudaStream_t s, unsigned* out_states, unsigned* out_counts);
	// the result from host copies of the accumulators and the device records of the fixed points
	std::unique_ptr<result> result_from(const void* win, const void* h, const void* fin, const void* counters,
										const unsigned* out_states, const unsigned* out_counts, long long n,
										int state_size);
};

class batch_engine
{
public:
	struct network
	{
		model_t model;
		model_layout L;
		dbuf dep, rec, ext, tt, self, ni_node;
		// the batched kernels compiled for this network alone (NVRTC, FAMILY_BATCH; on first use)
		std::unique_ptr<module> mod;
	};
	struct variant
	{
		int net = 0;
		long long n_traj = 0;
		unsigned long long first_traj = 0;
		std::vector<std::string> grad_params;
		std::map<std::string, float> overrides; // this variant's variable values (the rest: the model's)
		std::map<int, bool> mutants; // node -> forced on (true) / off: initial state 1 / 0, both rates 0
		std::vector<float> istate;   // initial-state probabilities (the model's, mutants forced)
		rate_set rates;
		int rate_shift = 0;
		std::vector<unsigned> q;
		plain_stats st;
		dbuf d_q, d_rate, d_rlog, d_istate, d_gptr, d_gp, d_gd, d_counters, d_grad, d_cot, out_states, out_counts;
		bool ready = false; // accumulators and per-variant buffers exist (created once, shared by both plans)
		std::unique_ptr<result> res;
		std::vector<double> grad; // d (sum_ws cot[w][s] P_w(s)) / d parameter
	};

	explicit batch_engine(context& c);
	~batch_engine();
	int add_model(const model_t& m);
	// `overrides`: variable values of this variant; `grad_params`: variables to differentiate
	int add_variant(int net, const std::map<std::string, float>& overrides, long long n_traj,
					unsigned long long first_traj, const std::vector<std::string>& grad_params = {},
					const std::map<std::string, bool>& mutants = {});
	// new values of some of variant v's variables: its rate tables are recomputed and uploaded in
	// place, so prepared runs, launch shapes and captured graphs stay valid
	void set_variables(int v, const std::map<std::string, float>& values);
	// one persistent launch over every variant; with cotangents (one [windows * 2^k] vector per
	// variant) it also computes the vector-Jacobian products
	void run(unsigned long long seed, const std::vector<std::vector<double>>* cotangents = nullptr);

	// Runs are captured once as a CUDA graph (clears, kernel, extraction, result copies) and replayed
	// with the seed updated; the launch shape is chosen by timing candidates on the batch first.
	bool use_graph = true;
	bool autotune = true;
	// A batch of one network runs the batched kernels compiled for that network (its sizes and
	// tables compile-time, the variants' rates runtime; NVRTC on the first run, a few seconds);
	// false: the ahead-of-time kernels that take any networks.
	bool specialize = true;
	struct tuning_point
	{
		bool grad;
		int block, blocks_per_sm;
		float kernel_ms;
	};
	std::vector<tuning_point> tuning; // every candidate timed so far

	context* ctx;
	std::vector<std::unique_ptr<network>> nets;
	std::vector<std::unique_ptr<variant>> vars_;
	float kernel_ms = 0;
	int last_block = 0, last_per_sm = 0;
	unsigned last_grid = 0;
	unsigned graph_nodes = 0; // nodes of the last captured graph

private:
	struct host_off_t
	{
		size_t win = 0, h = 0, fin = 0, ctr = 0, trans = 0, grad = 0;
	};
	struct prepared
	{
		bool grad = false;
		std::unique_ptr<mb_batch_params> B; // the kernel's parameter block
		const void* fn = nullptr;
		size_t smem_per_thread = 0, smem = 0;
		int block = 0, per_sm = 0;
		unsigned grid = 0;
		dbuf counters, gscratch;
		void* host = nullptr; // pinned
		std::vector<host_off_t> host_off;
		cudaEvent_t e0 = nullptr, e1 = nullptr;
		cudaGraph_t graph = nullptr;
		cudaGraphExec_t exec = nullptr;
		cudaGraphNode_t kernel = nullptr;
		// this plan's device descriptors (the forward and gradient plans differ in the cotangent
		// pointers) and their host copy
		dbuf d_nets, d_vars;
		std::vector<mb_variant> hvars;
		~prepared();
	};
	std::unique_ptr<prepared> prep[2]; // forward, gradient
	void invalidate();
	prepared& prepare(bool grad);
	int fit(prepared& ps, int block, size_t& smem) const;
	void compute_rates(variant& V) const;
	void upload_tables(variant& V, cudaStream_t s);
	void set_shape(prepared& ps, int block, int per_sm);
	void enqueue(prepared& ps, cudaStream_t s, bool capturing);
	void tune(prepared& ps, cudaStream_t s);
};

} // namespace mb
