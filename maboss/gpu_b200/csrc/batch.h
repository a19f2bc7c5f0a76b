// Batched runs over parameter variants and networks, and score-function gradients (see batch.cu).
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "codegen.h"
#include "model.h"
#include "runtime.h"

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
	std::unique_ptr<result> finalize_plain(long long n, int state_size, cudaStream_t s);
};

class batch_engine
{
public:
	struct network
	{
		model_t model;
		model_layout L;
		dbuf node, hdr, in1, in2, tt, self, ni_node;
	};
	struct variant
	{
		int net = 0;
		long long n_traj = 0;
		unsigned long long first_traj = 0;
		std::vector<std::string> grad_params;
		rate_set rates;
		int rate_shift = 0;
		std::vector<unsigned> q;
		plain_stats st;
		dbuf d_q, d_rate, d_istate, d_gptr, d_gp, d_gd, d_counters, d_grad, d_cot;
		std::unique_ptr<result> res;
		std::vector<double> grad; // d (sum_ws cot[w][s] P_w(s)) / d parameter
	};

	explicit batch_engine(context& c);
	~batch_engine();
	int add_model(const model_t& m);
	// `overrides`: variable values of this variant; `grad_params`: variables to differentiate
	int add_variant(int net, const std::map<std::string, float>& overrides, long long n_traj,
					unsigned long long first_traj, const std::vector<std::string>& grad_params = {});
	// one persistent launch over every variant; with cotangents (one [windows * 2^k] vector per
	// variant) it also computes the vector-Jacobian products
	void run(unsigned long long seed, const std::vector<std::vector<double>>* cotangents = nullptr);

	context* ctx;
	std::vector<std::unique_ptr<network>> nets;
	std::vector<std::unique_ptr<variant>> vars_;
	dbuf d_nets, d_vars;
	float kernel_ms = 0;
	int last_block = 0;
	unsigned last_grid = 0;
};

} // namespace mb
