// Code generator: model -> CUDA source compiled by NVRTC together with the engine kernels.
//
// The emitted per-node rate functions, `compute_transition_rates`,
// `compute_transition_entropy` and `get_non_internal_index` reproduce the text of the
// reference generator (src/generator.cpp:84-235) so that the compiled rate arithmetic is
// identical. On top of them it emits straight-line helpers (`mbg_*`) that the engine
// kernels call instead of materialising a `float rates[N]` array per thread.
#pragma once

#include <string>
#include <vector>

#include "model.h"

namespace mb {

// Static facts about a model that the host runtime needs next to the compiled module.
struct model_layout
{
	int state_size = 0;					// N
	int state_words = 0;				// W = ceil(N/32)
	std::vector<int> noninternal_nodes; // node indices in node order
	int noninternal_words = 0;			// number of distinct state words holding non-internal bits
	bool discrete_time = false;
	float max_time = 0.f;  // exact float constant (host side, window statistics)
	float time_tick = 0.f; // exact float constant (host side, window statistics)
	int sample_count = 0;
	unsigned long long seed = 0;
	std::vector<float> istate;
	std::vector<std::string> names;

	// Fast-path form `rate_up = @logic ? U : 0; rate_down = @logic ? 0 : D;` for every
	// node (generator.cpp:57-82). When true, `up`/`down` hold the rate values exactly as
	// the compiled code sees them (6-significant-digit literals converted to float).
	bool all_fast_path = false;
	std::vector<char> fast_path;
	std::vector<float> up, down;
	bool rates_nonnegative = false;

	// Incremental engine tables (valid when `incremental_ok`): node -> inputs of its logic
	// (CSR), the logic truth table over those inputs, and node -> dependents (CSR).
	bool incremental_ok = false;
	std::vector<int> in_ptr, in_idx;
	std::vector<int> tt_ptr;				// offset (in 32-bit words) of each node's truth table
	std::vector<unsigned> tt_words;			// truth tables, bit b = logic value for input pattern b
	std::vector<int> dep_ptr, dep_idx;		// nodes whose rate must be re-evaluated after a flip
	int rate_shift = 0;						// fast-mode rates in fixed point: q = round(rate * 2^shift)
	std::vector<unsigned> q_up, q_down;
	// The fast kernel's integer rates are usable (valid when `incremental_ok`): every state word's
	// largest rate sum is below 2^32 units and every positive rate is at least 2^20 units (relative
	// rounding error at most 2^-21). Otherwise fast mode takes the dense fp32 kernel.
	bool integer_rates_ok = false;

	int windows() const; // ceil(max_time / time_tick) in float, window_average_small.cpp:305
};

// Analyse a parsed model (throws model_error on semantic errors such as unknown nodes).
model_layout analyze_model(const model_t& m);

// Rates of the fast-path nodes for given variable values (exact floats, not the 6-digit literals of
// the generated code), with their derivatives with respect to the listed variables: entry 2i is
// node i's up rate, 2i+1 its down rate; grad_ptr/grad_p/grad_d are a CSR of (parameter, d rate / d
// parameter) pairs. Throws if a node is not of the fast-path form.
struct rate_set
{
	std::vector<float> up, down;
	std::vector<int> grad_ptr, grad_p;
	std::vector<float> grad_d;
};
rate_set fast_rates(const model_t& m, const std::map<std::string, float>& variables,
					const std::vector<std::string>& params);

// Tables of the incremental kernels for given rates (see codegen.cpp: emit_incremental_tables).
struct incremental_tables
{
	int rate_shift = 0;
	bool ok = false; // rates representable (rates finite and >= 0, word sums < 2^32 units, every positive rate >= 2^20 units)
	std::vector<unsigned> node, hdr, in1, in2; // uint4 records, 4 words each
	// compact dependent records (the NVRTC kernels): {k | m << 16 | (ni_pos(k) + 1) << 21, truth
	// table or offset, inputs 0-1, inputs 2-3}, and inputs 4-11 of records with more than 4 inputs
	std::vector<unsigned> crec, cext;
	std::vector<unsigned> tt;
	std::vector<int> self;
	std::vector<unsigned> q; // (q_up, q_down) per node
};
// The fixed-point scale of the integer rates: the largest shift <= 31 with every state word's
// largest possible rate sum (the larger of up and down per node) below 2^32 units, and the least
// number of units a positive rate must get (2^20: relative rounding error at most 2^-21).
int integer_rate_shift(const std::vector<float>& up, const std::vector<float>& down, int state_words);
constexpr double integer_rate_min_units = 1048576.0;

incremental_tables build_incremental_tables(const model_layout& L, const std::vector<float>& up,
											const std::vector<float>& down);

// The generated CUDA source for a model (model-specific part only).
std::string generate_code(const model_t& m);

} // namespace mb
