// Host runtime of the B200 trajectory engine: device context, NVRTC-compiled model modules,
// run drivers (fused persistent kernel and buffered epochs) and host-side results.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "codegen.h"
#include "maboss_b200.h"
#include "sparse_bins.h"
#include "kernels/params.cuh"

namespace mb {

// Status codes (MB_OK, MB_ERR_*) and run modes (MB_MODE_*) come from the C ABI header.

struct engine_error : std::runtime_error
{
	int code;
	engine_error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_throw(cudaError_t e, const char* what);
#define MB_CUDA(x) ::mb::cuda_throw((x), #x)

// mb_initialize_random: trajectories initialised per thread (consecutive ones, by subsequence jumps)
// and the grid of 256-thread blocks for n trajectories. Up to 8 per thread, as long as the threads
// still number 148 SMs x 512; below that the initialisation is latency bound and each thread takes
// one.
inline int init_random_per(long long n)
{
	const long long per = n / (148LL * 512);
	return per < 1 ? 1 : per > 8 ? 8 : (int)per;
}
inline unsigned init_random_blocks(long long n, int per)
{
	return (unsigned)((n + 256LL * per - 1) / (256LL * per));
}

// Device memory owned by the runtime.
struct dbuf
{
	void* p = nullptr;
	size_t bytes = 0;
	dbuf() = default;
	explicit dbuf(size_t n) { alloc(n); }
	dbuf(const dbuf&) = delete;
	dbuf& operator=(const dbuf&) = delete;
	dbuf(dbuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr, o.bytes = 0; }
	dbuf& operator=(dbuf&& o) noexcept
	{
		std::swap(p, o.p);
		std::swap(bytes, o.bytes);
		return *this;
	}
	~dbuf();
	void alloc(size_t n);
	template <typename T>
	T* as() const
	{
		return static_cast<T*>(p);
	}
};

struct context
{
	int device = 0;
	int sm_count = 0;
	int cc_major = 0, cc_minor = 0;
	cudaStream_t stream = nullptr; // owned, non-blocking
	explicit context(int device);
	~context();
};

// Kernel families, compiled (NVRTC) and loaded on first use: the generated per-node code is
// inlined only into the kernels of the family that needs it.
enum kernel_family : int
{
	FAMILY_EXACT = 0, // mb_fused_exact
	FAMILY_FAST = 1,  // mb_fused_fast (incremental or dense)
	FAMILY_EPOCH = 2, // mb_simulate_epoch (incremental for @logic-form models, else dense)
	FAMILY_EPOCH_DENSE = 3, // mb_simulate_epoch with every node's rate function evaluated per step
	FAMILY_BATCH = 4, // mb_batched_fast_static / mb_batched_grad_static: the batched kernels for this network
	FAMILY_COUNT = 5
};

// Kernel handles resolved from NVRTC-compiled modules.
struct module
{
	context* ctx = nullptr;
	CUmodule mods[FAMILY_COUNT] = { nullptr, nullptr, nullptr, nullptr, nullptr };
	// FAMILY_BATCH is loaded as a runtime-API library: its kernels are cudaKernel_t handles, which the
	// batch engine's runtime-API launches, occupancy queries and graph nodes take like its own kernels
	cudaLibrary_t batch_lib = nullptr;
	const void* batched_fast_static = nullptr;
	const void* batched_grad_static = nullptr;
	int state_size = 0, state_words = 0;
	int noninternal_count = -1; // from the generated code (mbg_noninternal_count), -1 if absent
	bool incremental = false;	// @logic-form model: exact and epoch modes use the incremental kernels (generated MBG_INCREMENTAL)
	bool integer_rates = false; // fast mode's incremental kernel too (generated MBG_INTEGER_RATES), else its dense kernel
	bool fast_incremental() const { return incremental && integer_rates; }
	bool has_layout = false; // compiled from a model (full layout known)
	model_layout layout;
	std::string source; // generated model source that was compiled with the engine
	std::mutex run_mu;	// whole runs (run()) of this module are serialised
	std::unique_ptr<struct runner> last_runner; // buffers of the last run(), reused for the same config
	std::string log;	// NVRTC log

	CUfunction fused_exact = nullptr, fused_fast = nullptr;
	CUfunction init_random = nullptr, init_state = nullptr, sim_epoch = nullptr, sim_epoch_dense = nullptr;
	CUfunction window_epoch = nullptr, final_epoch = nullptr, fixed_epoch = nullptr;
	CUfunction compact_count = nullptr, compact_scan = nullptr, compact_scatter = nullptr, fixed_extract = nullptr;
	CUfunction bins_extract = nullptr;

	void ensure(int family);		// compile + load a family if needed (thread-safe)
	void ensure_any();				// at least one family (the shared statistics kernels)
	double compile_seconds = 0;		// NVRTC time spent so far
	~module();
};

// Compile generated model code together with the engine kernels (NVRTC, -arch=sm_100a).
std::unique_ptr<module> compile_module(context& ctx, const std::string& generated_code);
// A module whose kernel families are all compiled on first use (compile_module compiles the fast
// family at once); the batch engine uses it for FAMILY_BATCH only.
std::unique_ptr<module> compile_batch_module(context& ctx, const std::string& generated_code);
// NVRTC compilation only (no device needed): returns the cubin, throws on failure.
std::vector<char> compile_cubin(const std::string& generated_code, std::string& log, int family = FAMILY_FAST);

void launch(CUfunction f, unsigned grid, unsigned block, size_t smem, cudaStream_t s, void** args);

// One epoch of the buffered simulation (mb_simulate_epoch) over n trajectories of a batch of capacity
// `stride`; `dense` selects the reference's per-step evaluation of every rate function.
void simulate_epoch(module& m, bool dense, cudaStream_t s, int n, int stride, int L, unsigned* last_states,
					float* last_times, void* rands, unsigned* traj_states, float* traj_times, float* traj_h,
					unsigned char* statuses, unsigned long long* transitions);

// Sorts n sparse-bin records by their 128-bit keys (window, then non-internal index) on the device
// (sort.cu); synchronises the stream.
// The non-zero cells of a dense window histogram (`occ` int64 or `cnt` u32, whichever is not null), in
// increasing cell order (window, then state): their cell indices into idx_out (u64) and values into
// val_out (int64), both grown as needed. Returns the number of cells, or -1 without writing them
// when there are more than max_entries (the dense copy is then cheaper).
long long compact_cells(const long long* occ, const unsigned* cnt, unsigned long long cells,
						unsigned long long max_entries, dbuf& idx_out, dbuf& val_out, int sm_count, cudaStream_t s);

void sort_bins(const mb_key128* keys, const long long* vals, unsigned n, mb_key128* out_keys, long long* out_vals,
			   cudaStream_t s);

// Stable partition of the CONTINUE trajectories of an epoch batch into another buffer set
// (last_states SoA [word * stride + i], last_times, random states); the number kept is written to
// the device word *kept. `scratch` holds partition_scratch_bytes(n) bytes. With rejected_rands the
// random states of the other trajectories fill out_rands[kept, n), last first.
size_t partition_scratch_bytes(int n);
void partition(module& m, cudaStream_t s, int n, int stride, const unsigned char* statuses, const unsigned* states,
			   const float* times, const void* rands, unsigned* out_states, float* out_times, void* out_rands,
			   void* scratch, unsigned* kept, bool rejected_rands = false);
int occupancy_blocks(CUfunction f, int block, size_t smem);

struct run_config
{
	int mode = MB_MODE_FUSED_EXACT;
	long long sample_count = 0;
	unsigned long long seed = 0;
	unsigned long long first_traj = 0; // RNG subsequence of trajectory 0
	float max_time = 0, time_tick = 0; // exact host floats for window statistics
	bool discrete_time = false;
	std::vector<float> istate;
	std::vector<int> noninternal_nodes;
	int traj_len = 100;				 // trajectory_len_limit (simulation_runner.cu:51)
	int batch_limit = 1000000;		 // trajectory_batch_limit (simulation_runner.cu:50)
	int block = 256;
	int blocks_per_sm = 0;			 // 0 = occupancy calculator
	int fixed_capacity_log2 = 0;	 // 0 = automatic
	long long stats_trajectories = 0; // trajectory count the fixed-point scales are chosen for (0 = sample_count)
	int bin_capacity_log2 = 0;		  // sparse bins (more than 20 non-internal nodes): table size, 0 = automatic
	bool refill_reuse_rng = false;	  // epoch modes: refilled slots continue the finished trajectories' random states
};

run_config config_from_layout(const model_layout& L, int mode);

// Dense window histograms of at least this many cells (T x 2^k; 134 MB of int64 sums) are returned as
// their non-zero cells only, when those are at most a quarter of the cells.
constexpr unsigned long long compact_min_cells = 1ull << 24;

struct result
{
	int state_size = 0, state_words = 0, n_windows = 0;
	unsigned n_bins = 0;
	long long n_traj = 0;
	bool discrete_time = false;
	float time_tick = 0, max_time = 0;
	std::vector<int> noninternal_nodes;
	double fx = 1, fx_h = 1; // fixed-point scales of win_occ / win_h
	std::vector<long long> win_occ;
	std::vector<unsigned> win_cnt;
	std::vector<long long> win_h;
	std::vector<unsigned> final_cnt;
	std::vector<uint32_t> fixed_states; // n_fixed * state_words, sorted like the reference's std::map
	std::vector<unsigned> fixed_counts;
	unsigned fixed_overflow = 0;
	unsigned rate_errors = 0; // trajectories stopped on a non-finite total rate
	unsigned sections = 7;	  // statistics present: 1 windows, 2 final states, 4 fixed points
	// more than 20 non-internal nodes: sparse window bins (sorted by window, then index; sp_begin[w]
	// is the first entry of window w) and sparse final states (sorted by index); n_bins is 0
	bool wide = false;
	// at most 20 non-internal nodes but a large histogram (compact_min_cells or more cells): only its
	// non-zero cells, in the same sparse form (sp_*), selected on the device; final states dense
	bool compact = false;
	bulk_vector<int> sp_w;
	bulk_vector<unsigned __int128> sp_idx;
	bulk_vector<long long> sp_val; // occupancy in fixed point (continuous) or count (discrete)
	std::vector<size_t> sp_begin;  // [n_windows + 1]
	std::vector<unsigned __int128> fin_idx;
	std::vector<unsigned> fin_cnt;
	unsigned bin_overflow = 0; // bin additions that found no slot in the table (lost)
	double sparse_prob(size_t i) const; // probability of window entry i
	unsigned long long transitions = 0;
	float kernel_ms = 0; // device time of the simulation kernels
	float total_ms = 0;	 // device time of the whole run (setup + kernels + result copies)
	int epochs = 0;

	double window_prob(int w, unsigned bin) const; // window_average_small.cpp:126-140 (fp64)
	bool sparse_windows() const { return wide || compact; }
	double window_th(int w) const;				   // TH column (window_average_small.cpp:222-223)
};

// Fixed points stored in the order of std::map<static_state_t> (state.h:43-49: compared from the
// highest word down), from `counts.size()` records of r.state_words words.
void set_fixed_sorted(result& r, const std::vector<unsigned>& states, const std::vector<unsigned>& counts);
// The statistics of the union of disjoint trajectory sets (shards of one run): integer sums of the
// accumulators and the union of the fixed points. The parts must share the model's dimensions, the
// windows and the fixed-point scales (runs with the same stats_trajectories).
std::unique_ptr<result> merge_results(const std::vector<const result*>& parts);

// Fixed-point exponents (shared with the oracle so that both convert slices identically).
int occupancy_exponent(long long n_traj, float tick, bool discrete);
int entropy_exponent(long long n_traj, float tick, bool discrete);

// Frees host memory from cudaMallocHost (pinned) or, where pinning failed, from malloc.
struct host_deleter
{
	bool pinned = true;
	void operator()(void* p) const;
};

// Device accumulators of the three built-in statistics plugins (window averages, final
// states, fixed points) for one run.
struct stats_state
{
	module* mod = nullptr;
	dbuf occ, cnt, h, fin, fp_keys, fp_counts, fp_states, counters, istate;
	dbuf out_counts, out_states; // compacted fixed points (finalize)
	dbuf bin_keys, bin_vals, out_bin_keys, out_bin_vals; // sparse bins (more than 20 non-internal nodes)
	dbuf cell_idx, cell_vals; // non-zero cells of a large dense histogram (compact results), kept across runs
	unsigned bin_cap = 0;
	// host copies of the sorted bins, kept across runs (no re-allocation, no first-touch page
	// faults), in pinned memory (copied at full link speed) unless pinning fails (then malloc)
	std::unique_ptr<uint64_t[], host_deleter> hbin_keys;
	std::unique_ptr<long long[], host_deleter> hbin_vals;
	size_t hbin_cap = 0;
	bool wide = false;
	unsigned fp_cap = 0;
	int n_windows = 0;
	unsigned n_bins = 0;
	bool discrete_time = false;
	float time_tick = 0, max_time = 0;
	double fx = 1, fx_h = 1;
	int h_in_smem = 0;
	std::vector<int> noninternal_nodes;
	unsigned sections = 7; // MB_STATS_WINDOWS | MB_STATS_FINAL | MB_STATS_FIXED
	mb_stats_params p{};   // device pointers + scales passed to the statistics kernels

	void init(module& m, float time_tick, float max_time, bool discrete, const std::vector<int>& noninternal,
			  long long n_traj, int fixed_capacity_log2, cudaStream_t s, unsigned sections = 7,
			  long long scale_traj = 0, // trajectories the fixed-point scales are chosen for (0 = n_traj)
			  int bin_capacity_log2 = 0);
	void zero(cudaStream_t s); // clear every accumulator (asynchronous)
	void set_istate(const std::vector<float>& istate, cudaStream_t s);
	size_t h_smem() const { return h_in_smem ? (size_t)n_windows * sizeof(long long) : 0; }
	void window_batch(cudaStream_t s, int n, int stride, int traj_len, const unsigned* traj_states,
					  const float* traj_times, const float* traj_h);
	void final_batch(cudaStream_t s, int n, int stride, const unsigned* last_states, const unsigned char* statuses);
	void fixed_batch(cudaStream_t s, int n, int stride, const unsigned* last_states, const unsigned char* statuses);
	// counters (u64 view): [0] work counter, [1] transitions, [2] low: fixed-table overflow,
	// high: extracted fixed points, [3] low: trajectories stopped on a non-finite total rate
	unsigned long long* next_traj() const { return counters.as<unsigned long long>(); }
	unsigned long long* transitions() const { return counters.as<unsigned long long>() + 1; }
	unsigned* fp_overflow_ctr() const { return counters.as<unsigned>() + 4; }
	unsigned* extract_ctr() const { return counters.as<unsigned>() + 5; }
	unsigned* error_ctr() const { return counters.as<unsigned>() + 6; }
	unsigned* bin_overflow_ctr() const { return counters.as<unsigned>() + 7; }
	unsigned* bin_extract_ctr() const { return counters.as<unsigned>() + 8; }
	// copy everything back (synchronises the stream)
	std::unique_ptr<result> finalize(long long n_traj, cudaStream_t s);
};

// A run whose device buffers are allocated once: launch() zeroes the accumulators and enqueues the
// simulation on a stream without synchronising (fused modes), collect() copies the results back.
struct runner
{
	module* mod = nullptr;
	run_config cfg;
	stats_state st;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	int epochs = 0;
	unsigned launches = 0; // engine kernels enqueued by the last launch()
	dbuf rng;			   // exact mode: XORWOW states of every trajectory (empty above max_rng_states)
	static constexpr long long max_rng_states = 1LL << 24;
	runner(module& m, const run_config& c);
	~runner();
	void launch(cudaStream_t s);
	std::unique_ptr<result> collect(cudaStream_t s);
	unsigned kernel_launches() const; // engine kernels enqueued by the last launch()
};

// Run a whole simulation with the built-in statistics.
std::unique_ptr<result> run(module& m, const run_config& cfg);

// Launch-shape autotuner of the fused kernels: times candidate (threads per block, resident blocks per
// SM) pairs on a slice of the run's own trajectories and returns them fastest first.
struct tuned_shape
{
	int block = 0, blocks_per_sm = 0;
	double transitions_per_s = 0;
};
std::vector<tuned_shape> autotune(module& m, const run_config& cfg);

} // namespace mb
