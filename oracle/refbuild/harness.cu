// ref_run: runs the reference MaBoSS.GPU trajectory path, built from its own sources, on a
// .bnd/.cfg pair (TEST INFRASTRUCTURE under oracle/: the parity checker and the reference arm
// of the benchmark; the engine never links or calls it).
//
// The flow is the reference's src/main.cpp:112-176 (parse, checks, generate, NVRTC + nvJitLink,
// simulation_runner::run_simulation with the three statistics plugins, finalize), calling the
// reference's own classes. Added around it:
//   * a `stats` plugin that counts recorded trajectory slots (slot s >= 1 with time > 0, the
//     transitions of the benchmark metric), added to a first untimed run only, through
//     stats_composite::add (src/statistics/stats_composite.cpp:3);
//   * CUDA events (legacy stream, which the reference launches on) around run_simulation, and a
//     host clock around run_simulation + finalize, for the timed runs;
//   * checks, before any GPU work, of the sizes for which the reference's own arithmetic stays in
//     bounds (see check_inputs); an input outside them is refused with exit code 3;
//   * a binary dump of the last run's raw statistics, and the reference's CSV writers.
//
// usage: ref_run [--samples N] [--seed S] [--warmup W] [--runs K] [--dump FILE]
//                [--csv PREFIX] [--visualize] [--emit-code] bnd cfg
// The last line on stdout is one JSON object with the timings and the transition count.
// --emit-code prints the reference generator's CUDA source for the model and exits (no GPU).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <optional>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "generator.h"
#include "kernel_compiler.h"
#include "simulation_runner.h"
#include "state.h"
#include "statistics/final_states.h"
#include "statistics/fixed_states.h"
#include "statistics/stats_composite.h"
#include "statistics/window_average_small.h"

namespace
{
// ---- read access to the plugins' result members --------------------------------------------
// The reference keeps its statistics in private members and offers only text output
// (visualize, write_csv) with 6 significant digits. The parity checks need the raw values, so
// the members are named through explicit template instantiation, the one context in which C++
// does not check access ([temp.explicit]); nothing in the reference is modified.
template <typename Tag, typename Tag::type M>
struct expose
{
	friend typename Tag::type member_of(Tag) { return M; }
};

#define EXPOSE(TAG, TYPE, MEMBER)                                                                                      \
	struct TAG                                                                                                         \
	{                                                                                                                  \
		using type = TYPE;                                                                                             \
		friend type member_of(TAG);                                                                                    \
	};                                                                                                                 \
	template struct expose<TAG, MEMBER>;

EXPOSE(composite_stats, std::vector<stats_ptr> stats_composite::*, &stats_composite::composed_stats_)
EXPOSE(wa_probs, std::vector<float> window_average_small_stats::*, &window_average_small_stats::result_probs_)
EXPOSE(wa_counts, std::vector<int> window_average_small_stats::*, &window_average_small_stats::result_probs_discrete_)
EXPOSE(wa_entropies, std::vector<float> window_average_small_stats::*,
	   &window_average_small_stats::result_tr_entropies_)
EXPOSE(fs_occurences, std::vector<int> final_states_stats::*, &final_states_stats::result_occurences_)

template <int W>
struct fixed_result
{
	using type = std::map<static_state_t<W>, int> fixed_states_stats<W>::*;
	friend type member_of(fixed_result<W>);
};
#define EXPOSE_FIXED(W) template struct expose<fixed_result<W>, &fixed_states_stats<W>::result_>;
EXPOSE_FIXED(1) EXPOSE_FIXED(2) EXPOSE_FIXED(3) EXPOSE_FIXED(4) EXPOSE_FIXED(5) EXPOSE_FIXED(6) EXPOSE_FIXED(7)
EXPOSE_FIXED(8) EXPOSE_FIXED(9) EXPOSE_FIXED(10) EXPOSE_FIXED(11) EXPOSE_FIXED(12) EXPOSE_FIXED(13)
EXPOSE_FIXED(14) EXPOSE_FIXED(15) EXPOSE_FIXED(16) EXPOSE_FIXED(17) EXPOSE_FIXED(18) EXPOSE_FIXED(19)
EXPOSE_FIXED(20) EXPOSE_FIXED(21) EXPOSE_FIXED(22) EXPOSE_FIXED(23) EXPOSE_FIXED(24) EXPOSE_FIXED(25)
EXPOSE_FIXED(26) EXPOSE_FIXED(27) EXPOSE_FIXED(28) EXPOSE_FIXED(29) EXPOSE_FIXED(30) EXPOSE_FIXED(31)
EXPOSE_FIXED(32)
static_assert((MAX_NODES + 31) / 32 <= 32, "fixed-point access is instantiated for at most 32 state words");

// fixed points of the plugin built by fixed_states_stats_builder for `words` state words, as
// (state words..., count) rows in the map's order
template <int W>
void fixed_rows(stats* s, int words, std::vector<uint32_t>& states, std::vector<int>& counts)
{
	if constexpr (W > 32)
		return;
	else if (W == words)
	{
		auto* fs = dynamic_cast<fixed_states_stats<W>*>(s);
		if (!fs)
			throw std::runtime_error("the fixed-point plugin has an unexpected type");
		for (const auto& [st, c] : fs->*member_of(fixed_result<W> {}))
		{
			states.insert(states.end(), st.data, st.data + W);
			counts.push_back(c);
		}
	}
	else
		fixed_rows<W + 1>(s, words, states, counts);
}

// ---- the transition counter -----------------------------------------------------------------
// Trajectory buffer layout of the reference (simulation.cu:91-93): times of trajectory t at
// [t * L + s]. Slot 0 holds the previous epoch's last time; a recorded step is a slot s >= 1
// whose time is non-zero (the buffer is cleared to 0 before each epoch, simulation_runner.cu:98,161).
__global__ void count_recorded_slots(const float* __restrict__ times, long long n_slots, int L,
									 unsigned long long* __restrict__ out)
{
	unsigned long long local = 0;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_slots;
		 i += (long long)gridDim.x * blockDim.x)
		local += (i % L != 0 && times[i] > 0.f) ? 1ull : 0ull;
	for (int o = 16; o > 0; o >>= 1)
		local += __shfl_down_sync(0xffffffffu, local, o);
	if ((threadIdx.x & 31) == 0 && local)
		atomicAdd(out, local);
}

class transition_counter : public stats
{
	int traj_len_;
	unsigned long long* d_count_ = nullptr;

public:
	unsigned long long transitions = 0;

	explicit transition_counter(int traj_len) : traj_len_(traj_len)
	{
		if (cudaMalloc(&d_count_, sizeof(unsigned long long)) != cudaSuccess
			|| cudaMemset(d_count_, 0, sizeof(unsigned long long)) != cudaSuccess)
			throw std::runtime_error("transition counter: device allocation failed");
	}
	~transition_counter() override { cudaFree(d_count_); }

	void process_batch(thrust::device_ptr<state_word_t>, thrust::device_ptr<float> traj_times,
					   thrust::device_ptr<float>, thrust::device_ptr<state_word_t>,
					   thrust::device_ptr<trajectory_status>, int n_trajectories) override
	{
		long long slots = (long long)n_trajectories * traj_len_;
		if (slots == 0)
			return;
		int blocks = (int)std::min<long long>((slots + 255) / 256, 148 * 16);
		count_recorded_slots<<<blocks, 256>>>(traj_times.get(), slots, traj_len_, d_count_);
		if (cudaGetLastError() != cudaSuccess)
			throw std::runtime_error("transition counter: launch failed");
	}

	void finalize() override
	{
		if (cudaMemcpy(&transitions, d_count_, sizeof(transitions), cudaMemcpyDeviceToHost) != cudaSuccess)
			throw std::runtime_error("transition counter: copy failed");
	}

	void visualize(int, const std::vector<std::string>&) override {}
	void write_csv(int, const std::vector<std::string>&, const std::string&) override {}
};

// ---- input checks -------------------------------------------------------------------------
// Sizes for which the reference's arithmetic stays in bounds, established by reading it:
//  * simulation_runner.cu:68-69 sizes the trajectory buffer as batch * 100 * words in int, and
//    window_average_small.cu:71 indexes it as id * state_words in int (id < batch * 100): both
//    overflow once batch * 100 * words exceeds INT_MAX (about 671,000 trajectories of 32 words),
//    and the window kernel would then read at a negative offset.
//  * window_average_small.cu:75-92 walks windows from floorf(t0 / tick) while (w + 1) * tick <
//    t1; with windows = ceil(max_time / tick) (window_average_small.cpp:30) the index stays below
//    `windows` when floorf(prev(max_time) / tick) < windows and windows * tick >= max_time (both
//    evaluated in float, as on the device); otherwise the kernel adds past the histogram.
//  * window_average_small.cu:123 (discrete) takes lroundf(t / tick) of a time t <= max_time -
//    tick (simulation.cu:113-114 sets any later time to max_time), so the index stays below
//    `windows` when lroundf((max_time - tick) / tick) < windows.
//  * main.cpp:142-152: at most 20 non-internal nodes and MAX_NODES nodes.
std::string check_inputs(long long n, int nodes, int noninternals, bool discrete, float max_time, float tick)
{
	const long long L = 100, B = std::min<long long>(1000000, n), W = (nodes + 31) / 32;
	if (noninternals > 20)
		return "more than 20 non-internal nodes (the reference refuses them, main.cpp:142)";
	if (nodes > MAX_NODES)
		return "more nodes than MAX_NODES";
	if (n < 1)
		return "no trajectories";
	if (B * L * W > 2147483647LL)
		return "batch * 100 * state words exceeds INT_MAX: the reference's int sizes and indices overflow "
			   "(simulation_runner.cu:68, window_average_small.cu:71)";
	if (!(tick > 0.f) || !(max_time > 0.f))
		return "max_time and time_tick must be positive";
	const float windows = std::ceil(max_time / tick);
	if (windows > 1e7f)
		return "too many windows";
	const int T = (int)windows;
	if (discrete)
	{
		if (lroundf((max_time - tick) / tick) >= T)
			return "discrete window index could reach the histogram's end (window_average_small.cu:123)";
	}
	else
	{
		float below = std::nextafter(max_time, 0.f);
		if ((int)std::floor(below / tick) >= T || (float)T * tick < max_time)
			return "window walk could pass the histogram's end (window_average_small.cu:75-92)";
	}
	return "";
}

void write_dump(const std::string& path, long long n, int nodes, int words, int noninternals, int T, uint32_t S,
				bool discrete, unsigned long long transitions, float max_time, float tick, stats_composite& sc)
{
	auto& all = sc.*member_of(composite_stats {});
	auto* fin = dynamic_cast<final_states_stats*>(all.at(0).get());
	auto* win = dynamic_cast<window_average_small_stats*>(all.at(2).get());
	if (!fin || !win)
		throw std::runtime_error("unexpected plugin order");
	std::vector<uint32_t> fstates;
	std::vector<int> fcounts;
	fixed_rows<1>(all.at(1).get(), words, fstates, fcounts);

	std::ofstream out(path, std::ios::binary);
	auto put64 = [&](long long v) { out.write(reinterpret_cast<const char*>(&v), 8); };
	auto putf = [&](float v) { out.write(reinterpret_cast<const char*>(&v), 4); };
	out.write("MBREF001", 8);
	put64(n);
	put64(nodes);
	put64(words);
	put64(noninternals);
	put64(T);
	put64(S);
	put64(discrete ? 1 : 0);
	put64((long long)transitions);
	put64((long long)fcounts.size());
	putf(max_time);
	putf(tick);
	if (discrete)
	{
		const auto& v = win->*member_of(wa_counts {});
		out.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * 4));
	}
	else
	{
		const auto& v = win->*member_of(wa_probs {});
		out.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * 4));
	}
	const auto& h = win->*member_of(wa_entropies {});
	out.write(reinterpret_cast<const char*>(h.data()), (std::streamsize)(h.size() * 4));
	const auto& f = fin->*member_of(fs_occurences {});
	out.write(reinterpret_cast<const char*>(f.data()), (std::streamsize)(f.size() * 4));
	out.write(reinterpret_cast<const char*>(fstates.data()), (std::streamsize)(fstates.size() * 4));
	out.write(reinterpret_cast<const char*>(fcounts.data()), (std::streamsize)(fcounts.size() * 4));
	if (!out)
		throw std::runtime_error("cannot write " + path);
}
} // namespace

int main(int argc, char** argv)
{
	std::vector<std::string> args(argv + 1, argv + argc);
	long long samples = -1, seed = -1;
	int warmup = 0, runs = 1;
	std::string dump, csv;
	bool visualize = false, emit_code = false;
	std::vector<std::string> pos;
	for (size_t i = 0; i < args.size(); i++)
	{
		auto next = [&]() -> std::string {
			if (i + 1 >= args.size())
				throw std::runtime_error("missing value after " + args[i]);
			return args[++i];
		};
		if (args[i] == "--samples")
			samples = std::stoll(next());
		else if (args[i] == "--seed")
			seed = std::stoll(next());
		else if (args[i] == "--warmup")
			warmup = std::stoi(next());
		else if (args[i] == "--runs")
			runs = std::stoi(next());
		else if (args[i] == "--dump")
			dump = next();
		else if (args[i] == "--csv")
			csv = next();
		else if (args[i] == "--visualize")
			visualize = true;
		else if (args[i] == "--emit-code")
			emit_code = true;
		else
			pos.push_back(args[i]);
	}
	if (pos.size() != 2 || runs < 1 || warmup < 0)
	{
		std::cerr << "usage: ref_run [--samples N] [--seed S] [--warmup W] [--runs K] [--dump FILE] [--csv PREFIX] "
					 "[--visualize] [--emit-code] bnd cfg\n";
		return 1;
	}

	// src/main.cpp:131-140
	driver drv;
	if (drv.parse(pos[0], pos[1]))
		return 1;
	if (emit_code)
	{
		std::cout << generator(drv).generate_code();
		return 0;
	}
	if (samples >= 0)
		drv.constants["sample_count"] = (float)samples;
	if (seed >= 0)
		drv.constants["seed_pseudorandom"] = (float)seed;

	bool discrete_time = drv.constants["discrete_time"] != 0;
	float max_time = drv.constants["max_time"];
	float time_tick = drv.constants["time_tick"];
	int sample_count = drv.constants["sample_count"];
	unsigned long long sim_seed = drv.constants["seed_pseudorandom"];
	std::vector<float> initial_probs;
	for (auto&& node : drv.nodes)
		initial_probs.push_back(node.istate);
	state_t noninternals_mask(drv.nodes.size());
	for (size_t i = 0; i < drv.nodes.size(); ++i)
		if (!drv.nodes[i].is_internal(drv))
			noninternals_mask.set(i);
	int noninternals_count = (int)std::count_if(drv.nodes.begin(), drv.nodes.end(),
												[&](const auto& node) { return !node.is_internal(drv); });
	std::vector<std::string> node_names;
	for (auto&& node : drv.nodes)
		node_names.push_back(node.name);
	const int nodes = (int)drv.nodes.size();
	const int words = (nodes + 31) / 32;

	std::string refusal = check_inputs(sample_count, nodes, noninternals_count, discrete_time, max_time, time_tick);
	if (!refusal.empty())
	{
		std::cerr << "ref_run: input refused: " << refusal << std::endl;
		std::cout << "{\"refused\": \"" << refusal << "\"}" << std::endl;
		return 3;
	}

	// src/main.cpp:40-54 (do_compilation)
	auto c0 = std::chrono::steady_clock::now();
	std::optional<kernel_compiler> compiler;
	{
		generator gen(drv);
		auto code = gen.generate_code();
		compiler.emplace();
		if (compiler->compile_simulation(code, discrete_time))
			return 1;
	}
	double compile_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();

	cudaEvent_t ev0, ev1;
	if (cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess)
		return 2;

	unsigned long long transitions = 0;
	std::vector<double> device_ms, host_ms;
	const int total = 1 + warmup + runs; // run 0 counts transitions, untimed
	const uint32_t S = 1u << noninternals_count;
	const int T = (int)std::ceil(max_time / time_tick);
	for (int r = 0; r < total; r++)
	{
		// src/main.cpp:56-83 (do_simulation)
		simulation_runner runner(sample_count, nodes, sim_seed, initial_probs);
		stats_composite sc;
		sc.add(std::make_unique<final_states_stats>(noninternals_mask, noninternals_count, compiler->final_states));
		fixed_states_stats_builder::add_fixed_states_stats(sc, noninternals_mask.words_n());
		sc.add(std::make_unique<window_average_small_stats>(time_tick, max_time, discrete_time, noninternals_mask,
															noninternals_count, runner.trajectory_len_limit,
															runner.trajectory_batch_limit,
															compiler->window_average_small));
		transition_counter* counter = nullptr;
		if (r == 0)
		{
			auto c = std::make_unique<transition_counter>(runner.trajectory_len_limit);
			counter = c.get();
			sc.add(std::move(c));
		}
		if (cudaDeviceSynchronize() != cudaSuccess)
			return 2;

		auto h0 = std::chrono::steady_clock::now();
		cudaEventRecord(ev0, 0);
		runner.run_simulation(sc, compiler->initialize_random, compiler->initialize_initial_state,
							  compiler->simulate);
		cudaEventRecord(ev1, 0);
		sc.finalize();
		if (cudaEventSynchronize(ev1) != cudaSuccess)
			return 2;
		double hms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
		float dms = 0.f;
		cudaEventElapsedTime(&dms, ev0, ev1);
		if (counter)
			transitions = counter->transitions;
		else if (r > warmup)
		{
			device_ms.push_back(dms);
			host_ms.push_back(hms);
		}

		if (r == total - 1)
		{
			if (!dump.empty())
				write_dump(dump, sample_count, nodes, words, noninternals_count, T, S, discrete_time, transitions,
						   max_time, time_tick, sc);
			if (!csv.empty())
				sc.write_csv(sample_count, node_names, csv);
			if (visualize)
				sc.visualize(sample_count, node_names);
		}
	}

	auto list = [](const std::vector<double>& v) {
		std::ostringstream os;
		os << "[";
		for (size_t i = 0; i < v.size(); i++)
			os << (i ? ", " : "") << v[i];
		os << "]";
		return os.str();
	};
	std::cout << "{\"trajectories\": " << sample_count << ", \"nodes\": " << nodes << ", \"state_words\": " << words
			  << ", \"noninternals\": " << noninternals_count << ", \"windows\": " << T
			  << ", \"discrete\": " << (discrete_time ? "true" : "false") << ", \"transitions\": " << transitions
			  << ", \"compile_s\": " << compile_s << ", \"device_ms\": " << list(device_ms)
			  << ", \"host_ms\": " << list(host_ms) << "}" << std::endl;
	return 0;
}
