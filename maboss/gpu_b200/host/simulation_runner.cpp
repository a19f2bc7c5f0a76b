#include "simulation_runner.h"

#include <algorithm>
#include <stdexcept>

#include "maboss_b200_mirror.h"
#include "timer.h"

namespace {

// device buffer of the context's device (reference: thrust::device_malloc / device_free)
struct device_buffer
{
	mb_context ctx;
	void* p = nullptr;
	device_buffer(mb_context c, size_t bytes) : ctx(c) { mirror::check(mb_device_malloc(c, bytes, &p), "allocate"); }
	~device_buffer() { mb_device_free(ctx, p); }
	device_buffer(const device_buffer&) = delete;
	device_buffer& operator=(const device_buffer&) = delete;
	template <typename T>
	T* as() const
	{
		return static_cast<T*>(p);
	}
};

} // namespace

simulation_runner::simulation_runner(int n_trajectories, int state_size, unsigned long long seed,
									 std::vector<float> initial_probs)
	: n_trajectories_(n_trajectories),
	  state_size_(state_size),
	  state_words_((state_size + 31) / 32),
	  seed_(seed),
	  initial_probs_(std::move(initial_probs))
{
	// src/simulation_runner.cu:44-52
	trajectory_batch_limit = std::min(1'000'000, n_trajectories);
	trajectory_len_limit = 100;
}

void simulation_runner::run_simulation(stats_composite& stats_runner, kernel_wrapper& initialize_random,
									   kernel_wrapper& initialize_initial_state, kernel_wrapper& simulate)
{
	mb_module module = simulate.module;
	if (!module || initialize_random.module != module || initialize_initial_state.module != module)
		throw std::runtime_error("run_simulation: the kernels must come from one compiled module");
	if ((int)initial_probs_.size() != state_size_)
		throw std::runtime_error("run_simulation: one initial probability per node is needed");
	if (n_trajectories_ < 0)
		throw std::runtime_error("run_simulation: negative number of trajectories");
	transitions_ = 0;
	epochs_ = 0;
	if ((mode == MB_MODE_FUSED_EXACT || mode == MB_MODE_FUSED_FAST) && stats_runner.fusable())
		run_fused(stats_runner, module);
	else
		run_buffered(stats_runner, module);
}

void simulation_runner::run_fused(stats_composite& stats_runner, mb_module module)
{
	timer_stats t("simulation_runner> fused run");
	const mirror::run_description d = stats_runner.describe();
	mb_run_params p{};
	p.time_tick = d.time_tick;
	p.max_time = d.max_time;
	p.discrete_time = d.discrete_time ? 1 : 0;
	p.initial_probs = initial_probs_.data();
	p.n_nodes = state_size_;
	p.noninternal_nodes = d.noninternal_nodes.data();
	p.n_noninternal = (int)d.noninternal_nodes.size();
	mb_run_config c{};
	c.mode = mode;
	c.sample_count = n_trajectories_;
	c.seed = seed_;
	c.first_traj = first_trajectory;
	c.traj_len = trajectory_len_limit;
	c.batch_limit = std::max(1, trajectory_batch_limit);
	c.block = 256;
	mb_result r = nullptr;
	mirror::check(mb_run_module(module, &c, &p, &r), "run_simulation");
	auto h = std::make_shared<mirror::result_handle>(r);
	mirror::check(mb_result_transitions(r, &transitions_), "run_simulation");
	epochs_ = 1;
	stats_runner.take_result(h);
}

// src/simulation_runner.cu:54-180 over SoA buffers
void simulation_runner::run_buffered(stats_composite& stats_runner, mb_module module)
{
	mb_context ctx = nullptr;
	mirror::check(mb_module_context(module, &ctx), "run_simulation");
	const long long n = n_trajectories_;
	const int B = std::max(1, std::min(trajectory_batch_limit, std::max(n_trajectories_, 1)));
	const int L = trajectory_len_limit;
	if (L < 2)
		throw std::runtime_error("run_simulation: trajectory_len_limit must be at least 2");
	const size_t W = state_words_, rs = mb_rand_state_size();

	timer_stats t_all("simulation_runner> buffered run");
	device_buffer ls0(ctx, W * B * 4), ls1(ctx, W * B * 4), lt0(ctx, (size_t)B * 4), lt1(ctx, (size_t)B * 4);
	device_buffer r0(ctx, B * rs), r1(ctx, B * rs), probs(ctx, initial_probs_.size() * 4);
	device_buffer ts(ctx, (size_t)L * W * B * 4), tt(ctx, (size_t)L * B * 4), th(ctx, (size_t)L * B * 4);
	device_buffer st(ctx, (size_t)B), trans(ctx, 8), scratch(ctx, mb_partition_scratch_size(B)), kept(ctx, 4);
	mirror::check(mb_memcpy(ctx, nullptr, probs.p, initial_probs_.data(), initial_probs_.size() * 4), "initialize");
	mirror::check(mb_memset_async(ctx, nullptr, trans.p, 0, 8), "initialize");
	stats_runner.bind(module, n, L);

	const device_buffer *cs = &ls0, *ct = &lt0, *cr = &r0, *ns = &ls1, *nt = &lt1, *nr = &r1;
	auto add_trajectories = [&](int count, int offset, unsigned long long first) {
		char* rr = cr->as<char>() + (size_t)offset * rs;
		mirror::check(mb_launch_initialize_random(module, nullptr, count, seed_, first, rr), "initialize_random");
		mirror::check(mb_launch_initialize_initial_state(module, nullptr, count, B, probs.as<float>(),
														 cs->as<uint32_t>() + offset, ct->as<float>() + offset, rr),
					  "initialize_initial_state");
	};
	int in_batch = (int)std::min<long long>(B, n);
	long long next_id = in_batch;
	if (in_batch > 0)
		add_trajectories(in_batch, 0, first_trajectory);
	while (in_batch > 0)
	{
		{
			timer_stats t("simulation_runner> simulate");
			mirror::check(mb_launch_simulate(module, nullptr, in_batch, B, L, cs->as<uint32_t>(), ct->as<float>(),
											 cr->p, ts.as<uint32_t>(), tt.as<float>(), th.as<float>(),
											 st.as<uint8_t>(), trans.as<unsigned long long>()),
						  "simulate");
		}
		{
			timer_stats t("simulation_runner> stats");
			stats_runner.process_batch({ ts.as<state_word_t>(), B }, { tt.as<float>(), B }, { th.as<float>(), B },
									   { cs->as<state_word_t>(), B }, { st.as<trajectory_status>(), B }, in_batch);
			// plugins may have used other streams
			mirror::check(mb_synchronize(ctx), "process_batch");
		}
		timer_stats t("simulation_runner> prepare_next_iter");
		mirror::check(mb_launch_partition(module, nullptr, in_batch, B, st.as<uint8_t>(), cs->as<uint32_t>(),
										  ct->as<float>(), cr->p, ns->as<uint32_t>(), nt->as<float>(), nr->p,
										  scratch.p, kept.as<unsigned>()),
					  "partition");
		unsigned remaining = 0;
		mirror::check(mb_memcpy(ctx, nullptr, &remaining, kept.p, sizeof remaining), "partition");
		std::swap(cs, ns);
		std::swap(ct, nt);
		std::swap(cr, nr);
		const int add = (int)std::max(0LL, std::min<long long>(B - (long long)remaining, n - next_id));
		if (add > 0)
			add_trajectories(add, (int)remaining, first_trajectory + (unsigned long long)next_id);
		next_id += add;
		in_batch = (int)remaining + add;
		epochs_++;
	}
	mirror::check(mb_memcpy(ctx, nullptr, &transitions_, trans.p, sizeof transitions_), "run_simulation");
}
