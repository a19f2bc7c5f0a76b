// Test driver for the C++ mirror of the reference's host classes (compiled by tests/test_mirror.py).
//
//   mirror_test frontend BND CFG OUT      parse with `driver`, set $variables/constants/istate via the
//                                         public members, write the generated code to OUT, print members
//   mirror_test plugin BND CFG N PREFIX   GPU: a buffered run with the three built-in statistics plus a
//                                         user plugin that counts recorded slots (time > 0) through the
//                                         SoA views; writes PREFIX_buffered_* and PREFIX_fused_* CSVs and
//                                         prints "transitions <runner> counted <plugin> fused <runner>
//                                         epochs <buffered> <fused>"
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "generator.h"
#include "kernel_compiler.h"
#include "simulation_runner.h"
#include "statistics/final_states.h"
#include "statistics/fixed_states.h"
#include "statistics/stats_composite.h"
#include "statistics/window_average_small.h"

namespace {

// A plugin of the kind a user of the reference writes: it reads the epoch's trajectory times back to
// the host and counts the recorded slots (the transition count of the benchmark).
class counting_stats : public stats
{
	mb_context ctx_;
	int traj_len_;
	unsigned long long count_ = 0;

public:
	counting_stats(mb_context ctx, int traj_len) : ctx_(ctx), traj_len_(traj_len) {}
	unsigned long long count() const { return count_; }

	void process_batch(soa_ptr<state_word_t>, soa_ptr<float> traj_times, soa_ptr<float>, soa_ptr<state_word_t>,
					   soa_ptr<trajectory_status>, int n) override
	{
		std::vector<float> t((size_t)traj_len_ * traj_times.stride);
		mirror::check(mb_memcpy(ctx_, nullptr, t.data(), traj_times.get(), t.size() * sizeof(float)), "copy");
		for (int s = 1; s < traj_len_; s++) // slot 0 holds the epoch's start time
			for (int i = 0; i < n; i++)
				count_ += t[(size_t)s * traj_times.stride + i] > 0.f ? 1 : 0;
	}
	void visualize(int, const std::vector<std::string>&) override {}
	void write_csv(int, const std::vector<std::string>&, const std::string&) override {}
};

state_t mask_of(driver& drv)
{
	state_t m(drv.nodes.size());
	for (size_t i = 0; i < drv.nodes.size(); i++)
		if (!drv.nodes[i].is_internal(drv))
			m.set((int)i);
	return m;
}

void add_builtins(stats_composite& sc, driver& drv, kernel_compiler& kc, const simulation_runner& r)
{
	const state_t mask = mask_of(drv);
	int k = 0;
	for (auto& n : drv.nodes)
		k += n.is_internal(drv) ? 0 : 1;
	sc.add(std::make_unique<final_states_stats>(mask, k, kc.final_states));
	fixed_states_stats_builder::add_fixed_states_stats(sc, (int)mask.words_n());
	sc.add(std::make_unique<window_average_small_stats>(drv.constants["time_tick"], drv.constants["max_time"],
														drv.constants["discrete_time"] != 0, mask, k,
														r.trajectory_len_limit, r.trajectory_batch_limit,
														kc.window_average_small));
}

int frontend(const char* bnd, const char* cfg, const char* out)
{
	driver drv;
	if (drv.parse(bnd, cfg))
		return 2;
	std::cout << "nodes " << drv.nodes.size() << "\n";
	for (auto& n : drv.nodes)
		std::cout << "node " << n.name << " " << n.istate << " " << (n.is_internal(drv) ? 1 : 0) << "\n";
	for (auto& [k, v] : drv.constants)
		std::cout << "constant " << k << " " << v << "\n";
	for (auto& [k, v] : drv.variables)
		std::cout << "variable " << k << " " << v << "\n";
	// edits through the public members reach the generated code
	if (!drv.variables.empty())
		drv.variables.begin()->second *= 2.f;
	drv.constants["max_time"] = 7.5f;
	drv.nodes[0].istate = 0.25f;
	std::ofstream(out) << generator(drv).generate_code();
	return 0;
}

int plugin(const char* bnd, const char* cfg, int n, const std::string& prefix)
{
	driver drv;
	if (drv.parse(bnd, cfg))
		return 2;
	std::vector<std::string> names;
	std::vector<float> probs;
	for (auto& node : drv.nodes)
	{
		names.push_back(node.name);
		probs.push_back(node.istate);
	}
	const unsigned long long seed = (unsigned long long)drv.constants["seed_pseudorandom"];
	kernel_compiler kc;
	if (kc.compile_simulation(generator(drv).generate_code(), drv.constants["discrete_time"] != 0))
		return 3;

	// buffered: a user plugin forces the reference's epoch loop; small batches exercise the refill
	simulation_runner rb(n, (int)drv.nodes.size(), seed, probs);
	rb.trajectory_batch_limit = std::max(1, n / 3);
	stats_composite sb;
	add_builtins(sb, drv, kc, rb);
	auto counter = std::make_unique<counting_stats>(kc.context(), rb.trajectory_len_limit);
	counting_stats* cp = counter.get();
	sb.add(std::move(counter));
	rb.run_simulation(sb, kc.initialize_random, kc.initialize_initial_state, kc.simulate);
	sb.finalize();
	sb.write_csv(n, names, prefix + "_buffered");

	// fused: built-in plugins only
	simulation_runner rf(n, (int)drv.nodes.size(), seed, probs);
	stats_composite sf;
	add_builtins(sf, drv, kc, rf);
	rf.run_simulation(sf, kc.initialize_random, kc.initialize_initial_state, kc.simulate);
	sf.finalize();
	sf.write_csv(n, names, prefix + "_fused");
	std::cout << "transitions " << rb.transitions() << " counted " << cp->count() << " fused " << rf.transitions()
			  << " epochs " << rb.epochs() << " " << rf.epochs() << std::endl;
	return 0;
}

} // namespace

int main(int argc, char** argv)
{
	try
	{
		const std::string cmd = argc > 1 ? argv[1] : "";
		if (cmd == "frontend" && argc == 5)
			return frontend(argv[2], argv[3], argv[4]);
		if (cmd == "plugin" && argc == 6)
			return plugin(argv[2], argv[3], std::atoi(argv[4]), argv[5]);
	}
	catch (const std::exception& e)
	{
		std::cerr << "error: " << e.what() << std::endl;
		return 1;
	}
	std::cerr << "usage: mirror_test frontend BND CFG OUT | plugin BND CFG N PREFIX" << std::endl;
	return 64;
}
