// MaBoSS.GPU command line: the reference's src/main.cpp:1-169 flow (driver -> generator ->
// kernel_compiler -> simulation_runner with the final-state, fixed-point and window statistics ->
// CSV files or stdout), written against the C++ mirror classes of this directory.
//
//   MaBoSS.GPU [options] [-o prefix] model.bnd model.cfg
//     -o prefix        write <prefix>_probtraj.csv and <prefix>_fp.csv instead of printing
//     --mode M         exact (default; bit-exact with the reference), fast, or epoch (the buffered
//                      epoch loop through the statistics plugins)
//     --device D       CUDA device ordinal (default 0)
//     --emit-code      print the generated CUDA source and exit (no GPU needed)
//     --stats          print transitions and epochs to stderr
//     --max-noninternal K  accept up to K non-internal nodes (default 20 as the reference; at most
//                      112: above 20 the window statistics are sparse bins)
//     --cfg-overrides  node attributes defined again in the .cfg replace the .bnd's (the reference
//                      keeps the first definition)
//     --final-csv      with -o, also write <prefix>_finalprob.csv (the reference writes no
//                      final-state file)
//   MABOSS_DIAGS=1 prints the timer_stats scopes to stderr.
#include <algorithm>
#include <iostream>
#include <optional>

#include "generator.h"
#include "kernel_compiler.h"
#include "simulation_runner.h"
#include "state_word.h"
#include "statistics/final_states.h"
#include "statistics/fixed_states.h"
#include "statistics/stats_composite.h"
#include "statistics/window_average_small.h"
#include "timer.h"

namespace {

state_t create_noninternals_mask(driver& drv)
{
	state_t mask(drv.nodes.size());
	for (size_t i = 0; i < drv.nodes.size(); ++i)
		if (!drv.nodes[i].is_internal(drv))
			mask.set((int)i);
	return mask;
}

std::vector<float> create_initial_probs(driver& drv)
{
	std::vector<float> probs;
	for (auto& node : drv.nodes)
		probs.push_back(node.istate);
	return probs;
}

int do_compilation(driver& drv, bool discrete_time, int device, std::optional<kernel_compiler>& compiler)
{
	timer_stats stats("main> compilation");
	generator gen(drv);
	const std::string code = gen.generate_code();
	compiler.emplace(device);
	return compiler->compile_simulation(code, discrete_time) ? 1 : 0;
}

stats_composite do_simulation(bool discrete_time, float max_time, float time_tick, int sample_count, int state_size,
							  unsigned long long seed, std::vector<float> initial_probs,
							  const state_t& noninternals_mask, int noninternals_count, kernel_compiler& compiler,
							  int mode, bool print_stats, bool final_csv)
{
	timer_stats stats("main> simulation");
	simulation_runner r(sample_count, state_size, seed, std::move(initial_probs));
	r.mode = mode;
	stats_composite stats_runner;
	// the three plugins in the order of src/main.cpp:65-74
	auto final_stats = std::make_unique<final_states_stats>(noninternals_mask, noninternals_count, compiler.final_states);
	final_stats->final_csv = final_csv;
	stats_runner.add(std::move(final_stats));
	fixed_states_stats_builder::add_fixed_states_stats(stats_runner, (int)noninternals_mask.words_n());
	stats_runner.add(std::make_unique<window_average_small_stats>(
		time_tick, max_time, discrete_time, noninternals_mask, noninternals_count, r.trajectory_len_limit,
		r.trajectory_batch_limit, compiler.window_average_small));
	r.run_simulation(stats_runner, compiler.initialize_random, compiler.initialize_initial_state, compiler.simulate);
	stats_runner.finalize();
	if (print_stats)
		std::cerr << "transitions: " << r.transitions() << "  epochs: " << r.epochs() << std::endl;
	return stats_runner;
}

void do_visualization(stats_composite& stats_runner, int sample_count, const std::vector<std::string>& node_names,
					  const std::string& output_prefix)
{
	timer_stats stats("main> visualization");
	if (!output_prefix.empty())
		stats_runner.write_csv(sample_count, node_names, output_prefix);
	else
		stats_runner.visualize(sample_count, node_names);
}

void usage()
{
	std::cout << "Usage: MaBoSS.GPU [--mode exact|fast|epoch] [--device D] [--emit-code] [--stats] "
				 "[--max-noninternal K] [--cfg-overrides] [--final-csv] [-o prefix] bnd_file cfg_file"
			  << std::endl;
}

} // namespace

int main(int argc, char** argv)
{
	std::vector<std::string> args(argv + 1, argv + argc);
	std::string output_prefix, mode_name = "exact";
	int device = 0, max_noninternal = 20;
	bool emit = false, print_stats = false, cfg_overrides = false, final_csv = false;
	std::vector<std::string> files;
	for (size_t i = 0; i < args.size(); i++)
	{
		const std::string& a = args[i];
		if (a == "-o" && i + 1 < args.size())
			output_prefix = args[++i];
		else if (a == "--mode" && i + 1 < args.size())
			mode_name = args[++i];
		else if (a == "--device" && i + 1 < args.size())
			device = std::stoi(args[++i]);
		else if (a == "--max-noninternal" && i + 1 < args.size())
			max_noninternal = std::stoi(args[++i]);
		else if (a == "--emit-code")
			emit = true;
		else if (a == "--stats")
			print_stats = true;
		else if (a == "--cfg-overrides")
			cfg_overrides = true;
		else if (a == "--final-csv")
			final_csv = true;
		else if (!a.empty() && a[0] == '-')
		{
			usage();
			return 1;
		}
		else
			files.push_back(a);
	}
	if (files.size() != 2 || (mode_name != "exact" && mode_name != "fast" && mode_name != "epoch"))
	{
		usage();
		return 1;
	}
	const int mode =
		mode_name == "fast" ? MB_MODE_FUSED_FAST : mode_name == "epoch" ? MB_MODE_EPOCH : MB_MODE_FUSED_EXACT;

	try
	{
		driver drv;
		{
			timer_stats stats("main> parse");
			if (drv.parse(files[0], files[1]))
				return 1;
			if (cfg_overrides)
				drv.apply_cfg_overrides();
		}
		if (emit)
		{
			std::cout << generator(drv).generate_code();
			return 0;
		}

		const bool discrete_time = drv.constants["discrete_time"] != 0;
		const float max_time = drv.constants["max_time"];
		const float time_tick = drv.constants["time_tick"];
		const int sample_count = (int)drv.constants["sample_count"];
		const unsigned long long seed = (unsigned long long)drv.constants["seed_pseudorandom"];
		auto initial_probs = create_initial_probs(drv);
		auto noninternals_mask = create_noninternals_mask(drv);
		const int noninternals_count = (int)std::count_if(drv.nodes.begin(), drv.nodes.end(),
														  [&](const node_t& node) { return !node.is_internal(drv); });
		std::vector<std::string> node_names;
		for (auto& node : drv.nodes)
			node_names.push_back(node.name);

		// src/main.cpp:142-146
		if (noninternals_count > std::min(max_noninternal, 112))
		{
			std::cerr << "This executable supports a maximum of " << std::min(max_noninternal, 112)
					  << " non-internal nodes." << std::endl;
			return 1;
		}

		std::optional<kernel_compiler> compiler;
		if (do_compilation(drv, discrete_time, device, compiler))
			return 1;
		auto stats_runner =
			do_simulation(discrete_time, max_time, time_tick, sample_count, (int)drv.nodes.size(), seed,
						  std::move(initial_probs), noninternals_mask, noninternals_count, *compiler, mode, print_stats,
						  final_csv);
		do_visualization(stats_runner, sample_count, node_names, output_prefix);
	}
	catch (const std::exception& e)
	{
		std::cerr << e.what() << std::endl;
		return 1;
	}
	timer_stats::print_aggregate_stats();
	return 0;
}
