#include "fixed_states.h"

#include <fstream>

#include "stats_composite.h"

fixed_states_stats::fixed_states_stats(int state_words)
	: builtin_stats(MB_STATS_FIXED, MB_SECTION_FIXED), state_words_(state_words)
{}

void fixed_states_stats::stats_params(float& tick, float& max_time, bool& discrete, std::vector<int>& ni) const
{
	tick = max_time = 1.f;
	discrete = false;
	ni.clear();
}

void fixed_states_stats::process_batch(soa_ptr<state_word_t>, soa_ptr<float>, soa_ptr<float>,
									   soa_ptr<state_word_t> last_states, soa_ptr<trajectory_status> traj_statuses,
									   int n_trajectories)
{
	if (!acc_)
		throw std::runtime_error("fixed_states_stats: process_batch outside a run");
	mirror::check(mb_launch_fixed_states_stats(acc_, nullptr, n_trajectories, last_states.stride, last_states.get(),
											   reinterpret_cast<const uint8_t*>(traj_statuses.get())),
				  "fixed_states");
}

void fixed_states_stats::write_csv(int, const std::vector<std::string>& nodes, const std::string& prefix)
{
	const std::string path = prefix + "_fp.csv";
	std::ofstream f(path);
	if (!f)
		throw std::runtime_error("cannot write " + path);
	f << mirror::format_section(result(), MB_SECTION_FIXED, MB_FORMAT_CSV, nodes);
}

void fixed_states_stats_builder::add_fixed_states_stats(stats_composite& stats_runner, int state_words)
{
	stats_runner.add(std::make_unique<fixed_states_stats>(state_words));
}
