#include "final_states.h"

#include <fstream>

final_states_stats::final_states_stats(state_t noninternals_mask, int noninternals, kernel_wrapper&)
	: builtin_stats(MB_STATS_FINAL, MB_SECTION_FINAL),
	  noninternals_mask_(std::move(noninternals_mask)),
	  noninternals_(noninternals)
{}

void final_states_stats::stats_params(float& tick, float& max_time, bool& discrete, std::vector<int>& ni) const
{
	tick = max_time = 1.f;
	discrete = false;
	ni.clear();
	for (size_t i = 0; i < noninternals_mask_.state_size; i++)
		if (noninternals_mask_.is_set((int)i))
			ni.push_back((int)i);
}

void final_states_stats::describe(mirror::run_description& d) const
{
	d.has_mask = true;
	float t, m;
	bool disc;
	stats_params(t, m, disc, d.noninternal_nodes);
}

void final_states_stats::process_batch(soa_ptr<state_word_t>, soa_ptr<float>, soa_ptr<float>,
									   soa_ptr<state_word_t> last_states, soa_ptr<trajectory_status> traj_statuses,
									   int n_trajectories)
{
	if (!acc_)
		throw std::runtime_error("final_states_stats: process_batch outside a run");
	mirror::check(mb_launch_final_states_stats(acc_, nullptr, n_trajectories, last_states.stride, last_states.get(),
											   reinterpret_cast<const uint8_t*>(traj_statuses.get())),
				  "final_states");
}

// final states are printed only (src/statistics/final_states.cpp:70), unless final_csv is set
void final_states_stats::write_csv(int, const std::vector<std::string>& nodes, const std::string& prefix)
{
	if (!final_csv)
		return;
	if (!result_)
		throw std::runtime_error("final_states_stats: write_csv before finalize");
	std::ofstream f(prefix + "_finalprob.csv");
	if (!f)
		throw std::runtime_error("cannot write " + prefix + "_finalprob.csv");
	f << mirror::format_section(result_->r, MB_SECTION_FINAL, MB_FORMAT_CSV_FINAL_STATES, nodes);
}
