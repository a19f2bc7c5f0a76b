#include "final_states.h"

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

// final states are printed only (src/statistics/final_states.cpp:70)
void final_states_stats::write_csv(int, const std::vector<std::string>&, const std::string&) {}
