// stats_composite (src/statistics/stats_composite.h:5-20): the plugins of a run, called in order.
#pragma once

#include "stats.h"

class stats_composite
{
	std::vector<stats_ptr> composed_stats_;

public:
	void add(stats_ptr&& stat);

	void process_batch(soa_ptr<state_word_t> traj_states, soa_ptr<float> traj_times,
					   soa_ptr<float> traj_tr_entropies, soa_ptr<state_word_t> last_states,
					   soa_ptr<trajectory_status> traj_statuses, int n_trajectories);

	void finalize();

	void visualize(int n_trajectories, const std::vector<std::string>& nodes);
	void write_csv(int n_trajectories, const std::vector<std::string>& nodes, const std::string& prefix);

	// ---- used by simulation_runner
	void bind(mb_module module, long long n_trajectories, int trajectory_len_limit);
	bool fusable() const; // every plugin is built in and one of them knows the non-internal mask
	mirror::run_description describe() const;
	void take_result(const std::shared_ptr<mirror::result_handle>& r);
};
