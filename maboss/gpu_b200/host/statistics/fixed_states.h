// fixed_states_stats (src/statistics/fixed_states.h:11-44): the distinct fixed points reached and
// how many trajectories ended in each. Output: <prefix>_fp.csv, or "fixed points:" on stdout.
// One class for every state width (the reference instantiates a template per word count).
#pragma once

#include "builtin.h"

class stats_composite;

class fixed_states_stats : public mirror::builtin_stats
{
	int state_words_;

	void stats_params(float& tick, float& max_time, bool& discrete, std::vector<int>& ni) const override;

public:
	explicit fixed_states_stats(int state_words);

	void process_batch(soa_ptr<state_word_t> traj_states, soa_ptr<float> traj_times,
					   soa_ptr<float> traj_tr_entropies, soa_ptr<state_word_t> last_states,
					   soa_ptr<trajectory_status> traj_statuses, int n_trajectories) override;
	void write_csv(int n_trajectories, const std::vector<std::string>& nodes, const std::string& prefix) override;
};

class fixed_states_stats_builder
{
public:
	static void add_fixed_states_stats(stats_composite& stats_runner, int state_words);
};
