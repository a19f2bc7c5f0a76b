// final_states_stats (src/statistics/final_states.h:8-34): histogram of the non-internal part of
// every trajectory's last state. Printed by visualize() only (no CSV, as the reference), unless
// final_csv is set.
#pragma once

#include "../kernel.h"
#include "../state.h"
#include "builtin.h"

class final_states_stats : public mirror::builtin_stats
{
	state_t noninternals_mask_;
	int noninternals_;

	void stats_params(float& tick, float& max_time, bool& discrete, std::vector<int>& ni) const override;

public:
	// Opt-in (no counterpart in the reference, which writes no final-state file): write_csv also
	// writes <prefix>_finalprob.csv (mb_result_write_final_csv's layout).
	bool final_csv = false;

	final_states_stats(state_t noninternals_mask, int noninternals, kernel_wrapper& final_states);

	void process_batch(soa_ptr<state_word_t> traj_states, soa_ptr<float> traj_times,
					   soa_ptr<float> traj_tr_entropies, soa_ptr<state_word_t> last_states,
					   soa_ptr<trajectory_status> traj_statuses, int n_trajectories) override;
	void write_csv(int n_trajectories, const std::vector<std::string>& nodes, const std::string& prefix) override;
	void describe(mirror::run_description& d) const override;
};
