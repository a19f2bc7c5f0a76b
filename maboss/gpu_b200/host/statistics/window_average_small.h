// window_average_small_stats (src/statistics/window_average_small.h:11-54): per window of time_tick,
// the time-averaged probability of every non-internal state and the transition entropy.
// Output: <prefix>_probtraj.csv, or the windows on stdout.
#pragma once

#include "../kernel.h"
#include "../state.h"
#include "builtin.h"

class window_average_small_stats : public mirror::builtin_stats
{
	float window_size_;
	float max_time_;
	bool discrete_time_;
	state_t noninternals_mask_;
	size_t max_traj_len_;
	size_t max_n_trajectories_;

	void stats_params(float& tick, float& max_time, bool& discrete, std::vector<int>& ni) const override;

public:
	// window_average_small.h:31: the dense index of a non-internal state -> the state
	static state_t non_internal_idx_to_state(const state_t& noninternals_mask, int idx);

	window_average_small_stats(float window_size, float max_time, bool discrete_time, state_t noninternals_mask,
							   size_t non_internals, size_t max_traj_len, size_t max_n_trajectories,
							   kernel_wrapper& window_average_small);

	void process_batch(soa_ptr<state_word_t> traj_states, soa_ptr<float> traj_times,
					   soa_ptr<float> traj_tr_entropies, soa_ptr<state_word_t> last_states,
					   soa_ptr<trajectory_status> traj_statuses, int n_trajectories) override;
	void write_csv(int n_trajectories, const std::vector<std::string>& nodes, const std::string& prefix) override;
	void describe(mirror::run_description& d) const override;
};
