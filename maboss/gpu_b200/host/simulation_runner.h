// simulation_runner (src/simulation_runner.h:8-24): simulates n trajectories and hands them to the
// statistics plugins.
//
// When every plugin of the stats_composite is one of the three built-in statistics, the run is one
// persistent fused kernel that computes them without trajectory buffers (`mode`, default
// MB_MODE_FUSED_EXACT: bit-identical trajectories to the reference algorithm). With any other
// plugin, or with mode = MB_MODE_EPOCH, it is the reference's buffered loop
// (src/simulation_runner.cu:54-180): epochs of trajectory_len_limit slots over a batch of
// trajectory_batch_limit trajectories in SoA buffers, process_batch of every plugin after each
// epoch, then the partition of the unfinished trajectories and the refill of the batch.
#pragma once

#include <vector>

#include "kernel.h"
#include "statistics/stats_composite.h"

class simulation_runner
{
	int n_trajectories_;
	int state_size_;
	int state_words_;
	unsigned long long seed_;
	std::vector<float> initial_probs_;
	unsigned long long transitions_ = 0;
	int epochs_ = 0;

	void run_fused(stats_composite& stats_runner, mb_module module);
	void run_buffered(stats_composite& stats_runner, mb_module module);

public:
	int trajectory_len_limit;
	int trajectory_batch_limit;
	int mode = MB_MODE_FUSED_EXACT;			// MB_MODE_FUSED_EXACT, MB_MODE_FUSED_FAST or MB_MODE_EPOCH
	unsigned long long first_trajectory = 0; // random stream of trajectory 0 (sharded runs)

	simulation_runner(int n_trajectories, int state_size, unsigned long long seed, std::vector<float> initial_probs);

	void run_simulation(stats_composite& stats_runner, kernel_wrapper& initialize_random,
						kernel_wrapper& initialize_initial_state, kernel_wrapper& simulate);

	unsigned long long transitions() const { return transitions_; } // recorded steps of the last run
	int epochs() const { return epochs_; }							// 1 for a fused run
};
