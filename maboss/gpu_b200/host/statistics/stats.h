// stats (src/statistics/stats.h:15-29): a statistics plugin fed with every epoch of trajectories.
//
// The trajectory buffers are Structure-of-Arrays with a row stride of the batch capacity B, handed
// over as soa_ptr views (the reference hands thrust::device_ptr to Array-of-Structures buffers):
//   traj_states[(slot * W + word) * B + i], traj_times[slot * B + i], traj_tr_entropies[slot * B + i],
//   last_states[word * B + i], traj_statuses[i]          for trajectories i < n_trajectories.
// A slot whose time is 0 holds no step. The buffers belong to the simulation_runner and are valid
// during the call only; kernels may be launched on any stream (the runner waits for the whole device
// before it reuses the buffers).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../maboss_b200_mirror.h"
#include "../state_word.h"
#include "../trajectory_status.h"

template <typename T>
struct soa_ptr
{
	T* ptr = nullptr;
	int stride = 0; // batch capacity B

	T* get() const { return ptr; }
};

class stats;
using stats_ptr = std::unique_ptr<stats>;

class stats
{
public:
	virtual ~stats() = default;

	virtual void process_batch(soa_ptr<state_word_t> traj_states, soa_ptr<float> traj_times,
							   soa_ptr<float> traj_tr_entropies, soa_ptr<state_word_t> last_states,
							   soa_ptr<trajectory_status> traj_statuses, int n_trajectories) = 0;

	virtual void finalize() {}

	virtual void visualize(int n_trajectories, const std::vector<std::string>& nodes) = 0;
	virtual void write_csv(int n_trajectories, const std::vector<std::string>& nodes, const std::string& prefix) = 0;

	// ---- hooks of the runner (defaults keep a user plugin on the buffered path)
	// Called once before the first batch of a buffered run.
	virtual void bind(mb_module module, long long n_trajectories, int trajectory_len_limit)
	{
		(void)module, (void)n_trajectories, (void)trajectory_len_limit;
	}
	// True for the built-in statistics, which the fused kernel computes without buffers.
	virtual bool fusable() const { return false; }
	// Fused runs: what the plugin knows of the run's statistics parameters, and the run's result.
	virtual void describe(mirror::run_description& d) const { (void)d; }
	virtual void take_result(std::shared_ptr<mirror::result_handle> r) { (void)r; }
};
