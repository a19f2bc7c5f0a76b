#include "stats_composite.h"

void stats_composite::add(stats_ptr&& stat) { composed_stats_.emplace_back(std::move(stat)); }

void stats_composite::process_batch(soa_ptr<state_word_t> traj_states, soa_ptr<float> traj_times,
									soa_ptr<float> traj_tr_entropies, soa_ptr<state_word_t> last_states,
									soa_ptr<trajectory_status> traj_statuses, int n_trajectories)
{
	for (auto& s : composed_stats_)
		s->process_batch(traj_states, traj_times, traj_tr_entropies, last_states, traj_statuses, n_trajectories);
}

void stats_composite::finalize()
{
	for (auto& s : composed_stats_)
		s->finalize();
}

void stats_composite::visualize(int n_trajectories, const std::vector<std::string>& nodes)
{
	for (auto& s : composed_stats_)
		s->visualize(n_trajectories, nodes);
}

void stats_composite::write_csv(int n_trajectories, const std::vector<std::string>& nodes, const std::string& prefix)
{
	for (auto& s : composed_stats_)
		s->write_csv(n_trajectories, nodes, prefix);
}

void stats_composite::bind(mb_module module, long long n_trajectories, int trajectory_len_limit)
{
	for (auto& s : composed_stats_)
		s->bind(module, n_trajectories, trajectory_len_limit);
}

bool stats_composite::fusable() const
{
	if (composed_stats_.empty())
		return false;
	for (auto& s : composed_stats_)
		if (!s->fusable())
			return false;
	return describe().has_mask;
}

mirror::run_description stats_composite::describe() const
{
	mirror::run_description d;
	for (auto& s : composed_stats_)
		s->describe(d);
	return d;
}

void stats_composite::take_result(const std::shared_ptr<mirror::result_handle>& r)
{
	for (auto& s : composed_stats_)
		s->take_result(r);
}
