#include "window_average_small.h"

#include <fstream>

namespace {

std::vector<int> mask_nodes(const state_t& mask)
{
	std::vector<int> ni;
	for (size_t i = 0; i < mask.state_size; i++)
		if (mask.is_set((int)i))
			ni.push_back((int)i);
	return ni;
}

} // namespace

window_average_small_stats::window_average_small_stats(float window_size, float max_time, bool discrete_time,
													   state_t noninternals_mask, size_t, size_t max_traj_len,
													   size_t max_n_trajectories, kernel_wrapper&)
	: builtin_stats(MB_STATS_WINDOWS, MB_SECTION_WINDOWS),
	  window_size_(window_size),
	  max_time_(max_time),
	  discrete_time_(discrete_time),
	  noninternals_mask_(std::move(noninternals_mask)),
	  max_traj_len_(max_traj_len),
	  max_n_trajectories_(max_n_trajectories)
{}

state_t window_average_small_stats::non_internal_idx_to_state(const state_t& noninternals_mask, int idx)
{
	state_t s(noninternals_mask.state_size);
	int k = 0;
	for (int i : mask_nodes(noninternals_mask))
		if ((idx >> k++) & 1)
			s.set(i);
	return s;
}

void window_average_small_stats::stats_params(float& tick, float& max_time, bool& discrete, std::vector<int>& ni) const
{
	tick = window_size_;
	max_time = max_time_;
	discrete = discrete_time_;
	ni = mask_nodes(noninternals_mask_);
}

void window_average_small_stats::describe(mirror::run_description& d) const
{
	d.has_windows = true;
	d.time_tick = window_size_;
	d.max_time = max_time_;
	d.discrete_time = discrete_time_;
	d.has_mask = true;
	d.noninternal_nodes = mask_nodes(noninternals_mask_);
}

void window_average_small_stats::process_batch(soa_ptr<state_word_t> traj_states, soa_ptr<float> traj_times,
											   soa_ptr<float> traj_tr_entropies, soa_ptr<state_word_t>,
											   soa_ptr<trajectory_status>, int n_trajectories)
{
	if (!acc_)
		throw std::runtime_error("window_average_small_stats: process_batch outside a run");
	mirror::check(mb_launch_window_average_stats(acc_, nullptr, n_trajectories, traj_states.stride, traj_len_,
												 traj_states.get(), traj_times.get(), traj_tr_entropies.get()),
				  "window_average_small");
}

void window_average_small_stats::write_csv(int, const std::vector<std::string>& nodes, const std::string& prefix)
{
	const std::string path = prefix + "_probtraj.csv";
	std::ofstream f(path);
	if (!f)
		throw std::runtime_error("cannot write " + path);
	f << mirror::format_section(result(), MB_SECTION_WINDOWS, MB_FORMAT_CSV, nodes);
}
