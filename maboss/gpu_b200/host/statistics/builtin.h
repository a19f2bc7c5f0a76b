// Common part of the three built-in statistics: their device accumulators (one section of
// mb_stats each) in a buffered run, or the shared result of a fused run.
#pragma once

#include "stats.h"

namespace mirror {

class builtin_stats : public stats
{
protected:
	unsigned section_bit_;	 // MB_STATS_WINDOWS / MB_STATS_FINAL / MB_STATS_FIXED
	int section_;			 // MB_SECTION_*
	mb_stats acc_ = nullptr; // buffered runs
	long long n_ = 0;
	int traj_len_ = 0;
	std::shared_ptr<result_handle> result_;

	explicit builtin_stats(unsigned section_bit, int section) : section_bit_(section_bit), section_(section) {}
	// parameters of mb_stats_create_sections for this plugin
	virtual void stats_params(float& tick, float& max_time, bool& discrete, std::vector<int>& ni) const = 0;
	mb_result result() const;

public:
	~builtin_stats() override;
	void bind(mb_module module, long long n_trajectories, int trajectory_len_limit) override;
	void finalize() override;
	bool fusable() const override { return true; }
	void take_result(std::shared_ptr<result_handle> r) override;
	void visualize(int n_trajectories, const std::vector<std::string>& nodes) override;
};

} // namespace mirror
