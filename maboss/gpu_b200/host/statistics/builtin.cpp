#include "builtin.h"

#include <iostream>

namespace mirror {

std::string format_section(mb_result r, int section, int format, const std::vector<std::string>& nodes)
{
	std::vector<const char*> names;
	for (auto& n : nodes)
		names.push_back(n.c_str());
	size_t len = 0;
	check(mb_result_format(r, section, format, names.data(), (int)names.size(), nullptr, 0, &len), "format");
	std::string text(len + 1, '\0');
	check(mb_result_format(r, section, format, names.data(), (int)names.size(), text.data(), text.size(), &len),
		  "format");
	text.resize(len);
	return text;
}

builtin_stats::~builtin_stats()
{
	if (acc_)
		mb_stats_free(acc_);
}

void builtin_stats::bind(mb_module module, long long n_trajectories, int trajectory_len_limit)
{
	float tick = 1.f, max_time = 1.f;
	bool discrete = false;
	std::vector<int> ni;
	stats_params(tick, max_time, discrete, ni);
	if (acc_)
		mb_stats_free(acc_);
	acc_ = nullptr;
	check(mb_stats_create_sections(module, tick, max_time, discrete ? 1 : 0, ni.data(), (int)ni.size(),
								   n_trajectories, section_bit_, &acc_),
		  "statistics");
	n_ = n_trajectories;
	traj_len_ = trajectory_len_limit;
	result_.reset();
}

void builtin_stats::finalize()
{
	if (!acc_)
		return; // fused run: the result is already there
	mb_result r = nullptr;
	check(mb_stats_finalize(acc_, n_, &r), "finalize");
	result_ = std::make_shared<result_handle>(r);
	mb_stats_free(acc_);
	acc_ = nullptr;
}

void builtin_stats::take_result(std::shared_ptr<result_handle> r)
{
	if (acc_)
		mb_stats_free(acc_);
	acc_ = nullptr;
	result_ = std::move(r);
}

mb_result builtin_stats::result() const
{
	if (!result_)
		throw std::runtime_error("statistics: no finalized result (run the simulation and finalize first)");
	return result_->r;
}

void builtin_stats::visualize(int, const std::vector<std::string>& nodes)
{
	std::cout << format_section(result(), section_, MB_FORMAT_VISUALIZE, nodes);
}

} // namespace mirror
