#include "timer.h"

#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>

std::map<std::string, size_t> timer_stats::aggregate_stats_;

bool timer_stats::enable_diags()
{
	static const bool on = [] {
		const char* v = std::getenv("MABOSS_DIAGS");
		return v && v[0] != '\0' && std::strcmp(v, "0") != 0;
	}();
	return on;
}

timer_stats::timer_stats(const char* name) : name_(name), start_(std::chrono::steady_clock::now()) {}

timer_stats::~timer_stats()
{
	if (!enable_diags())
		return;
	const auto us = (size_t)std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() -
																				  start_)
						.count();
	aggregate_stats_[name_] += us;
	std::cerr << std::left << std::setw(50) << name_ << ":" << std::right << std::setw(10) << us << " us" << std::endl;
}

void timer_stats::print_aggregate_stats()
{
	if (!enable_diags())
		return;
	std::cerr << "Aggregate stats:" << std::endl;
	for (auto& [name, us] : aggregate_stats_)
		std::cerr << std::left << std::setw(50) << name << ":" << std::right << std::setw(10) << us << " us"
				  << std::endl;
}
