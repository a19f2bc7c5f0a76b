// timer_stats (src/timer.h:26-41): named wall-clock scopes. The reference compiles the printing out
// (print_diags = false in src/timer.cpp:5); here it is switched on at run time by the environment
// variable MABOSS_DIAGS=1.
#pragma once

#include <chrono>
#include <map>
#include <string>

struct timer_stats
{
	explicit timer_stats(const char* name);
	~timer_stats();
	timer_stats(const timer_stats&) = delete;
	timer_stats& operator=(const timer_stats&) = delete;

	static void print_aggregate_stats();
	static bool enable_diags();

private:
	const char* name_;
	std::chrono::steady_clock::time_point start_;
	static std::map<std::string, size_t> aggregate_stats_;
};
