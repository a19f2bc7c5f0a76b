// Shared pieces of the C++ mirror of the reference's host classes (no reference counterpart):
// RAII for C ABI results and the error check used by every class.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "maboss_b200.h"

namespace mirror {

// Throws std::runtime_error with the C ABI's message when `s` is not MB_OK.
inline void check(mb_status s, const char* what)
{
	if (s != MB_OK)
		throw std::runtime_error(std::string(what) + ": " + mb_last_error());
}

struct result_handle
{
	mb_result r = nullptr;
	explicit result_handle(mb_result h) : r(h) {}
	~result_handle()
	{
		if (r)
			mb_result_free(r);
	}
	result_handle(const result_handle&) = delete;
	result_handle& operator=(const result_handle&) = delete;
};

// The statistics parameters of a run, gathered from the built-in plugins (the reference passes
// them to the plugins' constructors, src/main.cpp:65-74).
struct run_description
{
	bool has_windows = false;
	float time_tick = 1.f, max_time = 1.f;
	bool discrete_time = false;
	bool has_mask = false;
	std::vector<int> noninternal_nodes;
};

// Text of one section of a result (mb_result_format) with the caller's node names.
std::string format_section(mb_result r, int section, int format, const std::vector<std::string>& nodes);

} // namespace mirror
