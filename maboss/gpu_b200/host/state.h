// state_t (src/state.h:7-25): a host-side network state of runtime size.
#pragma once

#include <cstddef>
#include <string>
#include <vector>

#include "state_word.h"

struct state_t
{
	static constexpr int word_size = 32;

	size_t state_size;
	std::vector<state_word_t> data;

	explicit state_t(size_t state_size);
	state_t(size_t state_size, const state_word_t* data);

	size_t words_n() const;
	bool is_set(int bit) const;
	void set(int bit);
	// names of the set nodes joined by " -- ", "<nil>" when none is set (src/state.cpp:29-48)
	std::string to_string(const std::vector<std::string>& names) const;
};
