#include "state.h"

state_t::state_t(size_t n) : state_size(n), data((n + word_size - 1) / word_size, 0u) {}

state_t::state_t(size_t n, const state_word_t* words) : state_t(n)
{
	for (size_t w = 0; w < data.size(); w++)
		data[w] = words[w];
}

size_t state_t::words_n() const { return data.size(); }

bool state_t::is_set(int bit) const { return (data[bit / word_size] >> (bit % word_size)) & 1u; }

void state_t::set(int bit) { data[bit / word_size] |= 1u << (bit % word_size); }

std::string state_t::to_string(const std::vector<std::string>& names) const
{
	std::string out;
	for (size_t i = 0; i < state_size; i++)
	{
		if (!is_set((int)i))
			continue;
		if (!out.empty())
			out += " -- ";
		out += names[i];
	}
	return out.empty() ? std::string("<nil>") : out;
}
