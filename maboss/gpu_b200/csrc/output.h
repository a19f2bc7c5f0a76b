// Text outputs of a run, in the reference's formats.
#pragma once

#include <string>
#include <vector>

#include "runtime.h"

namespace mb {

// state_t::to_string (src/state.cpp:29-48): names of the set nodes joined by " -- ", "<nil>" if none.
std::string state_name(const std::vector<std::string>& names, const unsigned* words, int n_nodes);

// window_average_small_stats::non_internal_idx_to_state (window_average_small.cpp:109-124).
std::vector<unsigned> noninternal_index_to_state(const std::vector<int>& noninternal, int n_nodes,
												 unsigned __int128 idx);

// <prefix>_probtraj.csv (window_average_small.cpp:181-250).
std::string format_probtraj_csv(const result& r, const std::vector<std::string>& names);
// <prefix>_fp.csv (fixed_states.cu:154-187).
std::string format_fp_csv(const result& r, const std::vector<std::string>& names);
// The final-state distribution as a CSV file (opt-in; the reference writes no such file):
// "Final States (n)", "Proba\tState", then one line per final state in non-internal index order.
std::string format_final_csv(const result& r, const std::vector<std::string>& names);
// stdout output of final_states_stats, fixed_states_stats and window_average_small_stats
// visualize() in the order of src/main.cpp:65-74.
std::string format_visualize(const result& r, const std::vector<std::string>& names);
// The three parts of it: final_states.cpp:53-68, fixed_states.cu:127-152, window_average_small.cpp:142-179.
std::string format_final_visualize(const result& r, const std::vector<std::string>& names);
std::string format_fixed_visualize(const result& r, const std::vector<std::string>& names);
std::string format_windows_visualize(const result& r, const std::vector<std::string>& names);

} // namespace mb
