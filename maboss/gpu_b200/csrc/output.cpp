// Text outputs of a run in the reference's formats. Numbers go through `std::ostream << float`
// (default precision, 6 significant digits) exactly like the reference writers.
#include "output.h"

#include <cmath>
#include <sstream>

namespace mb {

std::string state_name(const std::vector<std::string>& names, const unsigned* words, int n_nodes)
{
	std::string s;
	bool first = true;
	for (int i = 0; i < n_nodes; i++)
	{
		if (words[i / 32] & (1u << (i % 32)))
		{
			if (!first)
				s += " -- ";
			first = false;
			s += names[i];
		}
	}
	return s.empty() ? "<nil>" : s;
}

std::vector<unsigned> noninternal_index_to_state(const std::vector<int>& noninternal, int n_nodes,
												 unsigned __int128 idx)
{
	std::vector<unsigned> w((n_nodes + 31) / 32, 0u);
	for (size_t k = 0; k < noninternal.size(); k++)
		if ((unsigned)(idx >> k) & 1u)
			w[noninternal[k] / 32] |= 1u << (noninternal[k] % 32);
	return w;
}

namespace {

// The non-zero probabilities of window w (as the reference prints them: floats), in increasing order
// of the non-internal index, from the dense histogram or the sparse entries (more than 20
// non-internal nodes, or a large histogram's non-zero cells).
std::vector<std::pair<unsigned __int128, float>> window_entries(const result& r, int w)
{
	std::vector<std::pair<unsigned __int128, float>> out;
	if (r.sparse_windows())
	{
		for (size_t i = r.sp_begin[w]; i < r.sp_begin[w + 1]; i++)
		{
			const float p = (float)r.sparse_prob(i);
			if (p != 0.f)
				out.push_back({ r.sp_idx[i], p });
		}
		return out;
	}
	for (unsigned b = 0; b < r.n_bins; b++)
	{
		const float p = (float)r.window_prob(w, b);
		if (p != 0.f)
			out.push_back({ b, p });
	}
	return out;
}

float window_entropy(const std::vector<std::pair<unsigned __int128, float>>& entries)
{
	float entropy = 0.f;
	for (auto& e : entries)
		entropy += -std::log2(e.second) * e.second;
	return entropy;
}

std::string idx_name(const result& r, const std::vector<std::string>& names, unsigned __int128 b)
{
	auto st = noninternal_index_to_state(r.noninternal_nodes, r.state_size, b);
	return state_name(names, st.data(), r.state_size);
}

} // namespace

std::string format_probtraj_csv(const result& r, const std::vector<std::string>& names)
{
	std::ostringstream ofs;
	std::vector<std::vector<std::pair<unsigned __int128, float>>> entries(r.n_windows);
	size_t max_states = 0;
	for (int w = 0; w < r.n_windows; w++)
	{
		entries[w] = window_entries(r, w);
		max_states = std::max(max_states, entries[w].size());
	}
	ofs << "Time\tTH\tErrorTH\tH\tHD=0";
	for (size_t i = 0; i < max_states; i++)
		ofs << "\tState\tProba\tErrorProba";
	ofs << std::endl;
	for (int w = 0; w < r.n_windows; w++)
	{
		const float th = (float)r.window_th(w);
		const float entropy = window_entropy(entries[w]);
		ofs << (float)w * r.time_tick << "\t";
		ofs << th << "\t" << 0.f << "\t" << entropy << "\t" << 0.f;
		for (auto& e : entries[w])
			ofs << "\t" << idx_name(r, names, e.first) << "\t" << e.second << "\t" << 0.f;
		ofs << std::endl;
	}
	return ofs.str();
}

std::string format_fp_csv(const result& r, const std::vector<std::string>& names)
{
	std::ostringstream ofs;
	const size_t nfp = r.fixed_counts.size();
	ofs << "Fixed Points (" << nfp << ")" << std::endl;
	ofs << "FP\tProba\tState";
	for (auto& n : names)
		ofs << "\t" << n;
	ofs << std::endl;
	for (size_t i = 0; i < nfp; i++)
	{
		const unsigned* w = r.fixed_states.data() + i * r.state_words;
		ofs << "#" << i << "\t" << ((float)r.fixed_counts[i]) / (float)r.n_traj << "\t"
			<< state_name(names, w, r.state_size);
		for (int n = 0; n < r.state_size; n++)
			ofs << "\t" << ((w[n / 32] >> (n % 32)) & 1u);
		ofs << std::endl;
	}
	return ofs.str();
}

std::string format_final_visualize(const result& r, const std::vector<std::string>& names)
{
	std::ostringstream os;
	os << "final points:" << std::endl;
	if (r.wide)
		for (size_t i = 0; i < r.fin_idx.size(); i++)
			os << (float)r.fin_cnt[i] / (float)r.n_traj << " " << idx_name(r, names, r.fin_idx[i]) << std::endl;
	for (unsigned b = 0; b < r.n_bins && b < r.final_cnt.size(); b++)
		if (r.final_cnt[b] != 0)
			os << (float)r.final_cnt[b] / (float)r.n_traj << " " << idx_name(r, names, b) << std::endl;
	return os.str();
}

std::string format_final_csv(const result& r, const std::vector<std::string>& names)
{
	// the final-state distribution in the layout of the fixed-point file (no counterpart in the
	// reference, whose final_states_stats::write_csv writes nothing, final_states.cpp:70)
	std::vector<std::pair<unsigned __int128, unsigned>> rows;
	if (r.wide)
		for (size_t i = 0; i < r.fin_idx.size(); i++)
			rows.push_back({ r.fin_idx[i], r.fin_cnt[i] });
	for (unsigned b = 0; b < r.n_bins && b < r.final_cnt.size(); b++)
		if (r.final_cnt[b] != 0)
			rows.push_back({ b, r.final_cnt[b] });
	std::ostringstream os;
	os << "Final States (" << rows.size() << ")" << std::endl;
	os << "Proba\tState" << std::endl;
	for (auto& [idx, c] : rows)
		os << (float)c / (float)r.n_traj << "\t" << idx_name(r, names, idx) << std::endl;
	return os.str();
}

std::string format_fixed_visualize(const result& r, const std::vector<std::string>& names)
{
	std::ostringstream os;
	os << "fixed points:" << std::endl;
	for (size_t i = 0; i < r.fixed_counts.size(); i++)
		os << (float)r.fixed_counts[i] / (float)r.n_traj << " "
		   << state_name(names, r.fixed_states.data() + i * r.state_words, r.state_size) << std::endl;
	return os.str();
}

std::string format_visualize(const result& r, const std::vector<std::string>& names)
{
	return format_final_visualize(r, names) + format_fixed_visualize(r, names) + format_windows_visualize(r, names);
}

std::string format_windows_visualize(const result& r, const std::vector<std::string>& names)
{
	std::ostringstream os;
	if (!(r.sections & 1u))
		return os.str();
	for (int w = 0; w < r.n_windows; w++)
	{
		const auto entries = window_entries(r, w);
		os << "window (" << (float)w * r.time_tick << ", " << (float)(w + 1) * r.time_tick << "]" << std::endl;
		os << "entropy: " << window_entropy(entries) << std::endl;
		os << "transition entropy: " << (float)r.window_th(w) << std::endl;
		for (auto& e : entries)
			os << e.second << " " << idx_name(r, names, e.first) << std::endl;
	}
	return os.str();
}

} // namespace mb
