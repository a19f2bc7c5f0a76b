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

std::vector<unsigned> noninternal_index_to_state(const std::vector<int>& noninternal, int n_nodes, unsigned idx)
{
	std::vector<unsigned> w((n_nodes + 31) / 32, 0u);
	for (size_t k = 0; k < noninternal.size(); k++)
		if (idx & (1u << k))
			w[noninternal[k] / 32] |= 1u << (noninternal[k] % 32);
	return w;
}

namespace {

// Probability as the reference prints it (a float).
float prob_f(const result& r, int w, unsigned b) { return (float)r.window_prob(w, b); }

float window_entropy(const result& r, int w)
{
	float entropy = 0.f;
	for (unsigned b = 0; b < r.n_bins; b++)
	{
		const float p = prob_f(r, w, b);
		if (p == 0.f)
			continue;
		entropy += -std::log2(p) * p;
	}
	return entropy;
}

std::string idx_name(const result& r, const std::vector<std::string>& names, unsigned b)
{
	auto st = noninternal_index_to_state(r.noninternal_nodes, r.state_size, b);
	return state_name(names, st.data(), r.state_size);
}

} // namespace

std::string format_probtraj_csv(const result& r, const std::vector<std::string>& names)
{
	std::ostringstream ofs;
	int max_states = 0;
	for (int w = 0; w < r.n_windows; w++)
	{
		int c = 0;
		for (unsigned b = 0; b < r.n_bins; b++)
			c += prob_f(r, w, b) != 0.f ? 1 : 0;
		max_states = std::max(max_states, c);
	}
	ofs << "Time\tTH\tErrorTH\tH\tHD=0";
	for (int i = 0; i < max_states; i++)
		ofs << "\tState\tProba\tErrorProba";
	ofs << std::endl;
	for (int w = 0; w < r.n_windows; w++)
	{
		const float th = (float)r.window_th(w);
		const float entropy = window_entropy(r, w);
		ofs << (float)w * r.time_tick << "\t";
		ofs << th << "\t" << 0.f << "\t" << entropy << "\t" << 0.f;
		for (unsigned b = 0; b < r.n_bins; b++)
		{
			const float p = prob_f(r, w, b);
			if (p == 0.f)
				continue;
			ofs << "\t" << idx_name(r, names, b) << "\t" << p << "\t" << 0.f;
		}
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
	for (unsigned b = 0; b < r.n_bins && b < r.final_cnt.size(); b++)
		if (r.final_cnt[b] != 0)
			os << (float)r.final_cnt[b] / (float)r.n_traj << " " << idx_name(r, names, b) << std::endl;
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
		os << "window (" << (float)w * r.time_tick << ", " << (float)(w + 1) * r.time_tick << "]" << std::endl;
		os << "entropy: " << window_entropy(r, w) << std::endl;
		os << "transition entropy: " << (float)r.window_th(w) << std::endl;
		for (unsigned b = 0; b < r.n_bins; b++)
		{
			const float p = prob_f(r, w, b);
			if (p == 0.f)
				continue;
			os << p << " " << idx_name(r, names, b) << std::endl;
		}
	}
	return os.str();
}

} // namespace mb
