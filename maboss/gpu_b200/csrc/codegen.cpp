// Model -> CUDA source. See codegen.h.
#include "codegen.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <set>
#include <sstream>

namespace mb {

namespace {

// Value of a printed literal as the CUDA compiler sees it: the text decides int vs
// double, and the value is the text parsed back.
struct cval
{
	bool is_double = false;
	double d = 0;
	long long i = 0;
	double as_double() const { return is_double ? d : (double)i; }
	bool truthy() const { return is_double ? d != 0 : i != 0; }
};

cval literal_cval(float v)
{
	std::string s = print_float(v);
	cval r;
	if (s.find_first_of(".eEnNiI") != std::string::npos)
	{
		r.is_double = true;
		r.d = std::strtod(s.c_str(), nullptr);
	}
	else
		r.i = std::strtoll(s.c_str(), nullptr, 10);
	return r;
}

struct not_evaluable : std::runtime_error
{
	not_evaluable() : std::runtime_error("not evaluable") {}
};

// Evaluate an emitted expression with C++ typing rules for a given node-state assignment.
// `bit(i)` returns the value of node i. Throws not_evaluable for forms whose emitted code
// would not compile (bitwise ops on doubles) or has undefined behaviour (int division by 0).
template <typename BitFn>
cval eval_c(const model_t& m, const expr& e, const std::string& current, BitFn&& bit)
{
	using K = expr::kind_t;
	switch (e.kind)
	{
		case K::literal: return literal_cval(e.value);
		case K::variable: return literal_cval(m.variables.at(e.name));
		case K::identifier:
		{
			int i = m.node_index(e.name);
			if (i < 0)
				throw model_error("unknown node name: " + e.name);
			cval r;
			r.i = bit(i) ? 1 : 0;
			return r;
		}
		case K::alias:
		{
			int i = m.node_index(current);
			return eval_c(m, m.nodes[i].get_attr(e.name.substr(1)), current, bit);
		}
		case K::paren: return eval_c(m, *e.a, current, bit);
		case K::ternary:
		{
			cval c = eval_c(m, *e.a, current, bit);
			cval x = eval_c(m, *e.b, current, bit);
			cval y = eval_c(m, *e.c, current, bit);
			cval r = c.truthy() ? x : y;
			if (x.is_double || y.is_double)
			{
				r.d = r.as_double();
				r.is_double = true;
			}
			return r;
		}
		case K::unary:
		{
			cval v = eval_c(m, *e.a, current, bit);
			cval r = v;
			if (e.op == op_t::MINUS)
			{
				r.d = -v.d;
				r.i = -v.i;
			}
			else if (e.op == op_t::NOT)
			{
				r.is_double = false;
				r.i = v.truthy() ? 0 : 1;
			}
			return r;
		}
		case K::binary:
		{
			cval a = eval_c(m, *e.a, current, bit);
			cval b = eval_c(m, *e.b, current, bit);
			cval r;
			const bool dbl = a.is_double || b.is_double;
			switch (e.op)
			{
				case op_t::PLUS:
				case op_t::MINUS:
				case op_t::STAR:
				case op_t::SLASH:
					if (dbl)
					{
						r.is_double = true;
						double x = a.as_double(), y = b.as_double();
						r.d = e.op == op_t::PLUS ? x + y : e.op == op_t::MINUS ? x - y : e.op == op_t::STAR ? x * y : x / y;
					}
					else
					{
						if (e.op == op_t::SLASH && b.i == 0)
							throw not_evaluable();
						r.i = e.op == op_t::PLUS ? a.i + b.i
							  : e.op == op_t::MINUS ? a.i - b.i
							  : e.op == op_t::STAR ? a.i * b.i
												   : a.i / b.i;
					}
					return r;
				case op_t::AND:
				case op_t::OR:
				case op_t::XOR:
					if (dbl)
						throw not_evaluable();
					r.i = e.op == op_t::AND ? (a.i & b.i) : e.op == op_t::OR ? (a.i | b.i) : (a.i ^ b.i);
					return r;
				default:
				{
					double x = a.as_double(), y = b.as_double();
					bool v = false;
					if (!dbl)
					{
						long long p = a.i, q = b.i;
						v = e.op == op_t::EQ ? p == q : e.op == op_t::NE ? p != q : e.op == op_t::LE ? p <= q
							: e.op == op_t::LT ? p < q : e.op == op_t::GE ? p >= q : p > q;
					}
					else
						v = e.op == op_t::EQ ? x == y : e.op == op_t::NE ? x != y : e.op == op_t::LE ? x <= y
							: e.op == op_t::LT ? x < y : e.op == op_t::GE ? x >= y : x > y;
					r.i = v ? 1 : 0;
					return r;
				}
			}
		}
	}
	throw not_evaluable();
}

void collect_nodes(const model_t& m, const expr& e, const std::string& current, std::set<int>& out, int depth = 0)
{
	using K = expr::kind_t;
	if (depth > 64)
		throw model_error("alias recursion too deep in node " + current);
	switch (e.kind)
	{
		case K::identifier:
		{
			int i = m.node_index(e.name);
			if (i < 0)
				throw model_error("unknown node name: " + e.name);
			out.insert(i);
			return;
		}
		case K::alias:
		{
			int i = m.node_index(current);
			collect_nodes(m, m.nodes[i].get_attr(e.name.substr(1)), current, out, depth + 1);
			return;
		}
		default:
			if (e.a)
				collect_nodes(m, *e.a, current, out, depth);
			if (e.b)
				collect_nodes(m, *e.b, current, out, depth);
			if (e.c)
				collect_nodes(m, *e.c, current, out, depth);
	}
}

// generator.cpp:57-82 (is_logic_ternary_expression). The reference evaluates the branches
// unconditionally and aborts on non-constant ones; here such nodes use the general form.
bool is_logic_ternary(const model_t& m, const expr* e, bool up, float& val)
{
	if (!e || e->kind != expr::kind_t::ternary)
		return false;
	if (e->a->kind != expr::kind_t::alias || e->a->name != "@logic")
		return false;
	if (!is_constant_expr(m, *e->b) || !is_constant_expr(m, *e->c))
		return false;
	float l = evaluate(m, *e->b), r = evaluate(m, *e->c);
	float zero = up ? r : l;
	val = up ? l : r;
	return zero == 0.f;
}

float compiled_literal(float v) { return (float)literal_cval(v).as_double(); }

std::string flit(float v)
{
	// exact float literal for engine-side constants
	char buf[64];
	std::snprintf(buf, sizeof buf, "%.9gf", v);
	std::string s = buf;
	if (s.find_first_of(".eEn") == std::string::npos)
		s.insert(s.size() - 1, ".0");
	return s;
}

std::string ident(const std::string& node_name) { return node_name; }

void emit_bit(std::ostream& os, int i) { os << "((state[" << i / 32 << "] & " << (1u << (i % 32)) << "u) != 0)"; }

template <typename T>
void emit_array(std::ostream& os, const char* type, const char* name, const std::vector<T>& v)
{
	os << "__device__ const " << type << " " << name << "[" << std::max<size_t>(1, v.size()) << "] = {";
	if (v.empty())
		os << "0";
	for (size_t i = 0; i < v.size(); i++)
		os << (i ? (i % 16 ? ", " : ",\n    ") : "") << v[i];
	os << "};" << std::endl;
}

// Tables of the incremental kernels (kernels/engine.cuh, MBG_INCREMENTAL), built by
// build_incremental_tables (the batched kernel uploads node/hdr/in1/in2 at run time):
//   node[i]    = {q_up, q_down, first dependent record, dependents | (ni_pos + 1) << 16}
//   hdr[r]     = {k | m << 16 | (ni_pos(k) + 1) << 21, q_up(k), q_down(k), truth table or offset}
//   in1[r]     = inputs 0..7 of k's logic as 16-bit node indices, in2[r] = inputs 8..15
//   self[i]    = the record of node i's own logic
// The NVRTC kernels read the same content in L1-sized pieces: mbg_inc_q (q_up, q_down) and
// mbg_inc_dep (first record, dependents | ni) of every node in 8 bytes each, and one 16-byte record
//   crec[r]    = {k | m << 16 | (ni_pos(k) + 1) << 21, truth table or offset, inputs 0-1, inputs 2-3}
// with inputs 4..11 in cext[r], read only for logics of more than 4 inputs. The truth table of k is
// inline when it has at most 5 inputs (32 patterns), else an offset into tt.
void emit_incremental_tables(std::ostream& ss, const model_layout& L)
{
	ss << std::endl << "// ---- incremental engine tables" << std::endl;
	if (!L.incremental_ok)
	{
		ss << "constexpr int mbg_inc_rate_shift = 0;" << std::endl;
		return;
	}
	const incremental_tables t = build_incremental_tables(L, L.up, L.down);
	auto u4 = [](const std::vector<unsigned>& v) {
		std::vector<std::string> out;
		for (size_t i = 0; i + 3 < v.size(); i += 4)
			out.push_back("{" + std::to_string(v[i]) + "u, " + std::to_string(v[i + 1]) + "u, " +
						  std::to_string(v[i + 2]) + "u, " + std::to_string(v[i + 3]) + "u}");
		return out;
	};
	ss << "#define MBG_INCREMENTAL 1" << std::endl;
	// the fast kernel's integer rates (else fast mode takes the dense fp32 kernel)
	if (t.ok && L.integer_rates_ok)
		ss << "#define MBG_INTEGER_RATES 1" << std::endl;
	ss << "constexpr int mbg_inc_rate_shift = " << t.rate_shift << ";" << std::endl;
	// the node records split in two 8-byte tables: (q_up, q_down) of every node alone: the flip selection scans these (8 bytes per node stay in L1)
	std::vector<unsigned> q2;
	for (size_t i = 0; i + 3 < t.node.size(); i += 4)
	{
		q2.push_back(t.node[i]);
		q2.push_back(t.node[i + 1]);
	}
	emit_array(ss, "unsigned", "mbg_inc_q", q2);
	// (first dependent record, dependents | (ni_pos + 1) << 16) of every node alone: a flip reads
	// these 8 bytes (L1-resident) instead of the 16-byte node record
	std::vector<unsigned> dep2;
	for (size_t i = 0; i + 3 < t.node.size(); i += 4)
	{
		dep2.push_back(t.node[i + 2]);
		dep2.push_back(t.node[i + 3]);
	}
	emit_array(ss, "unsigned", "mbg_inc_dep", dep2);
	// 16-byte dependent records (the node's rates come from mbg_inc_q); inputs 4-11 apart
	emit_array(ss, "uint4", "mbg_inc_crec", u4(t.crec));
	emit_array(ss, "uint4", "mbg_inc_cext", u4(t.cext));
	emit_array(ss, "unsigned", "mbg_inc_tt", t.tt);
	emit_array(ss, "int", "mbg_inc_self", t.self);
	// float rates (up, down) of every node as the generated rate functions return them (exact mode)
	std::vector<std::string> rate;
	for (int i = 0; i < L.state_size; i++)
	{
		rate.push_back(flit(L.up[i]));
		rate.push_back(flit(L.down[i]));
	}
	emit_array(ss, "float", "mbg_inc_rate", rate);
	std::vector<std::string> f_up, f_down, f_ul, f_dl;
	for (int i : L.noninternal_nodes)
	{
		const double u = L.up[i], d = L.down[i];
		f_up.push_back(flit(L.up[i]));
		f_down.push_back(flit(L.down[i]));
		f_ul.push_back(flit(u > 0 ? (float)(u * std::log2(u)) : 0.f));
		f_dl.push_back(flit(d > 0 ? (float)(d * std::log2(d)) : 0.f));
	}
	emit_array(ss, "float", "mbg_inc_ni_up", f_up);
	emit_array(ss, "float", "mbg_inc_ni_down", f_down);
	emit_array(ss, "float", "mbg_inc_ni_ul", f_ul);
	emit_array(ss, "float", "mbg_inc_ni_dl", f_dl);
	emit_array(ss, "int", "mbg_inc_ni_node", L.noninternal_nodes);
	// The fast kernels' entropy sums (sum of the unstable non-internal nodes' rates and of their
	// r log2 r, in non-internal order) straight-line: node words, bit masks and rates are constants,
	// and each state word is read once. Same operations in the same order as the loop over the
	// tables above (mbg_inc_ni_*).
	ss << "template <class V>" << std::endl;
	ss << "__device__ __forceinline__ void mbg_ni_rate_sums(const V& v, float& t, float& tl)" << std::endl;
	ss << "{" << std::endl;
	int cur_word = -1;
	for (size_t k = 0; k < L.noninternal_nodes.size(); k++)
	{
		const int i = L.noninternal_nodes[k];
		if (i / 32 != cur_word)
		{
			cur_word = i / 32;
			ss << "    {" << std::endl;
			ss << "        const uint32_t s = v.S(" << cur_word << "), u = v.U(" << cur_word << ");" << std::endl;
		}
		const unsigned bit = 1u << (i % 32);
		ss << "        if (u & " << bit << "u) { const bool on = (s & " << bit << "u) != 0u; t += on ? " << f_down[k]
		   << " : " << f_up[k] << "; tl += on ? " << f_dl[k] << " : " << f_ul[k] << "; }" << std::endl;
		const bool last_in_word = k + 1 == L.noninternal_nodes.size() || L.noninternal_nodes[k + 1] / 32 != cur_word;
		if (last_in_word)
			ss << "    }" << std::endl;
	}
	ss << "}" << std::endl;
	// the same sums with the rates of a parameter variant (batched kernels compiled for this
	// network): rate[2 i + on], rlog[2 i + on]
	ss << "template <class V>" << std::endl;
	ss << "__device__ __forceinline__ void mbg_ni_rate_sums_var(const V& v, const float* rate, const float* rlog, "
		  "float& t, float& tl)"
	   << std::endl;
	ss << "{" << std::endl;
	cur_word = -1;
	for (size_t k = 0; k < L.noninternal_nodes.size(); k++)
	{
		const int i = L.noninternal_nodes[k];
		if (i / 32 != cur_word)
		{
			cur_word = i / 32;
			ss << "    {" << std::endl;
			ss << "        const uint32_t s = v.S(" << cur_word << "), u = v.U(" << cur_word << ");" << std::endl;
		}
		const unsigned bit = 1u << (i % 32);
		ss << "        if (u & " << bit << "u) { const int e = " << 2 * i << " + ((s & " << bit
		   << "u) != 0u ? 1 : 0); t += __ldg(rate + e); tl += __ldg(rlog + e); }" << std::endl;
		const bool last_in_word = k + 1 == L.noninternal_nodes.size() || L.noninternal_nodes[k + 1] / 32 != cur_word;
		if (last_in_word)
			ss << "    }" << std::endl;
	}
	ss << "}" << std::endl;
}

// forward-mode derivative of the float evaluation (expressions.cpp evaluate) w.r.t. one variable
struct dual
{
	float v = 0, d = 0;
};

dual eval_dual(const model_t& m, const expr& e, const std::map<std::string, float>& vars, const std::string& p)
{
	using K = expr::kind_t;
	switch (e.kind)
	{
		case K::literal: return { e.value, 0.f };
		case K::variable:
		{
			auto it = vars.find(e.name);
			if (it == vars.end())
				throw model_error("unknown variable " + e.name);
			return { it->second, e.name == p ? 1.f : 0.f };
		}
		case K::paren: return eval_dual(m, *e.a, vars, p);
		case K::ternary:
		{
			const dual c = eval_dual(m, *e.a, vars, p);
			return c.v != 0.f ? eval_dual(m, *e.b, vars, p) : eval_dual(m, *e.c, vars, p);
		}
		case K::unary:
		{
			const dual a = eval_dual(m, *e.a, vars, p);
			if (e.op == op_t::MINUS)
				return { -a.v, -a.d };
			if (e.op == op_t::NOT)
				return { (float)!a.v, 0.f };
			return a;
		}
		case K::binary:
		{
			const dual a = eval_dual(m, *e.a, vars, p), b = eval_dual(m, *e.b, vars, p);
			switch (e.op)
			{
				case op_t::PLUS: return { a.v + b.v, a.d + b.d };
				case op_t::MINUS: return { a.v - b.v, a.d - b.d };
				case op_t::STAR: return { a.v * b.v, a.d * b.v + a.v * b.d };
				case op_t::SLASH: return { a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v) };
				case op_t::AND: return { (float)(a.v && b.v), 0.f };
				case op_t::OR: return { (float)(a.v || b.v), 0.f };
				case op_t::XOR: return { (float)((a.v != 0.f) != (b.v != 0.f)), 0.f };
				case op_t::EQ: return { (float)(a.v == b.v), 0.f };
				case op_t::NE: return { (float)(a.v != b.v), 0.f };
				case op_t::LE: return { (float)(a.v <= b.v), 0.f };
				case op_t::LT: return { (float)(a.v < b.v), 0.f };
				case op_t::GE: return { (float)(a.v >= b.v), 0.f };
				case op_t::GT: return { (float)(a.v > b.v), 0.f };
				default: throw model_error("Unknown binary operator");
			}
		}
		default: throw model_error("node or alias in a rate constant");
	}
}

} // namespace

int model_layout::windows() const
{
	// window_average_small.cpp:305: std::ceil(max_time / window_size) with float operands
	float q = max_time / time_tick;
	return (int)std::ceil(q);
}

model_layout analyze_model(const model_t& m)
{
	model_layout L;
	const int N = (int)m.nodes.size();
	L.state_size = N;
	L.state_words = (N + 31) / 32;
	L.discrete_time = m.constant("discrete_time") != 0;
	L.max_time = m.constant("max_time");
	L.time_tick = m.constant("time_tick");
	L.sample_count = (int)m.constant("sample_count");
	L.seed = (unsigned long long)m.constant("seed_pseudorandom");
	std::set<int> ni_words;
	for (int i = 0; i < N; i++)
	{
		L.names.push_back(m.nodes[i].name);
		L.istate.push_back(m.nodes[i].istate);
		if (!m.is_internal(i))
		{
			L.noninternal_nodes.push_back(i);
			ni_words.insert(i / 32);
		}
	}
	L.noninternal_words = (int)ni_words.size();

	L.fast_path.assign(N, 0);
	L.up.assign(N, 0.f);
	L.down.assign(N, 0.f);
	L.all_fast_path = N > 0;
	L.rates_nonnegative = true;
	for (int i = 0; i < N; i++)
	{
		const node_t& node = m.nodes[i];
		float u = 0, d = 0;
		bool fp = is_logic_ternary(m, node.find_attr("rate_up"), true, u)
				  && is_logic_ternary(m, node.find_attr("rate_down"), false, d) && node.find_attr("logic");
		L.fast_path[i] = fp;
		if (fp)
		{
			L.up[i] = compiled_literal(u);
			L.down[i] = compiled_literal(d);
			if (!(L.up[i] >= 0.f) || !(L.down[i] >= 0.f))
				L.rates_nonnegative = false;
		}
		else
		{
			L.all_fast_path = false;
			L.rates_nonnegative = false;
		}
	}

	// incremental tables (fast-path models with small logic fan-in only)
	// the incremental kernels keep 12 bytes of shared memory per state word and thread: at most 600
	// words (19200 nodes) fit a block of 32 threads; larger models take the dense kernels
	// (the incremental exact kernel's binary search over word-end rate sums needs rates >= 0)
	L.incremental_ok = L.all_fast_path && L.rates_nonnegative && N <= 65535 && L.state_words <= 600;
	constexpr int max_inputs = 12;
	if (L.incremental_ok)
	{
		std::vector<std::set<int>> inputs(N);
		for (int i = 0; i < N && L.incremental_ok; i++)
		{
			collect_nodes(m, m.nodes[i].get_attr("logic"), m.nodes[i].name, inputs[i]);
			if ((int)inputs[i].size() > max_inputs)
				L.incremental_ok = false;
		}
		if (L.incremental_ok)
		{
			L.in_ptr.push_back(0);
			L.tt_ptr.push_back(0);
			std::vector<std::vector<int>> deps(N);
			for (int i = 0; i < N; i++)
				deps[i].push_back(i);
			for (int i = 0; i < N && L.incremental_ok; i++)
			{
				std::vector<int> in(inputs[i].begin(), inputs[i].end());
				for (int j : in)
				{
					L.in_idx.push_back(j);
					if (j != i)
						deps[j].push_back(i);
				}
				L.in_ptr.push_back((int)L.in_idx.size());
				const int mi = (int)in.size();
				const int patterns = 1 << mi;
				const int words = (patterns + 31) / 32;
				std::vector<unsigned> tt(words, 0u);
				try
				{
					for (int p = 0; p < patterns; p++)
					{
						auto bit = [&](int node) {
							auto it = std::find(in.begin(), in.end(), node);
							return ((p >> (it - in.begin())) & 1) != 0;
						};
						cval v = eval_c(m, m.nodes[i].get_attr("logic"), m.nodes[i].name, bit);
						if (v.truthy())
							tt[p / 32] |= 1u << (p % 32);
					}
				}
				catch (const not_evaluable&)
				{
					L.incremental_ok = false;
				}
				L.tt_words.insert(L.tt_words.end(), tt.begin(), tt.end());
				L.tt_ptr.push_back((int)L.tt_words.size());
			}
			L.dep_ptr.push_back(0);
			for (int j = 0; j < N; j++)
			{
				std::sort(deps[j].begin(), deps[j].end());
				deps[j].erase(std::unique(deps[j].begin(), deps[j].end()), deps[j].end());
				L.dep_idx.insert(L.dep_idx.end(), deps[j].begin(), deps[j].end());
				L.dep_ptr.push_back((int)L.dep_idx.size());
			}
		}
		if (L.incremental_ok)
		{
			L.rate_shift = integer_rate_shift(L.up, L.down, L.state_words);
			L.q_up.resize(N);
			L.q_down.resize(N);
			L.integer_rates_ok = true;
			for (int i = 0; i < N; i++)
			{
				for (int which = 0; which < 2; which++)
				{
					const double r = which ? L.down[i] : L.up[i];
					const double q = std::nearbyint(std::max(0.0, r) * std::ldexp(1.0, L.rate_shift));
					// positive rates need enough resolution (relative rounding error at most 2^-21)
					if (!(r >= 0.0) || (r > 0 && q < integer_rate_min_units))
						L.integer_rates_ok = false;
					(which ? L.q_down[i] : L.q_up[i]) = (unsigned)std::min(q, 4294967295.0);
				}
			}
		}
		if (!L.incremental_ok)
		{
			L.q_up.clear();
			L.q_down.clear();
			L.in_ptr.clear();
			L.in_idx.clear();
			L.tt_ptr.clear();
			L.tt_words.clear();
			L.dep_ptr.clear();
			L.dep_idx.clear();
		}
	}
	return L;
}

rate_set fast_rates(const model_t& m, const std::map<std::string, float>& variables,
					const std::vector<std::string>& params)
{
	const int N = (int)m.nodes.size();
	rate_set r;
	r.up.assign(N, 0.f);
	r.down.assign(N, 0.f);
	r.grad_ptr.assign(1, 0);
	model_t mm = m;
	mm.variables = variables;
	for (int i = 0; i < N; i++)
	{
		const node_t& node = m.nodes[i];
		float u = 0, d = 0;
		if (!(is_logic_ternary(mm, node.find_attr("rate_up"), true, u) &&
			  is_logic_ternary(mm, node.find_attr("rate_down"), false, d) && node.find_attr("logic")))
			throw model_error("node " + node.name + " is not of the form rate_up = @logic ? U : 0; rate_down = @logic ? 0 : D");
		const expr& ue = *node.find_attr("rate_up")->b;	  // middle of rate_up
		const expr& de = *node.find_attr("rate_down")->c; // right of rate_down
		for (int dir = 0; dir < 2; dir++)
		{
			const expr& e = dir ? de : ue;
			const dual v = eval_dual(mm, e, variables, "");
			(dir ? r.down[i] : r.up[i]) = v.v;
			for (size_t p = 0; p < params.size(); p++)
			{
				const dual g = eval_dual(mm, e, variables, params[p]);
				if (g.d != 0.f)
				{
					r.grad_p.push_back((int)p);
					r.grad_d.push_back(g.d);
				}
			}
			r.grad_ptr.push_back((int)r.grad_p.size());
		}
	}
	return r;
}

int integer_rate_shift(const std::vector<float>& up, const std::vector<float>& down, int state_words)
{
	const int N = (int)up.size();
	double worst = 0;
	for (int w = 0; w < state_words; w++)
	{
		double sw = 0;
		for (int i = 32 * w; i < std::min(N, 32 * w + 32); i++)
			sw += std::max(std::max((double)up[i], (double)down[i]), 0.0);
		worst = std::max(worst, sw);
	}
	int shift = 31;
	while (shift > 0 && worst * std::ldexp(1.0, shift) >= 4294967296.0)
		shift--;
	return shift;
}

incremental_tables build_incremental_tables(const model_layout& L, const std::vector<float>& up,
											const std::vector<float>& down)
{
	incremental_tables t;
	const int N = L.state_size;
	const int shift = integer_rate_shift(up, down, L.state_words);
	t.rate_shift = shift;
	t.ok = true;
	std::vector<unsigned> qu(N), qd(N);
	for (int i = 0; i < N; i++)
	{
		for (int which = 0; which < 2; which++)
		{
			const double r = which ? down[i] : up[i];
			if (!(r >= 0.0))
				t.ok = false;
			const double q = std::nearbyint(std::max(0.0, r) * std::ldexp(1.0, shift));
			if (r > 0 && q < integer_rate_min_units)
				t.ok = false;
			(which ? qd[i] : qu[i]) = (unsigned)std::min(q, 4294967295.0);
		}
		t.q.push_back(qu[i]);
		t.q.push_back(qd[i]);
	}
	std::vector<int> ni_pos(N, -1);
	for (size_t k = 0; k < L.noninternal_nodes.size(); k++)
		ni_pos[L.noninternal_nodes[k]] = (int)k;
	t.self.assign(N, -1);
	auto push4 = [](std::vector<unsigned>& v, unsigned a, unsigned b, unsigned c, unsigned d) {
		v.push_back(a);
		v.push_back(b);
		v.push_back(c);
		v.push_back(d);
	};
	for (int j = 0; j < N; j++)
	{
		const int d0 = L.dep_ptr[j], d1 = L.dep_ptr[j + 1];
		push4(t.node, qu[j], qd[j], (unsigned)d0, (unsigned)(d1 - d0) | ((unsigned)(ni_pos[j] + 1) << 16));
		for (int d = d0; d < d1; d++)
		{
			const int k = L.dep_idx[d];
			if (k == j)
				t.self[j] = d;
			const int a0 = L.in_ptr[k], m = L.in_ptr[k + 1] - a0;
			const int t0 = L.tt_ptr[k], nt = L.tt_ptr[k + 1] - t0;
			unsigned ttw;
			if (m <= 5)
				ttw = L.tt_words[t0];
			else
			{
				ttw = (unsigned)t.tt.size();
				t.tt.insert(t.tt.end(), L.tt_words.begin() + t0, L.tt_words.begin() + t0 + nt);
			}
			push4(t.hdr, (unsigned)k | ((unsigned)m << 16) | ((unsigned)(ni_pos[k] + 1) << 21), qu[k], qd[k], ttw);
			unsigned in[16] = { 0 };
			for (int x = 0; x < m; x++)
				in[x] = (unsigned)L.in_idx[a0 + x];
			push4(t.in1, in[0] | in[1] << 16, in[2] | in[3] << 16, in[4] | in[5] << 16, in[6] | in[7] << 16);
			push4(t.in2, in[8] | in[9] << 16, in[10] | in[11] << 16, in[12] | in[13] << 16, in[14] | in[15] << 16);
			push4(t.crec, (unsigned)k | ((unsigned)m << 16) | ((unsigned)(ni_pos[k] + 1) << 21), ttw,
				  in[0] | in[1] << 16, in[2] | in[3] << 16);
			push4(t.cext, in[4] | in[5] << 16, in[6] | in[7] << 16, in[8] | in[9] << 16, in[10] | in[11] << 16);
		}
	}
	if (t.tt.empty())
		t.tt.push_back(0);
	return t;
}

std::string generate_code(const model_t& m)
{
	const model_layout L = analyze_model(m);
	const int N = L.state_size;
	std::ostringstream ss;

	// ---- reference-form prologue (generator.cpp:17-29)
	ss << "using uint8_t = unsigned char;" << std::endl;
	ss << "using uint32_t = unsigned int;" << std::endl << std::endl;
	ss << "constexpr int state_size = " << N << ";" << std::endl;
	ss << "constexpr int state_words = " << L.state_words << ";" << std::endl;
	ss << "constexpr bool discrete_time = " << (L.discrete_time ? 1 : 0) << ";" << std::endl;
	ss << "constexpr float max_time = " << print_float(m.constant("max_time")) << ";" << std::endl;
	ss << "constexpr float time_tick = " << print_float(m.constant("time_tick")) << ";" << std::endl;
	ss << "using state_word_t = uint32_t;" << std::endl << std::endl;

	// ---- per-node rate functions (generator.cpp:84-122); internal linkage so that kernels which
	// do not use them do not pay for their compilation
	ss << "namespace {" << std::endl << std::endl;
	for (int i = 0; i < N; i++)
	{
		const node_t& node = m.nodes[i];
		ss << "__device__ float " << ident(node.name) << "_rate(const state_word_t* __restrict__ state) " << std::endl;
		ss << "{" << std::endl;
		if (L.fast_path[i])
		{
			float up_val = 0, down_val = 0;
			is_logic_ternary(m, node.find_attr("rate_up"), true, up_val);
			is_logic_ternary(m, node.find_attr("rate_down"), false, down_val);
			ss << "    const bool is_up = ";
			emit_bit(ss, i);
			ss << ";" << std::endl;
			ss << "    const bool logic = ";
			emit_code(m, node.get_attr("logic"), node.name, ss);
			ss << ";" << std::endl;
			if (up_val == down_val)
				ss << "    return is_up == logic ? 0 : " << print_float(up_val) << ";" << std::endl;
			else
				ss << "    return is_up == logic ? 0 : (is_up ? " << print_float(down_val) << " : "
				   << print_float(up_val) << ");" << std::endl;
		}
		else
		{
			ss << "    return ";
			emit_bit(ss, i);
			ss << " ?" << std::endl;
			ss << "          (";
			emit_code(m, node.get_attr("rate_down"), node.name, ss);
			ss << ")" << std::endl;
			ss << "        : (";
			emit_code(m, node.get_attr("rate_up"), node.name, ss);
			ss << ");" << std::endl;
		}
		ss << "}" << std::endl << std::endl;
	}

	// ---- compute_transition_rates (generator.cpp:124-144)
	ss << "__device__ float compute_transition_rates(float* __restrict__ transition_rates, const state_word_t* "
		  "__restrict__ state)"
	   << std::endl;
	ss << "{" << std::endl << "    float sum = 0;" << std::endl << "    float tmp;" << std::endl << std::endl;
	for (int i = 0; i < N; i++)
	{
		ss << "    tmp = " << ident(m.nodes[i].name) << "_rate(state);" << std::endl;
		ss << "    transition_rates[" << i << "] = tmp;" << std::endl;
		ss << "    sum += tmp;" << std::endl << std::endl;
	}
	ss << "    return sum;" << std::endl << "}" << std::endl << std::endl;

	// ---- compute_transition_entropy (generator.cpp:146-175)
	ss << "__device__ float compute_transition_entropy(const float* __restrict__ transition_rates)" << std::endl;
	ss << "{" << std::endl;
	ss << "    float entropy = 0.f;" << std::endl;
	ss << "    float non_internal_total_rate = 0.f;" << std::endl;
	ss << "    float tmp_prob;" << std::endl << std::endl;
	for (int i : L.noninternal_nodes)
		ss << "    non_internal_total_rate += transition_rates[" << i << "];" << std::endl;
	ss << "    if (non_internal_total_rate == 0.f) return 0.f;" << std::endl << std::endl;
	for (int i : L.noninternal_nodes)
	{
		ss << "    tmp_prob = transition_rates[" << i << "] / non_internal_total_rate;" << std::endl;
		ss << "    entropy -= (tmp_prob == 0.f) ? 0.f : log2f(tmp_prob) * tmp_prob;" << std::endl;
	}
	ss << "    return entropy;" << std::endl << "}" << std::endl << std::endl;
	ss << "} // namespace" << std::endl << std::endl;

	// ---- get_non_internal_index (generator.cpp:207-235); the reference stops at 20 non-internal
	// nodes (main.cpp:142-146), this engine goes on to 112 with a 128-bit index and sparse window bins
	if (L.noninternal_nodes.size() > 112)
		throw model_error("more than 112 non-internal nodes (" + std::to_string(L.noninternal_nodes.size()) + ")");
	if (L.noninternal_nodes.size() > 20)
	{
		ss << "#define MBG_WIDE_INDEX 1" << std::endl;
		ss << "__device__ unsigned __int128 get_non_internal_index(const state_word_t* __restrict__ state)"
		   << std::endl;
		ss << "{" << std::endl << "    return" << std::endl << "\t\t\t";
		int k = 0;
		const int kc = (int)L.noninternal_nodes.size();
		for (int i : L.noninternal_nodes)
		{
			ss << "((unsigned __int128)((state[" << i / 32 << "] >> " << i % 32 << ") & 1u) << " << k++ << ")";
			if (k != kc)
				ss << " | ";
		}
		ss << ";" << std::endl << "}" << std::endl << std::endl;
	}
	else
	{
	ss << "__device__ uint32_t get_non_internal_index(const state_word_t* __restrict__ state)" << std::endl;
	ss << "{" << std::endl;
	if (L.noninternal_nodes.empty() || L.noninternal_nodes.size() > 32)
		ss << "    return 0u;" << std::endl;
	else
	{
		ss << "    return" << std::endl << "\t\t\t";
		int k = 0;
		const int kc = (int)L.noninternal_nodes.size();
		for (int i : L.noninternal_nodes)
		{
			ss << "((state[" << i / 32 << "] & " << (1u << (i % 32)) << "u)";
			int shift = (i % 32) - k++;
			if (shift > 0)
				ss << " >> " << shift;
			else if (shift < 0)
				ss << " << " << -shift;
			ss << ")";
			if (k != kc)
				ss << " | ";
		}
		ss << ";" << std::endl;
	}
	ss << "}" << std::endl << std::endl;
	}

	// ---- engine helpers (not part of the reference's generated text)
	ss << "// ---- B200 engine helpers" << std::endl;
	ss << "constexpr int mbg_noninternal_count = " << L.noninternal_nodes.size() << ";" << std::endl;
	ss << "constexpr bool mbg_rates_nonnegative = " << (L.rates_nonnegative ? "true" : "false") << ";" << std::endl;
	ss << "constexpr bool mbg_all_fast_path = " << (L.all_fast_path ? "true" : "false") << ";" << std::endl;
	ss << "constexpr bool mbg_incremental = " << (L.incremental_ok ? "true" : "false") << ";" << std::endl
	   << std::endl;

	// total rate in node order: the same fp32 sum sequence as compute_transition_rates
	ss << "__device__ __forceinline__ float mbg_total_rate(const state_word_t* __restrict__ state)" << std::endl;
	ss << "{" << std::endl << "    float sum = 0;" << std::endl;
	for (int i = 0; i < N; i++)
		ss << "    sum += " << ident(m.nodes[i].name) << "_rate(state);" << std::endl;
	ss << "    return sum;" << std::endl << "}" << std::endl << std::endl;

	// flip selection: idx = #{i : prefix_i < r} (simulation.cu:9-21). With non-negative rates
	// the prefix sums are monotone, so the count equals the first index reaching r.
	ss << "__device__ __forceinline__ int mbg_select_flip(const state_word_t* __restrict__ state, float r)"
	   << std::endl;
	ss << "{" << std::endl << "    float sum = 0;" << std::endl;
	if (L.rates_nonnegative)
	{
		for (int i = 0; i < N; i++)
			ss << "    sum += " << ident(m.nodes[i].name) << "_rate(state); if (!(sum < r)) return " << i << ";"
			   << std::endl;
		ss << "    return " << (N - 1) << ";" << std::endl;
	}
	else
	{
		ss << "    int idx = 0;" << std::endl;
		for (int i = 0; i < N; i++)
			ss << "    sum += " << ident(m.nodes[i].name) << "_rate(state); idx += (sum < r) ? 1 : 0;" << std::endl;
		ss << "    return idx < " << N << " ? idx : " << (N - 1) << ";" << std::endl;
	}
	ss << "}" << std::endl << std::endl;

	// transition entropy with the same arithmetic as compute_transition_entropy
	ss << "__device__ __forceinline__ float mbg_entropy(const state_word_t* __restrict__ state)" << std::endl;
	ss << "{" << std::endl;
	for (int i : L.noninternal_nodes)
		ss << "    const float r" << i << " = " << ident(m.nodes[i].name) << "_rate(state);" << std::endl;
	ss << "    float entropy = 0.f;" << std::endl;
	ss << "    float non_internal_total_rate = 0.f;" << std::endl;
	ss << "    float tmp_prob;" << std::endl;
	for (int i : L.noninternal_nodes)
		ss << "    non_internal_total_rate += r" << i << ";" << std::endl;
	ss << "    if (non_internal_total_rate == 0.f) return 0.f;" << std::endl;
	for (int i : L.noninternal_nodes)
	{
		ss << "    tmp_prob = r" << i << " / non_internal_total_rate;" << std::endl;
		ss << "    entropy -= (tmp_prob == 0.f) ? 0.f : log2f(tmp_prob) * tmp_prob;" << std::endl;
	}
	ss << "    (void)tmp_prob;" << std::endl;
	ss << "    return entropy;" << std::endl << "}" << std::endl << std::endl;

	// fast-mode entropy: h = log2(S) - (sum r log2 r) / S with r log2 r folded into constants
	ss << "__device__ __forceinline__ float mbg_entropy_fast(const state_word_t* __restrict__ state)" << std::endl;
	ss << "{" << std::endl << "    float t = 0.f, tl = 0.f;" << std::endl;
	for (int i : L.noninternal_nodes)
	{
		if (L.fast_path[i])
		{
			const double u = L.up[i], d = L.down[i];
			const float ul = u > 0 ? (float)(u * std::log2(u)) : 0.f;
			const float dl = d > 0 ? (float)(d * std::log2(d)) : 0.f;
			ss << "    { const bool up = ";
			emit_bit(ss, i);
			ss << "; const bool lg = ";
			emit_code(m, m.nodes[i].get_attr("logic"), m.nodes[i].name, ss);
			ss << "; if (up != lg) { t += up ? " << flit(L.down[i]) << " : " << flit(L.up[i]) << "; tl += up ? "
			   << flit(dl) << " : " << flit(ul) << "; } }" << std::endl;
		}
		else
		{
			ss << "    { const float r = " << ident(m.nodes[i].name)
			   << "_rate(state); t += r; tl += (r > 0.f) ? r * log2f(r) : 0.f; }" << std::endl;
		}
	}
	ss << "    if (!(t > 0.f)) return 0.f;" << std::endl;
	ss << "    const float h = log2f(t) - tl / t;" << std::endl;
	ss << "    return h > 0.f ? h : 0.f;" << std::endl << "}" << std::endl;

	emit_incremental_tables(ss, L);
	return ss.str();
}

} // namespace mb
