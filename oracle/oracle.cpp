// CPU ORACLE -- test infrastructure only. Not part of the product, never called by it.
//
// A plain C++/OpenMP restatement of the reference MaBoSS.GPU trajectory path, used to check the
// CUDA engine (tests/, __graft_entry__.smoke) and as the CPU baseline of bench.py. It has its own
// model parser and its own evaluator of the generated-code semantics, written independently of
// the engine's front-end. Every function cites the reference file:line it restates (paths
// relative to the reference project).
//
// Parity pins: the oracle's window probabilities, final states and fixed points are checked
// against the reference's golden outputs test/{cellcycle,sizek,metastasis,Montagud2022_Prostate_Cancer}.res
// (statistically, 4 sigma; tests/test_oracle_golden.py).
//
// Random numbers: curand's XORWOW generator through its header-only device API compiled for
// the host (curand_init(seed, trajectory, 0), curand_uniform), so the streams are the ones the
// GPU draws. Waiting times use the host logf; the device logf may differ in the last ulp, so
// continuous-time times can differ by a few ulps from the GPU while flips, steps and states agree.
//
// Modes: 0 = exact (reference semantics incl. the 100-slot epoch boundary), 1 = fast (Philox
// streams, no epoch boundary, entropy via sum r*log2 r), mirroring the engine's two fused modes.
//
// Gradient: gradient_integer states the score-function gradient that the engine's batched gradient
// kernel computes (the reference has no gradient) directly along the fast-mode trajectories; it is
// pinned against exact derivatives of small chains solved in closed form (tests/test_oracle_gradient.py).
#include <curand_kernel.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ------------------------------------------------------------------ expressions

enum class K
{
	num,
	node,
	var,
	alias,
	un,
	bin,
	tern,
	paren
};

struct E
{
	K k = K::num;
	float v = 0;
	std::string s;
	char op = 0; // '+','-','*','/','&','|','^','!','=' (==),'n' (!=),'<','l' (<=),'>','g' (>=)
	std::shared_ptr<E> a, b, c;
};
using P = std::shared_ptr<E>;

struct node_def
{
	std::string name;
	std::vector<std::pair<std::string, P>> attrs;
	float istate = 0.5f;
	P attr(const std::string& n) const
	{
		for (auto& a : attrs)
			if (a.first == n)
				return a.second; // first attribute wins (parse_types.cpp:6-13)
		return nullptr;
	}
};

struct model
{
	std::map<std::string, float> vars, consts;
	std::vector<node_def> nodes;
	int index(const std::string& n) const
	{
		for (size_t i = 0; i < nodes.size(); i++)
			if (nodes[i].name == n)
				return (int)i;
		return -1;
	}
};

// float evaluation (expressions.cpp evaluate methods)
float feval(const model& m, const E& e)
{
	switch (e.k)
	{
		case K::num: return e.v;
		case K::var:
		{
			auto it = m.vars.find(e.s);
			if (it == m.vars.end())
				throw std::runtime_error("unknown variable " + e.s);
			return it->second;
		}
		case K::paren: return feval(m, *e.a);
		case K::tern: return feval(m, *e.a) ? feval(m, *e.b) : feval(m, *e.c);
		case K::un:
			if (e.op == '-')
				return -feval(m, *e.a);
			if (e.op == '!')
				return !feval(m, *e.a);
			return feval(m, *e.a);
		case K::bin:
		{
			float x = feval(m, *e.a);
			switch (e.op)
			{
				case '&': return x && feval(m, *e.b);
				case '|': return x || feval(m, *e.b);
				default: break;
			}
			float y = feval(m, *e.b);
			switch (e.op)
			{
				case '+': return x + y;
				case '-': return x - y;
				case '*': return x * y;
				case '/': return x / y;
				case '^': return (x != 0) != (y != 0);
				case '=': return x == y;
				case 'n': return x != y;
				case '<': return x < y;
				case 'l': return x <= y;
				case '>': return x > y;
				case 'g': return x >= y;
			}
			throw std::runtime_error("bad operator");
		}
		default: throw std::runtime_error("node or alias in a constant expression");
	}
}

bool is_const(const model& m, const E& e)
{
	if (e.k == K::node || e.k == K::alias)
		return false;
	if (e.k == K::var)
		return m.vars.count(e.s) != 0;
	return (!e.a || is_const(m, *e.a)) && (!e.b || is_const(m, *e.b)) && (!e.c || is_const(m, *e.c));
}

// ---- C semantics of the generated CUDA code (generator.cpp + expressions.cpp generate_code):
// a literal or $variable is printed with 6 significant digits; the text is an int literal unless
// it has '.', 'e', "inf" or "nan"; identifiers become bool, & | ^ ! comparisons give int.
struct tv
{
	bool dbl = false;
	double d = 0;
	long long i = 0;
	double get() const { return dbl ? d : (double)i; }
	bool truth() const { return dbl ? d != 0 : i != 0; }
};

tv printed(float v)
{
	char buf[64];
	std::snprintf(buf, sizeof buf, "%g", (double)v);
	tv r;
	if (std::strpbrk(buf, ".eEnNiI"))
	{
		r.dbl = true;
		r.d = std::strtod(buf, nullptr);
	}
	else
		r.i = std::strtoll(buf, nullptr, 10);
	return r;
}

// ------------------------------------------------------------------ parser (scanner.ll, parser.yy)

struct tok
{
	char t = 0; // 'i' ident, 'v' $var, 'a' @alias, 'f' float, 'd' int, 'E' end, else punctuation code
	std::string s;
	double num = 0;
	int line = 1;
};

struct lex
{
	std::string src;
	size_t p = 0;
	int line = 1;
	tok next()
	{
		for (;;)
		{
			while (p < src.size() && std::strchr(" \t\r\n", src[p]))
				line += src[p++] == '\n';
			if (p + 1 < src.size() && src[p] == '/' && src[p + 1] == '/')
			{
				while (p < src.size() && src[p] != '\n')
					p++;
				continue;
			}
			break;
		}
		tok k;
		k.line = line;
		if (p >= src.size())
		{
			k.t = 'E';
			return k;
		}
		char c = src[p];
		auto alpha = [](char x) { return std::isalpha((unsigned char)x) != 0; };
		auto digit = [](char x) { return std::isdigit((unsigned char)x) != 0; };
		if (digit(c) || (c == '.' && p + 1 < src.size() && digit(src[p + 1])))
		{
			size_t q = p;
			bool f = false;
			while (q < src.size() && digit(src[q]))
				q++;
			if (q < src.size() && src[q] == '.')
			{
				f = true;
				q++;
				while (q < src.size() && digit(src[q]))
					q++;
			}
			if (q < src.size() && (src[q] == 'e' || src[q] == 'E'))
			{
				size_t r = q + 1;
				if (r < src.size() && (src[r] == '+' || src[r] == '-'))
					r++;
				if (r < src.size() && digit(src[r]))
				{
					while (r < src.size() && digit(src[r]))
						r++;
					q = r;
					f = true;
				}
			}
			k.s = src.substr(p, q - p);
			k.t = f ? 'f' : 'd';
			k.num = f ? (double)(float)std::strtod(k.s.c_str(), nullptr) : (double)std::strtol(k.s.c_str(), nullptr, 10);
			p = q;
			return k;
		}
		if (alpha(c) || ((c == '$' || c == '@') && p + 1 < src.size() && alpha(src[p + 1])))
		{
			size_t q = p + 1;
			while (q < src.size() && (alpha(src[q]) || digit(src[q]) || src[q] == '_'))
				q++;
			k.s = src.substr(p, q - p);
			p = q;
			std::string low = k.s;
			for (auto& ch : low)
				ch = (char)std::tolower((unsigned char)ch);
			k.t = c == '$' ? 'v' : c == '@' ? 'a' : 'i';
			if (k.t == 'i')
			{
				if (low == "and")
					k.t = '&';
				else if (low == "or")
					k.t = '|';
				else if (low == "xor")
					k.t = '^';
				else if (low == "not")
					k.t = '!';
				else if (low == "true" || low == "false")
				{
					k.t = 'd';
					k.num = low == "true";
				}
			}
			return k;
		}
		auto two = [&](const char* o) { return p + 1 < src.size() && src[p] == o[0] && src[p + 1] == o[1]; };
		if (two("&&") || two("||"))
		{
			k.t = src[p];
			p += 2;
			return k;
		}
		if (two("=="))
			k.t = '=';
		else if (two("!="))
			k.t = 'n';
		else if (two("<="))
			k.t = 'l';
		else if (two(">="))
			k.t = 'g';
		if (k.t)
		{
			p += 2;
			return k;
		}
		if (std::strchr("-+*/()=?:&|^!<>{}.;[],", c))
		{
			k.t = c == '=' ? 'A' : c; // single '=' is assignment
			p++;
			return k;
		}
		throw std::runtime_error("line " + std::to_string(line) + ": invalid character " + std::string(1, c));
	}
};

struct parser
{
	lex L;
	tok cur;
	model& m;
	parser(const std::string& s, model& mm) : m(mm)
	{
		L.src = s;
		cur = L.next();
	}
	[[noreturn]] void err(const std::string& what)
	{
		throw std::runtime_error("line " + std::to_string(cur.line) + ": " + what);
	}
	tok take(char t)
	{
		if (cur.t != t)
			err(std::string("expected '") + t + "'");
		tok k = cur;
		cur = L.next();
		return k;
	}
	static int prec(char t)
	{
		switch (t)
		{
			case '^': return 1;
			case '|': return 2;
			case '&': return 3;
			case '=':
			case 'n': return 4;
			case '<':
			case 'l':
			case '>':
			case 'g': return 5;
			case '+':
			case '-': return 6;
			case '*':
			case '/': return 7;
		}
		return 0;
	}
	P mk(K k)
	{
		auto e = std::make_shared<E>();
		e->k = k;
		return e;
	}
	P atom()
	{
		tok t = cur;
		if (t.t == '-' || t.t == '+' || t.t == '!')
		{
			cur = L.next();
			P e = mk(K::un);
			e->op = t.t;
			e->a = atom();
			return e;
		}
		cur = L.next();
		P e;
		switch (t.t)
		{
			case 'f':
			case 'd':
				e = mk(K::num);
				e->v = (float)t.num;
				return e;
			case 'i': e = mk(K::node); break;
			case 'v': e = mk(K::var); break;
			case 'a': e = mk(K::alias); break;
			case '(':
				e = mk(K::paren);
				e->a = expr();
				take(')');
				return e;
			default: err("unexpected token in expression");
		}
		e->s = t.s;
		return e;
	}
	P binary(int minp)
	{
		P l = atom();
		for (;;)
		{
			int p = prec(cur.t);
			if (!p || p < minp)
				return l;
			char op = cur.t;
			cur = L.next();
			P r = binary(p + 1);
			P e = mk(K::bin);
			e->op = op;
			e->a = l;
			e->b = r;
			l = e;
		}
	}
	P expr()
	{
		P c = binary(1);
		if (cur.t != '?')
			return c;
		cur = L.next();
		P e = mk(K::tern);
		e->a = c;
		e->b = expr();
		take(':');
		e->c = expr();
		return e;
	}
	void bnd()
	{
		while (cur.t != 'E')
		{
			tok kw = take('i');
			std::string low = kw.s;
			for (auto& ch : low)
				ch = (char)std::tolower((unsigned char)ch);
			if (low != "node")
				err("expected 'node'");
			node_def n;
			n.name = take('i').s;
			take('{');
			do
			{
				std::string an = take('i').s;
				take('A');
				P e = expr();
				take(';');
				n.attrs.emplace_back(an, e);
			} while (cur.t == 'i');
			take('}');
			if (m.index(n.name) >= 0)
				err("duplicate node " + n.name);
			if (!n.attr("rate_up") || !n.attr("rate_down"))
				err("node " + n.name + " lacks rate_up/rate_down");
			m.nodes.push_back(n);
		}
	}
	void cfg()
	{
		while (cur.t != 'E')
		{
			if (cur.t == 'v')
			{
				std::string n = take('v').s;
				take('A');
				P e = expr();
				take(';');
				m.vars[n] = feval(m, *e);
			}
			else if (cur.t == 'i')
			{
				std::string n = take('i').s;
				if (cur.t == '.')
				{
					take('.');
					std::string a = take('i').s;
					take('A');
					P e = expr();
					take(';');
					int i = m.index(n);
					if (i < 0)
						err("unknown node " + n);
					if (a == "istate")
						m.nodes[i].istate = feval(m, *e);
					else
						m.nodes[i].attrs.emplace_back(a, e);
				}
				else
				{
					take('A');
					P e = expr();
					take(';');
					m.consts[n] = feval(m, *e);
				}
			}
			else if (cur.t == '[')
			{
				take('[');
				std::string n = take('i').s;
				take(']');
				take('.');
				if (take('i').s != "istate")
					err("expected istate");
				take('A');
				P l = expr();
				take('[');
				int il = (int)take('d').num;
				take(']');
				take(',');
				P r = expr();
				take('[');
				int ir = (int)take('d').num;
				take(']');
				take(';');
				if (!((il == 0 && ir == 1) || (il == 1 && ir == 0)))
					err("numbers in [] must be 0 and 1");
				int i = m.index(n);
				if (i < 0)
					err("unknown node " + n);
				float a = feval(m, *l), b = feval(m, *r);
				m.nodes[i].istate = il == 1 ? a / (a + b) : b / (a + b);
			}
			else
				err("unexpected token");
		}
	}
};

// ------------------------------------------------------------------ compiled model

// Flattened expression with identifiers resolved to node indices, $variables and literals
// resolved to their printed C literal (int or double), and @aliases inlined.
struct flat
{
	struct op_t
	{
		K k;
		char op;
		int node;
		tv lit;
		int a, b, c;
	};
	std::vector<op_t> ops;
	int root = -1;

	int add(const model& m, const E& e, int self, int depth = 0)
	{
		if (depth > 64)
			throw std::runtime_error("alias recursion");
		op_t o{ e.k, e.op, -1, tv{}, -1, -1, -1 };
		switch (e.k)
		{
			case K::num: o.lit = printed(e.v); break;
			case K::var:
				o.k = K::num;
				o.lit = printed(m.vars.at(e.s));
				break;
			case K::node:
				o.node = m.index(e.s);
				if (o.node < 0)
					throw std::runtime_error("unknown node " + e.s);
				break;
			case K::alias:
			{
				P a = m.nodes[self].attr(e.s.substr(1));
				if (!a)
					throw std::runtime_error("missing attribute " + e.s);
				return add(m, *a, self, depth + 1);
			}
			case K::paren: return add(m, *e.a, self, depth);
			default:
				o.a = e.a ? add(m, *e.a, self, depth) : -1;
				o.b = e.b ? add(m, *e.b, self, depth) : -1;
				o.c = e.c ? add(m, *e.c, self, depth) : -1;
		}
		ops.push_back(o);
		return (int)ops.size() - 1;
	}

	tv eval(int i, const uint32_t* s) const
	{
		const op_t& o = ops[i];
		switch (o.k)
		{
			case K::num: return o.lit;
			case K::node:
			{
				tv r;
				r.i = (s[o.node / 32] >> (o.node % 32)) & 1u;
				return r;
			}
			case K::tern:
			{
				tv c = eval(o.a, s), x = eval(o.b, s), y = eval(o.c, s);
				tv r = c.truth() ? x : y;
				if (x.dbl || y.dbl)
				{
					r.d = r.get();
					r.dbl = true;
				}
				return r;
			}
			case K::un:
			{
				tv x = eval(o.a, s);
				if (o.op == '-')
				{
					x.d = -x.d;
					x.i = -x.i;
				}
				else if (o.op == '!')
				{
					tv r;
					r.i = x.truth() ? 0 : 1;
					return r;
				}
				return x;
			}
			case K::bin:
			{
				tv x = eval(o.a, s), y = eval(o.b, s), r;
				const bool dbl = x.dbl || y.dbl;
				switch (o.op)
				{
					case '+':
					case '-':
					case '*':
					case '/':
						if (dbl)
						{
							r.dbl = true;
							double p = x.get(), q = y.get();
							r.d = o.op == '+' ? p + q : o.op == '-' ? p - q : o.op == '*' ? p * q : p / q;
						}
						else
						{
							if (o.op == '/' && y.i == 0)
								throw std::runtime_error("integer division by zero in a rate");
							r.i = o.op == '+' ? x.i + y.i : o.op == '-' ? x.i - y.i : o.op == '*' ? x.i * y.i : x.i / y.i;
						}
						return r;
					case '&':
					case '|':
					case '^':
						if (dbl)
							throw std::runtime_error("bitwise operator on a floating-point operand");
						r.i = o.op == '&' ? (x.i & y.i) : o.op == '|' ? (x.i | y.i) : (x.i ^ y.i);
						return r;
					default:
					{
						bool v;
						if (dbl)
						{
							double p = x.get(), q = y.get();
							v = o.op == '=' ? p == q : o.op == 'n' ? p != q : o.op == '<' ? p < q : o.op == 'l' ? p <= q
								: o.op == '>' ? p > q : p >= q;
						}
						else
						{
							long long p = x.i, q = y.i;
							v = o.op == '=' ? p == q : o.op == 'n' ? p != q : o.op == '<' ? p < q : o.op == 'l' ? p <= q
								: o.op == '>' ? p > q : p >= q;
						}
						r.i = v;
						return r;
					}
				}
			}
			default: throw std::runtime_error("bad flat expression");
		}
	}
	tv eval(const uint32_t* s) const { return eval(root, s); }
};

struct compiled
{
	model m;
	int N = 0, W = 0;
	std::vector<int> ni;			// non-internal nodes in order
	std::vector<char> fast;			// fast-path form (generator.cpp:57-82)
	std::vector<float> up, down;	// fast-path rate values as compiled
	std::vector<float> ul, dl;		// r * log2(r) constants of the fast-mode entropy
	std::vector<P> up_expr, down_expr; // U and D expressions of fast-path nodes
	std::vector<flat> logic, rup, rdown;
	// truth tables of fast-path logic (exactly the flat evaluation, tabulated over the inputs)
	std::vector<std::vector<int>> tt_in;
	std::vector<std::vector<uint64_t>> tt;
	bool nonneg = true;
	// integer-rate fast mode (all rates of the @logic form, logic fan-in <= 12, enough resolution)
	bool integer_rates = false;
	int shift = 0;
	std::vector<unsigned> q_up, q_down;
	// node -> the nodes whose rate a flip of it can change (itself and every node whose logic reads
	// it), for the incremental restatement (trajectory_integer_incremental)
	std::vector<std::vector<int>> deps;
	bool discrete = false;
	float max_time_f = 0, tick_f = 0;	  // exact floats (window statistics)
	float max_time_sim = 0, tick_sim = 0; // 6-significant-digit constexprs used by simulate
	long long sample_count = 0;
	unsigned long long seed = 0;
	int T = 0;

	float constant(const char* n) const
	{
		auto it = m.consts.find(n);
		return it == m.consts.end() ? 0.f : it->second;
	}

	bool logic_ternary(const P& e, bool is_up, float& val) const
	{
		if (!e || e->k != K::tern || e->a->k != K::alias || e->a->s != "@logic")
			return false;
		if (!is_const(m, *e->b) || !is_const(m, *e->c))
			return false;
		float l = feval(m, *e->b), r = feval(m, *e->c);
		val = is_up ? l : r;
		return (is_up ? r : l) == 0.f;
	}

	// <node>_rate of the generated code (generator.cpp:84-122)
	float rate(int i, const uint32_t* s) const
	{
		const bool is_up = (s[i / 32] >> (i % 32)) & 1u;
		if (fast[i])
		{
			bool lg;
			if (!tt[i].empty())
			{
				unsigned p = 0;
				const std::vector<int>& in = tt_in[i];
				for (size_t k = 0; k < in.size(); k++)
					p |= ((s[in[k] / 32] >> (in[k] % 32)) & 1u) << k;
				lg = (tt[i][p >> 6] >> (p & 63)) & 1u;
			}
			else
				lg = logic[i].eval(s).truth();
			return is_up == lg ? 0.f : (is_up ? down[i] : up[i]);
		}
		tv r = is_up ? rdown[i].eval(s) : rup[i].eval(s);
		return (float)r.get();
	}

	unsigned __int128 ni_index(const uint32_t* s) const
	{
		unsigned __int128 idx = 0;
		for (size_t k = 0; k < ni.size(); k++)
			idx |= (unsigned __int128)((s[ni[k] / 32] >> (ni[k] % 32)) & 1u) << k;
		return idx;
	}
};

float print6(float v)
{
	char buf[64];
	std::snprintf(buf, sizeof buf, "%g", (double)v);
	return (float)std::strtod(buf, nullptr);
}

void setup_integer_rates(compiled& c);

std::unique_ptr<compiled> compile(const std::string& bnd, const std::string& cfg)
{
	auto c = std::make_unique<compiled>();
	model& m = c->m;
	m.consts["discrete_time"] = 0; // driver.cpp:7-14
	m.consts["sample_count"] = 1000000;
	m.consts["max_time"] = 10;
	m.consts["time_tick"] = 0.1f;
	m.consts["seed_pseudorandom"] = 0;
	parser(bnd, m).bnd();
	parser(cfg, m).cfg();
	c->N = (int)m.nodes.size();
	c->W = (c->N + 31) / 32;
	c->fast.assign(c->N, 0);
	c->up.assign(c->N, 0);
	c->down.assign(c->N, 0);
	c->ul.assign(c->N, 0);
	c->dl.assign(c->N, 0);
	for (int i = 0; i < c->N; i++)
	{
		const node_def& n = m.nodes[i];
		P internal = n.attr("is_internal");
		if (!(internal && feval(m, *internal) != 0.f))
			c->ni.push_back(i);
		float u = 0, d = 0;
		const bool f =
			n.attr("logic") && c->logic_ternary(n.attr("rate_up"), true, u) && c->logic_ternary(n.attr("rate_down"), false, d);
		c->fast[i] = f;
		c->up_expr.push_back(f ? n.attr("rate_up")->b : nullptr);
		c->down_expr.push_back(f ? n.attr("rate_down")->c : nullptr);
		if (f)
		{
			c->up[i] = (float)printed(u).get();
			c->down[i] = (float)printed(d).get();
			c->ul[i] = c->up[i] > 0 ? (float)((double)c->up[i] * std::log2((double)c->up[i])) : 0.f;
			c->dl[i] = c->down[i] > 0 ? (float)((double)c->down[i] * std::log2((double)c->down[i])) : 0.f;
			if (!(c->up[i] >= 0) || !(c->down[i] >= 0))
				c->nonneg = false;
		}
		else
			c->nonneg = false;
	}
	c->logic.resize(c->N);
	c->rup.resize(c->N);
	c->rdown.resize(c->N);
	for (int i = 0; i < c->N; i++)
	{
		const node_def& n = m.nodes[i];
		if (c->fast[i])
			c->logic[i].root = c->logic[i].add(m, *n.attr("logic"), i);
		else
		{
			c->rup[i].root = c->rup[i].add(m, *n.attr("rate_up"), i);
			c->rdown[i].root = c->rdown[i].add(m, *n.attr("rate_down"), i);
		}
	}
	c->tt_in.resize(c->N);
	c->tt.resize(c->N);
	for (int i = 0; i < c->N; i++)
	{
		if (!c->fast[i])
			continue;
		std::vector<int> in;
		for (auto& o : c->logic[i].ops)
			if (o.k == K::node && std::find(in.begin(), in.end(), o.node) == in.end())
				in.push_back(o.node);
		if (in.size() > 16)
			continue;
		std::vector<uint64_t> t(((1u << in.size()) + 63) / 64, 0);
		std::vector<uint32_t> st(c->W, 0u);
		for (unsigned p = 0; p < (1u << in.size()); p++)
		{
			for (size_t k = 0; k < in.size(); k++)
			{
				const uint32_t bit = 1u << (in[k] % 32);
				st[in[k] / 32] = (p >> k) & 1u ? (st[in[k] / 32] | bit) : (st[in[k] / 32] & ~bit);
			}
			if (c->logic[i].eval(st.data()).truth())
				t[p >> 6] |= 1ull << (p & 63);
		}
		c->tt_in[i] = in;
		c->tt[i] = t;
	}
	setup_integer_rates(*c);
	c->discrete = c->constant("discrete_time") != 0;
	c->max_time_f = c->constant("max_time");
	c->tick_f = c->constant("time_tick");
	c->max_time_sim = print6(c->max_time_f);
	c->tick_sim = print6(c->tick_f);
	c->sample_count = (long long)c->constant("sample_count");
	c->seed = (unsigned long long)c->constant("seed_pseudorandom");
	c->T = (int)std::ceil(c->max_time_f / c->tick_f);
	return c;
}

// integer-rate eligibility and fixed-point scale: largest per-32-node-word sum of max(up, down)
// below 2^31 (the engine's build_incremental_tables)
void setup_integer_rates(compiled& cc)
{
	compiled* c = &cc;
	c->integer_rates = c->N > 0;
	for (int i = 0; i < c->N; i++)
		if (!c->fast[i] || c->tt_in[i].size() > 12 || c->tt[i].empty())
			c->integer_rates = false;
	if (c->integer_rates)
	{
		// the engine's rule (codegen.cpp: integer_rate_shift): the largest shift <= 31 with every
		// word's largest rate sum below 2^32 units; every positive rate at least 2^20 units
		double worst = 0;
		for (int w = 0; w < c->W; w++)
		{
			double sw = 0;
			for (int i = 32 * w; i < std::min(c->N, 32 * w + 32); i++)
				sw += std::max(std::max((double)c->up[i], (double)c->down[i]), 0.0);
			worst = std::max(worst, sw);
		}
		int sh = 31;
		while (sh > 0 && worst * std::ldexp(1.0, sh) >= 4294967296.0)
			sh--;
		c->shift = sh;
		c->q_up.resize(c->N);
		c->q_down.resize(c->N);
		for (int i = 0; i < c->N; i++)
		{
			const double qu = std::nearbyint(std::max(0.0, (double)c->up[i]) * std::ldexp(1.0, sh));
			const double qd = std::nearbyint(std::max(0.0, (double)c->down[i]) * std::ldexp(1.0, sh));
			if (!(c->up[i] >= 0.f) || !(c->down[i] >= 0.f) || (c->up[i] > 0 && qu < 1048576.0) ||
				(c->down[i] > 0 && qd < 1048576.0))
				c->integer_rates = false;
			c->q_up[i] = (unsigned)qu;
			c->q_down[i] = (unsigned)qd;
		}
		c->deps.assign(c->N, {});
		for (int i = 0; i < c->N; i++)
		{
			c->deps[i].push_back(i);
			for (int x : c->tt_in[i])
				if (x != i)
					c->deps[x].push_back(i);
		}
	}
}


// ------------------------------------------------------------------ simulation

// static_state_t::operator< (state.h:43-49): compare from the highest word down
struct state_less
{
	bool operator()(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) const
	{
		for (size_t w = a.size(); w-- > 0;)
			if (a[w] != b[w])
				return a[w] < b[w];
		return false;
	}
};

struct sinks
{
	int T = 0;
	uint32_t S = 0;
	double fx = 1, fxh = 1;
	std::vector<long long> occ, h;
	std::vector<unsigned> cnt, fin;
	std::map<std::vector<uint32_t>, unsigned, state_less> fixed;
	unsigned long long transitions = 0;
	// sparse bins (more than 20 non-internal nodes, or forced): (window, index) -> occupancy or count,
	// and index -> final count, merged from the threads' maps at the end of a run
	bool sparse = false;
	std::map<std::pair<int, unsigned __int128>, long long> sp;
	std::map<unsigned __int128, unsigned long long> sp_fin;
};

template <typename T>
void atomic_add(T* p, T v)
{
	__atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}

struct run_acc
{
	int ow = -1;
	unsigned __int128 oi = 0;
	long long oq = 0;
	int hw = -1;
	long long hq = 0;
	std::map<std::pair<int, unsigned __int128>, long long> sp; // this thread's sparse bins
	std::map<unsigned __int128, unsigned long long> sp_fin;
	void add_occ(sinks& s, int w, unsigned __int128 idx, long long q)
	{
		if (s.sparse)
			sp[{ w, idx }] += q;
		else
			atomic_add(&s.occ[(size_t)w * s.S + idx], q);
	}
	void add_cnt(sinks& s, int w, unsigned __int128 idx)
	{
		if (s.sparse)
			sp[{ w, idx }] += 1;
		else
			atomic_add(&s.cnt[(size_t)w * s.S + idx], 1u);
	}
	void add_fin(sinks& s, unsigned __int128 idx)
	{
		if (s.sparse)
			sp_fin[idx] += 1;
		else
			atomic_add(&s.fin[idx], 1u);
	}
	void flush(sinks& s)
	{
		if (ow >= 0 && oq)
			add_occ(s, ow, oi, oq);
		if (hw >= 0 && hq)
			atomic_add(&s.h[hw], hq);
		ow = hw = -1;
		oq = hq = 0;
	}
	// the thread's sparse bins into the run's (after flush)
	void merge(sinks& s)
	{
		if (!s.sparse)
			return;
#pragma omp critical(oracle_sparse)
		{
			for (auto& kv : sp)
				s.sp[kv.first] += kv.second;
			for (auto& kv : sp_fin)
				s.sp_fin[kv.first] += kv.second;
		}
		sp.clear();
		sp_fin.clear();
	}
};

// window_average_small.cu:66-92 (continuous) and :117-130 (discrete)
void record(const compiled& c, sinks& s, run_acc& a, unsigned __int128 idx, float t0, float t1, float h)
{
	if (t1 == 0.f)
		return;
	if (c.discrete)
	{
		const int w = (int)lroundf(t0 / c.tick_f);
		if (w >= 0 && w < s.T)
		{
			a.add_cnt(s, w, idx);
			long long q = llrint((double)h * s.fxh);
			if (q)
				atomic_add(&s.h[w], q);
		}
		return;
	}
	float sb = t0;
	int w = (int)floorf(sb / c.tick_f);
	for (int guard = 0; t1 > sb && guard <= s.T + 2; guard++)
	{
		const float we = (float)(w + 1) * c.tick_f;
		const float se = std::fmin(t1, we);
		const float sl = se - sb;
		if (w >= 0 && w < s.T)
		{
			const long long q = llrint((double)sl * s.fx);
			if (w == a.ow && idx == a.oi)
				a.oq += q;
			else
			{
				if (a.ow >= 0 && a.oq)
					a.add_occ(s, a.ow, a.oi, a.oq);
				a.ow = w;
				a.oi = idx;
				a.oq = q;
			}
			const float hs = h * sl;
			const long long hq = llrint((double)hs * s.fxh);
			if (w == a.hw)
				a.hq += hq;
			else
			{
				if (a.hw >= 0 && a.hq)
					atomic_add(&s.h[a.hw], a.hq);
				a.hw = w;
				a.hq = hq;
			}
		}
		w++;
		sb = se;
	}
}

// compute_transition_entropy over the rates of one step (generator.cpp:146-175)
float entropy_exact(const compiled& c, const float* rates)
{
	float tot = 0.f;
	for (int i : c.ni)
		tot += rates[i];
	if (tot == 0.f)
		return 0.f;
	float e = 0.f;
	for (int i : c.ni)
	{
		const float p = rates[i] / tot;
		e -= (p == 0.f) ? 0.f : log2f(p) * p;
	}
	return e;
}

// fast-mode entropy: log2(S) - (sum r log2 r) / S with r log2 r from per-node constants
float entropy_fast(const compiled& c, const float* rates, const uint32_t* s)
{
	float t = 0.f, tl = 0.f;
	for (int i : c.ni)
	{
		const float r = rates[i];
		if (c.fast[i])
		{
			if (r != 0.f)
			{
				const bool up = (s[i / 32] >> (i % 32)) & 1u;
				t += up ? c.down[i] : c.up[i];
				tl += up ? c.dl[i] : c.ul[i];
			}
		}
		else
		{
			t += r;
			tl += (r > 0.f) ? r * log2f(r) : 0.f;
		}
	}
	if (!(t > 0.f))
		return 0.f;
	const float h = log2f(t) - tl / t;
	return h > 0.f ? h : 0.f;
}

// One trajectory (simulation.cu:34-71 initial state, :77-164 loop; simulation_runner.cu:104-162
// epochs). `trace` (optional) receives (flip, time) per step.
// Fast mode with integer rates (the engine's incremental kernel): rates in fixed point
// q = round(rate * 2^shift), the flip drawn as the first node (in node order) whose cumulative
// integer rate exceeds r = floor(u64 * total / 2^64), u64 from two raw 32-bit draws.
void trajectory_integer(const compiled& c, sinks& s, unsigned long long seed, unsigned long long traj, run_acc& acc,
						unsigned long long& trans, std::vector<std::pair<int, float>>* trace)
{
	curandStatePhilox4_32_10_t rng;
	curand_init(seed, traj, 0ull, &rng);
	std::vector<uint32_t> st(c.W, 0u);
	std::vector<float> rates(c.N);
	std::vector<unsigned> q(c.N);
	for (int i = 0; i < c.N; i++)
		if (curand_uniform(&rng) <= c.m.nodes[i].istate)
			st[i / 32] |= 1u << (i % 32);
	const float inv_scale = 1.0f / (float)(1u << c.shift);
	// the stream continues at the next whole Philox block; each step consumes one block of four
	// 32-bit outputs: x for the waiting time, (y, z) for the flip
	curand_init(seed, traj, (unsigned long long)((c.N + 3) & ~3), &rng);
	float time = 0.f;
	bool fixed = false;
	for (;;)
	{
		const uint4 rb = curand4(&rng);
		unsigned long long total = 0;
		for (int i = 0; i < c.N; i++)
		{
			rates[i] = c.rate(i, st.data());
			q[i] = 0;
		}
		for (int i = 0; i < c.N; i++)
		{
			const bool on = (st[i / 32] >> (i % 32)) & 1u;
			// unstable <=> bit differs from logic <=> the generated rate takes the U/D branch
			unsigned p = 0;
			const std::vector<int>& in = c.tt_in[i];
			for (size_t k = 0; k < in.size(); k++)
				p |= ((st[in[k] / 32] >> (in[k] % 32)) & 1u) << k;
			const bool lg = (c.tt[i][p >> 6] >> (p & 63)) & 1u;
			if (on != lg)
				q[i] = on ? c.q_down[i] : c.q_up[i];
			total += q[i];
		}
		float h = 0.f, tn;
		if (total == 0)
		{
			fixed = true;
			tn = c.max_time_sim;
		}
		else
		{
			if (c.discrete)
			{
				tn = time + c.tick_sim;
				tn = c.max_time_sim - c.tick_sim < tn ? c.max_time_sim : tn;
			}
			else
			{
				const float total_f = (float)total * inv_scale;
				const float u = (float)((rb.x >> 8) + 1u) * 5.9604644775390625e-8f; // (top 24 bits + 1) / 2^24
				tn = time + -logf(u) / total_f;
			}
			tn = std::fmin(tn, c.max_time_sim);
			h = entropy_fast(c, rates.data(), st.data());
		}
		trans += tn != 0.f;
		record(c, s, acc, c.ni_index(st.data()), time, tn, h);
		time = tn;
		if (time >= c.max_time_sim)
		{
			if (trace)
				trace->emplace_back(-1, time);
			break;
		}
		const unsigned long long r64 = ((unsigned long long)rb.y << 32) | rb.z;
		const unsigned long long r = (unsigned long long)(((unsigned __int128)r64 * total) >> 64);
		unsigned long long cum = 0;
		int j = -1;
		for (int i = 0; i < c.N; i++)
		{
			cum += q[i];
			if (r < cum)
			{
				j = i;
				break;
			}
		}
		if (trace)
			trace->emplace_back(j, time);
		st[j / 32] ^= 1u << (j % 32);
	}
	acc.add_fin(s, c.ni_index(st.data()));
	if (fixed)
	{
#pragma omp critical(oracle_fixed)
		s.fixed[st]++;
	}
}

// The same process, random numbers and results as trajectory_integer (bit for bit), computed the
// way the engine's incremental fast kernel does: the unstable nodes (bit != logic), the integer
// rate sum of every state word and the total are kept across steps; after a flip only the
// flipped node and the nodes whose logic reads it are re-evaluated, and the flip is found by
// skipping whole words by their sums, then scanning the chosen word's unstable bits in node order
// (the first node whose cumulative integer rate exceeds r, as the full scan finds it). This is
// the CPU baseline on the GPU kernel's algorithm (mode 2); tests check it equals mode 1.
void trajectory_integer_incremental(const compiled& c, sinks& s, unsigned long long seed, unsigned long long traj,
									run_acc& acc, unsigned long long& trans)
{
	curandStatePhilox4_32_10_t rng;
	curand_init(seed, traj, 0ull, &rng);
	std::vector<uint32_t> st(c.W, 0u), un(c.W, 0u);
	std::vector<unsigned long long> wsum(c.W, 0ull);
	for (int i = 0; i < c.N; i++)
		if (curand_uniform(&rng) <= c.m.nodes[i].istate)
			st[i / 32] |= 1u << (i % 32);
	auto logic = [&](int i) {
		unsigned p = 0;
		const std::vector<int>& in = c.tt_in[i];
		for (size_t k = 0; k < in.size(); k++)
			p |= ((st[in[k] / 32] >> (in[k] % 32)) & 1u) << k;
		return ((c.tt[i][p >> 6] >> (p & 63)) & 1u) != 0;
	};
	auto q_of = [&](int i) -> unsigned {
		if (!((un[i / 32] >> (i % 32)) & 1u))
			return 0u;
		return ((st[i / 32] >> (i % 32)) & 1u) ? c.q_down[i] : c.q_up[i];
	};
	unsigned long long total = 0;
	for (int i = 0; i < c.N; i++)
	{
		const bool on = (st[i / 32] >> (i % 32)) & 1u;
		if (on != logic(i))
			un[i / 32] |= 1u << (i % 32);
		const unsigned q = q_of(i);
		wsum[i / 32] += q;
		total += q;
	}
	// entropy_fast over the non-internal nodes: a node contributes when its integer rate is
	// non-zero, which holds exactly when its float rate is (positive rates have >= 2^20 units)
	auto entropy = [&]() {
		float t = 0.f, tl = 0.f;
		for (int i : c.ni)
			if (q_of(i) != 0u)
			{
				const bool up = (st[i / 32] >> (i % 32)) & 1u;
				t += up ? c.down[i] : c.up[i];
				tl += up ? c.dl[i] : c.ul[i];
			}
		if (!(t > 0.f))
			return 0.f;
		const float h = log2f(t) - tl / t;
		return h > 0.f ? h : 0.f;
	};
	const float inv_scale = 1.0f / (float)(1u << c.shift);
	curand_init(seed, traj, (unsigned long long)((c.N + 3) & ~3), &rng);
	float time = 0.f;
	bool fixed = false;
	for (;;)
	{
		const uint4 rb = curand4(&rng);
		float h = 0.f, tn;
		if (total == 0)
		{
			fixed = true;
			tn = c.max_time_sim;
		}
		else
		{
			if (c.discrete)
			{
				tn = time + c.tick_sim;
				tn = c.max_time_sim - c.tick_sim < tn ? c.max_time_sim : tn;
			}
			else
			{
				const float total_f = (float)total * inv_scale;
				const float u = (float)((rb.x >> 8) + 1u) * 5.9604644775390625e-8f;
				tn = time + -logf(u) / total_f;
			}
			tn = std::fmin(tn, c.max_time_sim);
			h = entropy();
		}
		trans += tn != 0.f;
		record(c, s, acc, c.ni_index(st.data()), time, tn, h);
		time = tn;
		if (time >= c.max_time_sim)
			break;
		const unsigned long long r64 = ((unsigned long long)rb.y << 32) | rb.z;
		const unsigned long long r = (unsigned long long)(((unsigned __int128)r64 * total) >> 64);
		unsigned long long cum = 0;
		int w = 0;
		while (w < c.W - 1 && r >= cum + wsum[w])
			cum += wsum[w++];
		int j = 32 * w + 31;
		for (uint32_t um = un[w]; um; um &= um - 1u)
		{
			const int i = 32 * w + __builtin_ctz(um);
			cum += q_of(i);
			if (r < cum)
			{
				j = i;
				break;
			}
		}
		st[j / 32] ^= 1u << (j % 32);
		for (int k : c.deps[j])
		{
			const unsigned qo = (k == j) ? ((((st[k / 32] >> (k % 32)) & 1u) ? c.q_up[k] : c.q_down[k]) *
											 ((un[k / 32] >> (k % 32)) & 1u))
										 : q_of(k);
			const bool on = (st[k / 32] >> (k % 32)) & 1u;
			if (on != logic(k))
				un[k / 32] |= 1u << (k % 32);
			else
				un[k / 32] &= ~(1u << (k % 32));
			const unsigned qn = q_of(k);
			wsum[k / 32] += (unsigned long long)qn - qo;
			total += (unsigned long long)qn - qo;
		}
	}
	acc.add_fin(s, c.ni_index(st.data()));
	if (fixed)
	{
#pragma omp critical(oracle_fixed)
		s.fixed[st]++;
	}
}

// Score-function (likelihood-ratio) gradient of sum_w,b cot[w][b] * (window statistic) along the
// trajectories of trajectory_integer (same Philox streams, integer rates, flips), stated directly:
// the score of parameter p at time t is S_p(t) = J_p(t) - I_p(t), J_p the sum over the jumps so far
// of (d rate_j / d theta_p) / rate_j and I_p the integral of d a0 / d theta_p, recomputed from all
// unstable nodes at every step; every window slice adds cot * integral of S_p over the slice
// (continuous time) or cot * S_p (discrete time, whose score is sum over jumps of
// d log rate_j - d log a0). The engine's batched gradient kernel keeps the same quantities
// incrementally; this checks it. dR is a CSR over entry 2i (node i's up rate) and 2i + 1 (its down
// rate) of (parameter, d rate / d parameter); grad receives the sum over trajectories (unscaled).
void gradient_integer(const compiled& c, unsigned long long seed, unsigned long long traj, const double* cot,
					  int P, const int* gptr, const int* gp, const float* gd, std::vector<double>& G)
{
	curandStatePhilox4_32_10_t rng;
	curand_init(seed, traj, 0ull, &rng);
	std::vector<uint32_t> st(c.W, 0u);
	for (int i = 0; i < c.N; i++)
		if (curand_uniform(&rng) <= c.m.nodes[i].istate)
			st[i / 32] |= 1u << (i % 32);
	const float inv_scale = 1.0f / (float)(1u << c.shift);
	curand_init(seed, traj, (unsigned long long)((c.N + 3) & ~3), &rng);
	const size_t S = (size_t)1 << c.ni.size();
	std::vector<unsigned> q(c.N);
	std::vector<double> J(P, 0.0), I(P, 0.0), D(P, 0.0);
	float time = 0.f;
	for (;;)
	{
		const uint4 rb = curand4(&rng);
		unsigned long long total = 0;
		std::fill(D.begin(), D.end(), 0.0);
		for (int i = 0; i < c.N; i++)
		{
			const bool on = (st[i / 32] >> (i % 32)) & 1u;
			unsigned p = 0;
			const std::vector<int>& in = c.tt_in[i];
			for (size_t k = 0; k < in.size(); k++)
				p |= ((st[in[k] / 32] >> (in[k] % 32)) & 1u) << k;
			const bool lg = (c.tt[i][p >> 6] >> (p & 63)) & 1u;
			q[i] = 0;
			if (on != lg)
			{
				q[i] = on ? c.q_down[i] : c.q_up[i];
				const int e = 2 * i + (on ? 1 : 0);
				for (int k = gptr[e]; k < gptr[e + 1]; k++)
					D[gp[k]] += gd[k];
			}
			total += q[i];
		}
		float tn;
		if (total == 0)
			tn = c.max_time_sim;
		else
		{
			if (c.discrete)
			{
				tn = time + c.tick_sim;
				tn = c.max_time_sim - c.tick_sim < tn ? c.max_time_sim : tn;
			}
			else
			{
				const float total_f = (float)total * inv_scale;
				const float u = (float)((rb.x >> 8) + 1u) * 5.9604644775390625e-8f;
				tn = time + -logf(u) / total_f;
			}
			tn = std::fmin(tn, c.max_time_sim);
		}
		const size_t idx = (size_t)c.ni_index(st.data());
		if (tn != 0.f)
		{
			if (c.discrete)
			{
				const int w = (int)lroundf(time / c.tick_f);
				if (w >= 0 && w < c.T)
					for (int p = 0; p < P; p++)
						G[p] += cot[(size_t)w * S + idx] * (J[p] - I[p]);
			}
			else
			{
				// the window slices of record(), each integrated exactly: S_p is linear on the step
				float sb = time;
				int w = (int)floorf(sb / c.tick_f);
				for (int guard = 0; tn > sb && guard <= c.T + 2; guard++)
				{
					const float se = std::fmin(tn, (float)(w + 1) * c.tick_f);
					if (w >= 0 && w < c.T)
					{
						const double cw = cot[(size_t)w * S + idx];
						const double len = (double)se - (double)sb, mid = 0.5 * ((double)sb + (double)se);
						for (int p = 0; p < P; p++)
							G[p] += cw * len * (J[p] - I[p] - D[p] * (mid - (double)time));
					}
					w++;
					sb = se;
				}
				for (int p = 0; p < P; p++)
					I[p] += D[p] * ((double)tn - (double)time);
			}
		}
		time = tn;
		if (time >= c.max_time_sim)
			break;
		const unsigned long long r64 = ((unsigned long long)rb.y << 32) | rb.z;
		const unsigned long long r = (unsigned long long)(((unsigned __int128)r64 * total) >> 64);
		unsigned long long cum = 0;
		int j = -1;
		for (int i = 0; i < c.N; i++)
		{
			cum += q[i];
			if (r < cum)
			{
				j = i;
				break;
			}
		}
		const bool on_j = (st[j / 32] >> (j % 32)) & 1u;
		const double rj = on_j ? c.down[j] : c.up[j];
		const int e = 2 * j + (on_j ? 1 : 0);
		for (int k = gptr[e]; k < gptr[e + 1]; k++)
			J[gp[k]] += (double)gd[k] / rj;
		if (c.discrete)
		{
			const double a0 = (double)((float)total * inv_scale);
			for (int p = 0; p < P; p++)
				I[p] += D[p] / a0;
		}
		st[j / 32] ^= 1u << (j % 32);
	}
}

template <typename RNG>
void trajectory(const compiled& c, sinks& s, RNG& rng, bool exact, int traj_len, run_acc& acc,
				unsigned long long& trans, std::vector<std::pair<int, float>>* trace)
{
	std::vector<uint32_t> st(c.W, 0u);
	std::vector<float> rates(c.N);
	for (int i = 0; i < c.N; i++)
		if (curand_uniform(&rng) <= c.m.nodes[i].istate)
			st[i / 32] |= 1u << (i % 32);
	float time = 0.f;
	int slot = 1;
	bool fixed = false;
	for (;;)
	{
		// compute_transition_rates: rates in node order, sequential fp32 sum (generator.cpp:124-144)
		float total = 0.f;
		for (int i = 0; i < c.N; i++)
		{
			rates[i] = c.rate(i, st.data());
			total += rates[i];
		}
		float h = 0.f, tn;
		if (total == 0.f)
		{
			fixed = true;
			tn = c.max_time_sim;
		}
		else
		{
			if (c.discrete)
			{
				tn = time + c.tick_sim;
				tn = c.max_time_sim - c.tick_sim < tn ? c.max_time_sim : tn;
			}
			else
			{
				const float u = curand_uniform(&rng);
				tn = time + -logf(u) / total;
			}
			tn = std::fmin(tn, c.max_time_sim);
			h = exact ? entropy_exact(c, rates.data()) : entropy_fast(c, rates.data(), st.data());
		}
		trans += tn != 0.f;
		record(c, s, acc, c.ni_index(st.data()), time, tn, h);
		time = tn;
		if (time >= c.max_time_sim)
		{
			if (trace)
				trace->emplace_back(-1, time);
			break;
		}
		if (exact && traj_len > 1 && ++slot >= traj_len)
		{
			slot = 1;
			if (trace)
				trace->emplace_back(-2, time);
			continue;
		}
		// select_flip_bit, simulation.cu:9-21
		const float r = curand_uniform(&rng) * total;
		float sum = 0.f;
		int idx = 0;
		for (int i = 0; i < c.N; i++)
		{
			sum += rates[i];
			idx += (sum < r) ? 1 : 0;
		}
		if (idx >= c.N)
			idx = c.N - 1;
		if (trace)
			trace->emplace_back(idx, time);
		st[idx / 32] ^= 1u << (idx % 32);
	}
	acc.add_fin(s, c.ni_index(st.data()));
	if (fixed)
	{
#pragma omp critical(oracle_fixed)
		s.fixed[st]++;
	}
}

} // namespace

// ------------------------------------------------------------------ C interface (ctypes)

struct oracle_model
{
	std::unique_ptr<compiled> c;
	std::string err;
};

struct oracle_result
{
	sinks s;
	std::vector<uint32_t> fixed_states;
	std::vector<unsigned> fixed_counts;
	double seconds = 0;
};

extern "C" {

oracle_model* oracle_model_load(const char* bnd_text, const char* cfg_text, char* err, size_t errcap)
{
	try
	{
		auto m = new oracle_model;
		m->c = compile(bnd_text, cfg_text);
		return m;
	}
	catch (const std::exception& e)
	{
		if (err && errcap)
			std::snprintf(err, errcap, "%s", e.what());
		return nullptr;
	}
}

void oracle_model_free(oracle_model* m) { delete m; }

// dims: nodes, words, non-internal count, windows, discrete, sample_count, seed, tick, max_time
int oracle_model_dims(const oracle_model* m, int* nodes, int* words, int* noninternal, int* windows, int* discrete,
					  long long* sample_count, unsigned long long* seed, float* tick, float* max_time)
{
	const compiled& c = *m->c;
	*nodes = c.N;
	*words = c.W;
	*noninternal = (int)c.ni.size();
	*windows = c.T;
	*discrete = c.discrete;
	*sample_count = c.sample_count;
	*seed = c.seed;
	*tick = c.tick_f;
	*max_time = c.max_time_f;
	return 0;
}

// Set $variables and recompute the rates of @logic-form nodes as exact floats (no 6-digit
// rounding), as the engine's batched runs do. Returns 0, or -1 for an unknown variable.
int oracle_model_set_variables(oracle_model* m, const char* const* names, const float* values, int n)
{
	compiled& c = *m->c;
	for (int i = 0; i < n; i++)
	{
		if (!c.m.vars.count(names[i]))
			return -1;
		c.m.vars[names[i]] = values[i];
	}
	for (int i = 0; i < c.N; i++)
	{
		if (!c.fast[i])
			continue;
		c.up[i] = feval(c.m, *c.up_expr[i]);
		c.down[i] = feval(c.m, *c.down_expr[i]);
		c.ul[i] = c.up[i] > 0 ? (float)((double)c.up[i] * std::log2((double)c.up[i])) : 0.f;
		c.dl[i] = c.down[i] > 0 ? (float)((double)c.down[i] * std::log2((double)c.down[i])) : 0.f;
	}
	setup_integer_rates(c);
	return 0;
}

// 1 when fast mode uses integer rates (the engine's incremental kernel); writes the scale
int oracle_model_integer_rates(const oracle_model* m, int* shift)
{
	if (shift)
		*shift = m->c->shift;
	return m->c->integer_rates ? 1 : 0;
}

int oracle_model_noninternal(const oracle_model* m, int* out)
{
	for (size_t k = 0; k < m->c->ni.size(); k++)
		out[k] = m->c->ni[k];
	return (int)m->c->ni.size();
}

// Rate of node i and the total in state `s` (for unit tests of the model semantics).
float oracle_model_rate(const oracle_model* m, int i, const uint32_t* s) { return m->c->rate(i, s); }

// Run n trajectories [first, first + n). Fixed-point exponents must be those of the GPU run.
// flags: 1 = sparse bins even with at most 20 non-internal nodes (to pin the sparse path against
// the dense one); more than 20 non-internal nodes (at most 112) always use sparse bins.
oracle_result* oracle_run_ex(const oracle_model* m, int mode, long long n, unsigned long long seed,
							 unsigned long long first, int traj_len, int occ_exp, int ent_exp, int threads, int flags)
{
	const compiled& c = *m->c;
	if (c.ni.size() > 112)
		return nullptr;
	auto r = new oracle_result;
	sinks& s = r->s;
	s.T = c.T;
	s.sparse = c.ni.size() > 20 || (flags & 1);
	s.S = s.sparse ? 0u : 1u << c.ni.size();
	s.fx = std::ldexp(1.0, occ_exp);
	s.fxh = std::ldexp(1.0, ent_exp);
	if (!s.sparse && c.discrete)
		s.cnt.assign((size_t)s.T * s.S, 0u);
	else if (!s.sparse)
		s.occ.assign((size_t)s.T * s.S, 0);
	s.h.assign(s.T, 0);
	if (!s.sparse)
		s.fin.assign(s.S, 0u);
#ifdef _OPENMP
	const double t0 = omp_get_wtime();
	if (threads > 0)
		omp_set_num_threads(threads);
#endif
	unsigned long long trans = 0;
#pragma omp parallel reduction(+ : trans)
	{
		run_acc acc;
#pragma omp for schedule(dynamic, 16)
		for (long long t = 0; t < n; t++)
		{
			if (mode == 0)
			{
				curandState rng;
				curand_init(seed, first + (unsigned long long)t, 0ull, &rng);
				trajectory(c, s, rng, true, traj_len, acc, trans, nullptr);
			}
			else if (c.integer_rates && mode == 2)
				trajectory_integer_incremental(c, s, seed, first + (unsigned long long)t, acc, trans);
			else if (c.integer_rates)
				trajectory_integer(c, s, seed, first + (unsigned long long)t, acc, trans, nullptr);
			else
			{
				curandStatePhilox4_32_10_t rng;
				curand_init(seed, first + (unsigned long long)t, 0ull, &rng);
				trajectory(c, s, rng, false, 0, acc, trans, nullptr);
			}
		}
		acc.flush(s);
		acc.merge(s);
	}
	s.transitions = trans;
#ifdef _OPENMP
	r->seconds = omp_get_wtime() - t0;
#endif
	for (auto& kv : s.fixed)
	{
		r->fixed_states.insert(r->fixed_states.end(), kv.first.begin(), kv.first.end());
		r->fixed_counts.push_back(kv.second);
	}
	return r;
}

oracle_result* oracle_run(const oracle_model* m, int mode, long long n, unsigned long long seed,
						  unsigned long long first, int traj_len, int occ_exp, int ent_exp, int threads)
{
	return oracle_run_ex(m, mode, n, seed, first, traj_len, occ_exp, ent_exp, threads, 0);
}

void oracle_result_free(oracle_result* r) { delete r; }

// Sparse bins of a run: entry counts, then (window, index, value) sorted by window and index, and the
// final states (index, count) sorted by index.
int oracle_result_sparse_size(const oracle_result* r, long long* window_entries, long long* final_entries)
{
	*window_entries = (long long)r->s.sp.size();
	*final_entries = (long long)r->s.sp_fin.size();
	return r->s.sparse ? 1 : 0;
}

int oracle_result_sparse(const oracle_result* r, int* windows, uint64_t* idx, long long* vals, uint64_t* fin_idx,
						 unsigned long long* fin_cnt)
{
	// indices as (bits 0-63, bits 64-127) pairs
	size_t i = 0;
	for (auto& kv : r->s.sp)
	{
		windows[i] = kv.first.first;
		idx[2 * i] = (uint64_t)kv.first.second;
		idx[2 * i + 1] = (uint64_t)(kv.first.second >> 64);
		vals[i] = kv.second;
		i++;
	}
	i = 0;
	for (auto& kv : r->s.sp_fin)
	{
		fin_idx[2 * i] = (uint64_t)kv.first;
		fin_idx[2 * i + 1] = (uint64_t)(kv.first >> 64);
		fin_cnt[i] = kv.second;
		i++;
	}
	return 0;
}

int oracle_result_get(const oracle_result* r, long long* occ, unsigned* cnt, long long* h, unsigned* fin,
					  unsigned long long* transitions, double* seconds)
{
	const sinks& s = r->s;
	if (occ && !s.occ.empty())
		std::memcpy(occ, s.occ.data(), s.occ.size() * sizeof(long long));
	if (cnt && !s.cnt.empty())
		std::memcpy(cnt, s.cnt.data(), s.cnt.size() * sizeof(unsigned));
	if (h)
		std::memcpy(h, s.h.data(), s.h.size() * sizeof(long long));
	if (fin)
		std::memcpy(fin, s.fin.data(), s.fin.size() * sizeof(unsigned));
	if (transitions)
		*transitions = s.transitions;
	if (seconds)
		*seconds = r->seconds;
	return 0;
}

int oracle_result_num_fixed(const oracle_result* r) { return (int)r->fixed_counts.size(); }

int oracle_result_fixed(const oracle_result* r, uint32_t* states, unsigned* counts)
{
	if (states && !r->fixed_states.empty())
		std::memcpy(states, r->fixed_states.data(), r->fixed_states.size() * sizeof(uint32_t));
	if (counts && !r->fixed_counts.empty())
		std::memcpy(counts, r->fixed_counts.data(), r->fixed_counts.size() * sizeof(unsigned));
	return 0;
}

// Trace of one trajectory: flip indices (-1 = end, -2 = epoch boundary) and the time before
// each event. Returns the number of events (may exceed cap; only cap are written).
// gradient_integer summed over trajectories first .. first + n - 1 (integer-rate models only;
// returns -1 otherwise). grad[P] receives the unscaled sum.
int oracle_gradient(const oracle_model* m, unsigned long long seed, unsigned long long first, long long n,
					const double* cot, int P, const int* gptr, const int* gp, const float* gd, double* grad)
{
	const compiled& c = *m->c;
	if (!c.integer_rates || c.ni.size() > 20)
		return -1;
	std::vector<double> total(P, 0.0);
#pragma omp parallel
	{
		std::vector<double> G(P, 0.0);
#pragma omp for schedule(dynamic, 16)
		for (long long t = 0; t < n; t++)
			gradient_integer(c, seed, first + (unsigned long long)t, cot, P, gptr, gp, gd, G);
#pragma omp critical(oracle_gradient)
		for (int p = 0; p < P; p++)
			total[p] += G[p];
	}
	for (int p = 0; p < P; p++)
		grad[p] = total[p];
	return 0;
}

int oracle_trace(const oracle_model* m, int mode, unsigned long long seed, unsigned long long traj, int traj_len,
				 int* flips, float* times, int cap)
{
	const compiled& c = *m->c;
	sinks s;
	s.T = c.T;
	s.sparse = c.ni.size() > 20;
	s.S = s.sparse ? 0u : 1u << c.ni.size();
	s.occ.assign((size_t)s.T * s.S, 0);
	s.cnt.assign((size_t)s.T * s.S, 0);
	s.h.assign(s.T, 0);
	s.fin.assign(s.S, 0);
	std::vector<std::pair<int, float>> tr;
	run_acc acc;
	unsigned long long trans = 0;
	if (mode == 0)
	{
		curandState rng;
		curand_init(seed, traj, 0ull, &rng);
		trajectory(c, s, rng, true, traj_len, acc, trans, &tr);
	}
	else if (c.integer_rates)
		trajectory_integer(c, s, seed, traj, acc, trans, &tr);
	else
	{
		curandStatePhilox4_32_10_t rng;
		curand_init(seed, traj, 0ull, &rng);
		trajectory(c, s, rng, false, 0, acc, trans, &tr);
	}
	for (int i = 0; i < (int)tr.size() && i < cap; i++)
	{
		flips[i] = tr[i].first;
		times[i] = tr[i].second;
	}
	return (int)tr.size();
}

} // extern "C"
