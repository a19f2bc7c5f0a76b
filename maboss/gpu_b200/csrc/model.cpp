// Recursive-descent parser for .bnd/.cfg model files and the float evaluator / CUDA
// emitter for their expressions.
//
// Token set and lexical rules follow the reference scanner (src/parser/scanner.ll:51-94):
// blanks and `//` comments are skipped; `&`, `&&`, AND (any case) are one token, likewise
// `|`/`||`/OR, `^`/XOR, `!`/NOT; TRUE/FALSE are the numbers 1/0; `[0-9]+` is an integer,
// fractional or exponent forms are floats; `$id` is a variable, `@id` an alias.
// Grammar and operator precedence follow src/parser/parser.yy:74-158:
//   ?: (right, lowest) < XOR < OR < AND < (== !=) < (< <= > >=) < (+ -) < (* /) < unary.
// Semantic actions follow src/parser/driver.cpp:45-99.
#include "model.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace mb {

// ---------------------------------------------------------------- model basics

model_t::model_t()
{
	// driver.cpp:7-14
	constants["discrete_time"] = 0;
	constants["sample_count"] = 1'000'000;
	constants["max_time"] = 10;
	constants["time_tick"] = 0.1f;
	constants["seed_pseudorandom"] = 0;
}

const expr* node_t::find_attr(const std::string& attr) const
{
	for (auto& a : attrs)
		if (a.first == attr)
			return a.second.get();
	return nullptr;
}

void apply_cfg_overrides(model_t& m)
{
	for (auto& node : m.nodes)
	{
		decltype(node.attrs) kept;
		for (auto& a : node.attrs)
		{
			auto it = std::find_if(kept.begin(), kept.end(), [&](auto& k) { return k.first == a.first; });
			if (it == kept.end())
				kept.push_back(a);
			else
				it->second = a.second; // a later definition replaces the earlier one in place
		}
		node.attrs = std::move(kept);
	}
}

const expr& node_t::get_attr(const std::string& attr) const
{
	const expr* e = find_attr(attr);
	if (!e)
		throw model_error("Node " + name + " does not have attribute " + attr);
	return *e;
}

int model_t::node_index(const std::string& name) const
{
	for (size_t i = 0; i < nodes.size(); i++)
		if (nodes[i].name == name)
			return (int)i;
	return -1;
}

bool model_t::is_internal(size_t i) const
{
	const expr* e = nodes[i].find_attr("is_internal");
	return e && evaluate(*this, *e) != 0.f;
}

float model_t::constant(const std::string& name) const
{
	auto it = constants.find(name);
	return it == constants.end() ? 0.f : it->second;
}

int model_t::noninternal_count() const
{
	int c = 0;
	for (size_t i = 0; i < nodes.size(); i++)
		c += is_internal(i) ? 0 : 1;
	return c;
}

std::string print_float(float v)
{
	std::ostringstream os;
	os << v;
	return os.str();
}

// ---------------------------------------------------------------- lexer

namespace {

enum class tok
{
	END,
	IDENT,
	VARIABLE,
	ALIAS,
	FLOAT,
	NUMBER,
	ASSIGN,
	TERNARY,
	COLON,
	MINUS,
	PLUS,
	STAR,
	SLASH,
	AND,
	OR,
	XOR,
	NOT,
	EQ,
	NE,
	LT,
	LE,
	GT,
	GE,
	LPAREN,
	RPAREN,
	LBRACE,
	RBRACE,
	DOT,
	SEMICOLON,
	LBRACKET,
	RBRACKET,
	COMMA
};

const char* tok_name(tok t)
{
	switch (t)
	{
		case tok::END: return "end of file";
		case tok::IDENT: return "IDENTIFIER";
		case tok::VARIABLE: return "VARIABLE";
		case tok::ALIAS: return "ALIAS";
		case tok::FLOAT: return "FLOAT";
		case tok::NUMBER: return "NUMBER";
		case tok::ASSIGN: return "=";
		case tok::TERNARY: return "?";
		case tok::COLON: return ":";
		case tok::MINUS: return "-";
		case tok::PLUS: return "+";
		case tok::STAR: return "*";
		case tok::SLASH: return "/";
		case tok::AND: return "&&";
		case tok::OR: return "||";
		case tok::XOR: return "^";
		case tok::NOT: return "!";
		case tok::EQ: return "==";
		case tok::NE: return "!=";
		case tok::LT: return "<";
		case tok::LE: return "<=";
		case tok::GT: return ">";
		case tok::GE: return ">=";
		case tok::LPAREN: return "(";
		case tok::RPAREN: return ")";
		case tok::LBRACE: return "{";
		case tok::RBRACE: return "}";
		case tok::DOT: return ".";
		case tok::SEMICOLON: return ";";
		case tok::LBRACKET: return "[";
		case tok::RBRACKET: return "]";
		case tok::COMMA: return ",";
	}
	return "?";
}

struct token
{
	tok kind = tok::END;
	std::string text;
	float fval = 0.f;
	int ival = 0;
	int line = 1, col = 1;
};

class lexer
{
	const std::string& s_;
	const std::string& file_;
	size_t p_ = 0;
	int line_ = 1, col_ = 1;

	void advance(size_t n)
	{
		for (size_t i = 0; i < n; i++)
		{
			if (s_[p_] == '\n')
			{
				line_++;
				col_ = 1;
			}
			else
				col_++;
			p_++;
		}
	}

public:
	lexer(const std::string& s, const std::string& file) : s_(s), file_(file) {}

	[[noreturn]] void fail(int line, int col, const std::string& msg) const
	{
		throw model_error(file_ + ":" + std::to_string(line) + "." + std::to_string(col) + ": " + msg);
	}

	token next()
	{
		// skip blanks, newlines and line comments
		for (;;)
		{
			if (p_ >= s_.size())
				break;
			char c = s_[p_];
			if (c == ' ' || c == '\t' || c == '\r' || c == '\n')
			{
				advance(1);
				continue;
			}
			if (c == '/' && p_ + 1 < s_.size() && s_[p_ + 1] == '/')
			{
				while (p_ < s_.size() && s_[p_] != '\n')
					advance(1);
				continue;
			}
			break;
		}

		token t;
		t.line = line_;
		t.col = col_;
		if (p_ >= s_.size())
		{
			t.kind = tok::END;
			return t;
		}

		auto is_digit = [](char c) { return c >= '0' && c <= '9'; };
		auto is_alpha = [](char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z'); };
		auto is_idc = [&](char c) { return is_alpha(c) || is_digit(c) || c == '_'; };

		const char c = s_[p_];
		const char c1 = p_ + 1 < s_.size() ? s_[p_ + 1] : '\0';

		// numbers: longest of int / fracconst exppart? / int exppart
		if (is_digit(c) || (c == '.' && is_digit(c1)))
		{
			size_t q = p_;
			while (q < s_.size() && is_digit(s_[q]))
				q++;
			bool is_float = false;
			if (q < s_.size() && s_[q] == '.')
			{
				// "[0-9]+\." , "[0-9]+\.[0-9]+" or "\.[0-9]+"
				q++;
				while (q < s_.size() && is_digit(s_[q]))
					q++;
				is_float = true;
			}
			// optional exponent part [eE][-+]?[0-9]+
			if (q < s_.size() && (s_[q] == 'e' || s_[q] == 'E'))
			{
				size_t r = q + 1;
				if (r < s_.size() && (s_[r] == '-' || s_[r] == '+'))
					r++;
				if (r < s_.size() && is_digit(s_[r]))
				{
					while (r < s_.size() && is_digit(s_[r]))
						r++;
					q = r;
					is_float = true;
				}
			}
			t.text = s_.substr(p_, q - p_);
			if (is_float)
			{
				errno = 0;
				double d = std::strtod(t.text.c_str(), nullptr);
				if (errno == ERANGE)
					fail(t.line, t.col, "float is out of range: " + t.text);
				t.kind = tok::FLOAT;
				t.fval = (float)d;
			}
			else
			{
				errno = 0;
				long n = std::strtol(t.text.c_str(), nullptr, 10);
				if (!(INT_MIN <= n && n <= INT_MAX && errno != ERANGE))
					fail(t.line, t.col, "integer is out of range: " + t.text);
				t.kind = tok::NUMBER;
				t.ival = (int)n;
			}
			advance(q - p_);
			return t;
		}

		if (is_alpha(c) || ((c == '$' || c == '@') && is_alpha(c1)))
		{
			size_t q = p_ + ((c == '$' || c == '@') ? 1 : 0);
			while (q < s_.size() && is_idc(s_[q]))
				q++;
			t.text = s_.substr(p_, q - p_);
			advance(q - p_);
			if (c == '$')
			{
				t.kind = tok::VARIABLE;
				return t;
			}
			if (c == '@')
			{
				t.kind = tok::ALIAS;
				return t;
			}
			std::string low = t.text;
			std::transform(low.begin(), low.end(), low.begin(), ::tolower);
			if (low == "and")
				t.kind = tok::AND;
			else if (low == "or")
				t.kind = tok::OR;
			else if (low == "xor")
				t.kind = tok::XOR;
			else if (low == "not")
				t.kind = tok::NOT;
			else if (low == "true")
			{
				t.kind = tok::NUMBER;
				t.ival = 1;
			}
			else if (low == "false")
			{
				t.kind = tok::NUMBER;
				t.ival = 0;
			}
			else
				t.kind = tok::IDENT;
			return t;
		}

		auto two = [&](const char* op) { return c == op[0] && c1 == op[1]; };
		size_t len = 1;
		if (two("&&"))
			t.kind = tok::AND, len = 2;
		else if (two("||"))
			t.kind = tok::OR, len = 2;
		else if (two("=="))
			t.kind = tok::EQ, len = 2;
		else if (two("!="))
			t.kind = tok::NE, len = 2;
		else if (two("<="))
			t.kind = tok::LE, len = 2;
		else if (two(">="))
			t.kind = tok::GE, len = 2;
		else
		{
			switch (c)
			{
				case '-': t.kind = tok::MINUS; break;
				case '+': t.kind = tok::PLUS; break;
				case '*': t.kind = tok::STAR; break;
				case '/': t.kind = tok::SLASH; break;
				case '(': t.kind = tok::LPAREN; break;
				case ')': t.kind = tok::RPAREN; break;
				case '=': t.kind = tok::ASSIGN; break;
				case '?': t.kind = tok::TERNARY; break;
				case ':': t.kind = tok::COLON; break;
				case '&': t.kind = tok::AND; break;
				case '|': t.kind = tok::OR; break;
				case '^': t.kind = tok::XOR; break;
				case '!': t.kind = tok::NOT; break;
				case '<': t.kind = tok::LT; break;
				case '>': t.kind = tok::GT; break;
				case '{': t.kind = tok::LBRACE; break;
				case '}': t.kind = tok::RBRACE; break;
				case '.': t.kind = tok::DOT; break;
				case ';': t.kind = tok::SEMICOLON; break;
				case '[': t.kind = tok::LBRACKET; break;
				case ']': t.kind = tok::RBRACKET; break;
				case ',': t.kind = tok::COMMA; break;
				default: fail(t.line, t.col, std::string("invalid character: ") + c);
			}
		}
		t.text = s_.substr(p_, len);
		advance(len);
		return t;
	}
};

// ---------------------------------------------------------------- parser

expr_ptr make_literal(float v)
{
	auto e = std::make_shared<expr>();
	e->kind = expr::kind_t::literal;
	e->value = v;
	return e;
}

expr_ptr make_named(expr::kind_t k, std::string name)
{
	auto e = std::make_shared<expr>();
	e->kind = k;
	e->name = std::move(name);
	return e;
}

expr_ptr make_op(expr::kind_t k, op_t op, expr_ptr a, expr_ptr b = nullptr, expr_ptr c = nullptr)
{
	auto e = std::make_shared<expr>();
	e->kind = k;
	e->op = op;
	e->a = std::move(a);
	e->b = std::move(b);
	e->c = std::move(c);
	return e;
}

class parser
{
	lexer lex_;
	model_t& m_;
	token cur_;

	void shift() { cur_ = lex_.next(); }

	[[noreturn]] void unexpected(const char* expecting)
	{
		std::string msg = std::string("syntax error, unexpected ") + tok_name(cur_.kind);
		if (expecting)
			msg += std::string(", expecting ") + expecting;
		lex_.fail(cur_.line, cur_.col, msg);
	}

	token expect(tok k)
	{
		if (cur_.kind != k)
			unexpected(tok_name(k));
		token t = cur_;
		shift();
		return t;
	}

	// Wrap semantic errors thrown while evaluating with the location of the statement.
	template <typename F>
	void action(const token& at, F&& f)
	{
		try
		{
			f();
		}
		catch (const model_error&)
		{
			throw;
		}
		catch (const std::exception& e)
		{
			lex_.fail(at.line, at.col, e.what());
		}
	}

	// exp grammar, lowest precedence first
	expr_ptr parse_exp()
	{
		expr_ptr cond = parse_binary(0);
		if (cur_.kind == tok::TERNARY)
		{
			shift();
			expr_ptr mid = parse_exp();
			expect(tok::COLON);
			expr_ptr right = parse_exp();
			return make_op(expr::kind_t::ternary, op_t::PLUS, cond, mid, right);
		}
		return cond;
	}

	// binary precedence levels: 0 XOR, 1 OR, 2 AND, 3 EQ/NE, 4 relational, 5 additive, 6 multiplicative
	static int level_of(tok k, op_t& op)
	{
		switch (k)
		{
			case tok::XOR: op = op_t::XOR; return 0;
			case tok::OR: op = op_t::OR; return 1;
			case tok::AND: op = op_t::AND; return 2;
			case tok::EQ: op = op_t::EQ; return 3;
			case tok::NE: op = op_t::NE; return 3;
			case tok::LT: op = op_t::LT; return 4;
			case tok::LE: op = op_t::LE; return 4;
			case tok::GT: op = op_t::GT; return 4;
			case tok::GE: op = op_t::GE; return 4;
			case tok::PLUS: op = op_t::PLUS; return 5;
			case tok::MINUS: op = op_t::MINUS; return 5;
			case tok::STAR: op = op_t::STAR; return 6;
			case tok::SLASH: op = op_t::SLASH; return 6;
			default: return -1;
		}
	}

	expr_ptr parse_binary(int level)
	{
		if (level > 6)
			return parse_unary();
		expr_ptr left = parse_binary(level + 1);
		for (;;)
		{
			op_t op = op_t::PLUS;
			int l = level_of(cur_.kind, op);
			if (l != level)
				return left;
			shift();
			expr_ptr right = parse_binary(level + 1);
			left = make_op(expr::kind_t::binary, op, left, right);
		}
	}

	expr_ptr parse_unary()
	{
		switch (cur_.kind)
		{
			case tok::MINUS: shift(); return make_op(expr::kind_t::unary, op_t::MINUS, parse_unary());
			case tok::PLUS: shift(); return make_op(expr::kind_t::unary, op_t::PLUS, parse_unary());
			case tok::NOT: shift(); return make_op(expr::kind_t::unary, op_t::NOT, parse_unary());
			default: return parse_primary();
		}
	}

	expr_ptr parse_primary()
	{
		token t = cur_;
		switch (t.kind)
		{
			case tok::FLOAT: shift(); return make_literal(t.fval);
			case tok::NUMBER: shift(); return make_literal((float)t.ival);
			case tok::IDENT: shift(); return make_named(expr::kind_t::identifier, t.text);
			case tok::VARIABLE: shift(); return make_named(expr::kind_t::variable, t.text);
			case tok::ALIAS: shift(); return make_named(expr::kind_t::alias, t.text);
			case tok::LPAREN:
			{
				shift();
				expr_ptr inner = parse_exp();
				expect(tok::RPAREN);
				return make_op(expr::kind_t::paren, op_t::PLUS, inner);
			}
			default: unexpected("expression");
		}
	}

public:
	parser(const std::string& text, const std::string& file, model_t& m) : lex_(text, file), m_(m) { shift(); }

	void parse_bnd()
	{
		while (cur_.kind != tok::END)
		{
			token kw = expect(tok::IDENT);
			std::string low = kw.text;
			std::transform(low.begin(), low.end(), low.begin(), ::tolower);
			if (low != "node")
				lex_.fail(kw.line, kw.col, "expected 'node' keyword");
			token name = expect(tok::IDENT);
			expect(tok::LBRACE);
			std::vector<node_attr_t> attrs;
			do
			{
				token an = expect(tok::IDENT);
				expect(tok::ASSIGN);
				expr_ptr e = parse_exp();
				expect(tok::SEMICOLON);
				attrs.emplace_back(an.text, e);
			} while (cur_.kind == tok::IDENT);
			expect(tok::RBRACE);
			// driver::register_node (driver.cpp:50-63)
			node_t node;
			node.name = name.text;
			node.attrs = std::move(attrs);
			if (m_.node_index(node.name) >= 0)
				lex_.fail(name.line, name.col, "Node " + node.name + " already exists");
			if (!node.find_attr("rate_up"))
				lex_.fail(name.line, name.col, "Node " + node.name + " does not have rate_up attribute");
			if (!node.find_attr("rate_down"))
				lex_.fail(name.line, name.col, "Node " + node.name + " does not have rate_down attribute");
			m_.nodes.emplace_back(std::move(node));
		}
	}

	void parse_cfg()
	{
		while (cur_.kind != tok::END)
		{
			token first = cur_;
			if (first.kind == tok::VARIABLE)
			{
				// var_declaration (parser.yy:97) -> driver::register_variable (driver.cpp:45)
				shift();
				expect(tok::ASSIGN);
				expr_ptr e = parse_exp();
				expect(tok::SEMICOLON);
				action(first, [&] { m_.variables[first.text] = evaluate(m_, *e); });
			}
			else if (first.kind == tok::IDENT)
			{
				shift();
				if (cur_.kind == tok::DOT)
				{
					// attr_declaration (parser.yy:94) -> driver::register_node_attribute (driver.cpp:65-77)
					shift();
					token attr = expect(tok::IDENT);
					expect(tok::ASSIGN);
					expr_ptr e = parse_exp();
					expect(tok::SEMICOLON);
					int idx = m_.node_index(first.text);
					if (idx < 0)
						lex_.fail(first.line, first.col, "Unknown node " + first.text);
					if (attr.text == "istate")
						action(first, [&] { m_.nodes[idx].istate = evaluate(m_, *e); });
					else
						m_.nodes[idx].attrs.emplace_back(attr.text, e);
				}
				else
				{
					// const_declaration (parser.yy:100) -> driver::register_constant (driver.cpp:47)
					expect(tok::ASSIGN);
					expr_ptr e = parse_exp();
					expect(tok::SEMICOLON);
					action(first, [&] { m_.constants[first.text] = evaluate(m_, *e); });
				}
			}
			else if (first.kind == tok::LBRACKET)
			{
				// istate_declaration (parser.yy:102-108) -> driver::register_node_istate (driver.cpp:79-99).
				// The reference scanner never emits '[' ']' ','; this parser accepts the form.
				shift();
				token node = expect(tok::IDENT);
				expect(tok::RBRACKET);
				expect(tok::DOT);
				token kw = expect(tok::IDENT);
				if (kw.text != "istate")
					lex_.fail(kw.line, kw.col, "expected 'istate' keyword");
				expect(tok::ASSIGN);
				expr_ptr el = parse_exp();
				expect(tok::LBRACKET);
				token nl = expect(tok::NUMBER);
				expect(tok::RBRACKET);
				expect(tok::COMMA);
				expr_ptr er = parse_exp();
				expect(tok::LBRACKET);
				token nr = expect(tok::NUMBER);
				expect(tok::RBRACKET);
				expect(tok::SEMICOLON);
				if (!((nl.ival == 0 && nr.ival == 1) || (nl.ival == 1 && nr.ival == 0)))
					lex_.fail(nl.line, nl.col, "numbers in [] must be 0 and 1");
				int idx = m_.node_index(node.text);
				if (idx < 0)
					lex_.fail(node.line, node.col, "Unknown node " + node.text);
				action(first, [&] {
					float l = evaluate(m_, *el), r = evaluate(m_, *er);
					m_.nodes[idx].istate = nl.ival == 1 ? l / (l + r) : r / (l + r);
				});
			}
			else
				unexpected(nullptr);
		}
	}
};

std::string read_file(const std::string& path)
{
	std::ifstream in(path, std::ios::binary);
	if (!in)
		throw model_error("cannot open " + path);
	std::ostringstream ss;
	ss << in.rdbuf();
	return ss.str();
}

} // namespace

void parse_bnd(model_t& m, const std::string& text, const std::string& file)
{
	parser(text, file, m).parse_bnd();
}

void parse_cfg(model_t& m, const std::string& text, const std::string& file)
{
	parser(text, file, m).parse_cfg();
}

void parse_model_files(model_t& m, const std::string& bnd_path, const std::string& cfg_path)
{
	parse_bnd(m, read_file(bnd_path), bnd_path);
	parse_cfg(m, read_file(cfg_path), cfg_path);
}

// ---------------------------------------------------------------- evaluation

float evaluate(const model_t& m, const expr& e)
{
	using K = expr::kind_t;
	switch (e.kind)
	{
		case K::literal: return e.value;
		case K::identifier: throw model_error("identifier " + e.name + " in expression which needs to be evaluated");
		case K::alias: throw model_error("alias " + e.name + " in expression which needs to be evaluated");
		case K::variable:
		{
			auto it = m.variables.find(e.name);
			if (it == m.variables.end())
				throw model_error("unknown variable " + e.name);
			return it->second;
		}
		case K::paren: return evaluate(m, *e.a);
		case K::ternary: return evaluate(m, *e.a) ? evaluate(m, *e.b) : evaluate(m, *e.c);
		case K::unary:
			switch (e.op)
			{
				case op_t::PLUS: return evaluate(m, *e.a);
				case op_t::MINUS: return -evaluate(m, *e.a);
				case op_t::NOT: return !evaluate(m, *e.a);
				default: throw model_error("Unknown unary operator");
			}
		case K::binary:
		{
			switch (e.op)
			{
				case op_t::PLUS: return evaluate(m, *e.a) + evaluate(m, *e.b);
				case op_t::MINUS: return evaluate(m, *e.a) - evaluate(m, *e.b);
				case op_t::STAR: return evaluate(m, *e.a) * evaluate(m, *e.b);
				case op_t::SLASH: return evaluate(m, *e.a) / evaluate(m, *e.b);
				case op_t::AND: return evaluate(m, *e.a) && evaluate(m, *e.b);
				case op_t::OR: return evaluate(m, *e.a) || evaluate(m, *e.b);
				case op_t::XOR: return (evaluate(m, *e.a) != 0.f) != (evaluate(m, *e.b) != 0.f);
				case op_t::EQ: return evaluate(m, *e.a) == evaluate(m, *e.b);
				case op_t::NE: return evaluate(m, *e.a) != evaluate(m, *e.b);
				case op_t::LE: return evaluate(m, *e.a) <= evaluate(m, *e.b);
				case op_t::LT: return evaluate(m, *e.a) < evaluate(m, *e.b);
				case op_t::GE: return evaluate(m, *e.a) >= evaluate(m, *e.b);
				case op_t::GT: return evaluate(m, *e.a) > evaluate(m, *e.b);
				default: throw model_error("Unknown binary operator");
			}
		}
	}
	throw model_error("bad expression");
}

bool is_constant_expr(const model_t& m, const expr& e)
{
	using K = expr::kind_t;
	switch (e.kind)
	{
		case K::literal: return true;
		case K::variable: return m.variables.count(e.name) != 0;
		case K::identifier:
		case K::alias: return false;
		default:
			return (!e.a || is_constant_expr(m, *e.a)) && (!e.b || is_constant_expr(m, *e.b))
				   && (!e.c || is_constant_expr(m, *e.c));
	}
}

// ---------------------------------------------------------------- CUDA emission

void emit_code(const model_t& m, const expr& e, const std::string& current_node, std::ostream& os)
{
	using K = expr::kind_t;
	switch (e.kind)
	{
		case K::literal: os << print_float(e.value); return;
		case K::variable:
		{
			auto it = m.variables.find(e.name);
			if (it == m.variables.end())
				throw model_error("unknown variable " + e.name);
			os << print_float(it->second);
			return;
		}
		case K::identifier:
		{
			// expressions.cpp:194-205
			int i = m.node_index(e.name);
			if (i < 0)
				throw model_error("unknown node name: " + e.name);
			os << "((state[" << i / 32 << "] & " << (1u << (i % 32)) << "u) != 0)";
			return;
		}
		case K::alias:
		{
			// expressions.cpp:223-231: the current node's attribute named after the alias
			int i = m.node_index(current_node);
			if (i < 0)
				throw model_error("unknown node name: " + current_node);
			emit_code(m, m.nodes[i].get_attr(e.name.substr(1)), current_node, os);
			return;
		}
		case K::paren:
			os << "(";
			emit_code(m, *e.a, current_node, os);
			os << ")";
			return;
		case K::ternary:
			emit_code(m, *e.a, current_node, os);
			os << " ? ";
			emit_code(m, *e.b, current_node, os);
			os << " : ";
			emit_code(m, *e.c, current_node, os);
			return;
		case K::unary:
			switch (e.op)
			{
				case op_t::PLUS: os << "+"; break;
				case op_t::MINUS: os << "-"; break;
				case op_t::NOT: os << "!"; break;
				default: throw model_error("Unknown unary operator");
			}
			emit_code(m, *e.a, current_node, os);
			return;
		case K::binary:
		{
			const char* s = nullptr;
			switch (e.op)
			{
				case op_t::PLUS: s = " + "; break;
				case op_t::MINUS: s = " - "; break;
				case op_t::STAR: s = " * "; break;
				case op_t::SLASH: s = " / "; break;
				case op_t::AND: s = " & "; break;
				case op_t::OR: s = " | "; break;
				case op_t::XOR: s = " ^ "; break; // the reference throws here (no XOR case)
				case op_t::EQ: s = " == "; break;
				case op_t::NE: s = " != "; break;
				case op_t::LE: s = " <= "; break;
				case op_t::LT: s = " < "; break;
				case op_t::GE: s = " >= "; break;
				case op_t::GT: s = " > "; break;
				default: throw model_error("Unknown binary operator");
			}
			emit_code(m, *e.a, current_node, os);
			os << s;
			emit_code(m, *e.b, current_node, os);
			return;
		}
	}
}

} // namespace mb
