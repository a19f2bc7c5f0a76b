// Parser for the reference build (TEST INFRASTRUCTURE under oracle/, never part of the engine).
//
// The reference generates its scanner and parser with flex and bison from
// src/parser/scanner.ll and src/parser/parser.yy; neither tool is installed here. This file
// replaces those two generated files with a hand-written lexer and recursive-descent parser
// that accept the same language and perform the same semantic actions on the reference's own
// `driver` (src/parser/driver.cpp) and expression classes (src/parser/expressions.cpp):
//
//   tokens (scanner.ll:27-86): blanks and `//` comments skipped; `&&`, `&`, AND -> AND;
//     `||`, `|`, OR -> OR; `^`, XOR -> XOR; `!`, NOT -> NOT (keywords case-insensitive, whole
//     identifiers only, as flex's longest match gives); TRUE/FALSE -> NUMBER 1/0; integers
//     -> NUMBER (strtol, int range); fractions and exponents -> FLOAT ((float)strtod);
//     identifiers [a-zA-Z][a-zA-Z_0-9]*, `$id` -> VARIABLE, `@id` -> ALIAS (the sigil is kept
//     in the text); any other character is a syntax error ("invalid character").
//   grammar (parser.yy:69-162): a .cfg file is a list of `node.attr = exp;`, `$var = exp;`,
//     `const = exp;`; a .bnd file is a list of `node NAME { attr = exp; ... }` (the keyword
//     compared case-insensitively with "node"); expressions with the precedence, lowest first,
//     `?:` (right), XOR, OR, AND, `== !=`, `< <= > >=`, `+ -`, `* /`, unary `- + !` (all binary
//     operators left-associative). The `[X].istate = ...` rule needs `[ ] ,` tokens that the
//     reference's scanner never emits, so it is unreachable there and not accepted here either.
//   actions: driver::register_node / register_node_attribute / register_variable /
//     register_constant, in source order, with the reference's expression objects.
#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "driver.h"

namespace
{
enum class tok
{
	END,
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
	IDENTIFIER,
	VARIABLE,
	ALIAS,
	FLOAT,
	NUMBER
};

struct token
{
	tok kind = tok::END;
	std::string text;
	float fvalue = 0.f;
	int ivalue = 0;
	int line = 1, column = 1;
};

struct syntax_error : std::runtime_error
{
	int line, column;
	syntax_error(int l, int c, const std::string& m) : std::runtime_error(m), line(l), column(c) {}
};

bool ieq(const std::string& a, const char* b)
{
	size_t n = std::strlen(b);
	if (a.size() != n)
		return false;
	for (size_t i = 0; i < n; i++)
		if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i]))
			return false;
	return true;
}

bool is_alpha(char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z'); }
bool is_digit(char c) { return c >= '0' && c <= '9'; }
bool is_idchar(char c) { return is_alpha(c) || is_digit(c) || c == '_'; }

std::vector<token> lex(const std::string& s)
{
	std::vector<token> out;
	size_t i = 0;
	int line = 1, col = 1;
	auto advance = [&](size_t k) {
		for (size_t j = 0; j < k; j++, i++)
		{
			if (s[i] == '\n')
			{
				line++;
				col = 1;
			}
			else
				col++;
		}
	};
	while (i < s.size())
	{
		char c = s[i];
		if (c == ' ' || c == '\t' || c == '\r' || c == '\n')
		{
			advance(1);
			continue;
		}
		if (c == '/' && i + 1 < s.size() && s[i + 1] == '/')
		{
			while (i < s.size() && s[i] != '\n')
				advance(1);
			continue;
		}
		token t;
		t.line = line;
		t.column = col;
		// numbers: {int}, {fracconst}{exppart}?, [0-9]+{exppart} -- longest match
		if (is_digit(c) || (c == '.' && i + 1 < s.size() && is_digit(s[i + 1])))
		{
			size_t j = i;
			while (j < s.size() && is_digit(s[j]))
				j++;
			bool is_float = false;
			if (j < s.size() && s[j] == '.')
			{
				is_float = true;
				j++;
				while (j < s.size() && is_digit(s[j]))
					j++;
			}
			// exponent part only when complete ([eE][+-]?[0-9]+)
			if (j < s.size() && (s[j] == 'e' || s[j] == 'E'))
			{
				size_t k = j + 1;
				if (k < s.size() && (s[k] == '+' || s[k] == '-'))
					k++;
				if (k < s.size() && is_digit(s[k]))
				{
					while (k < s.size() && is_digit(s[k]))
						k++;
					j = k;
					is_float = true;
				}
			}
			t.text = s.substr(i, j - i);
			if (is_float)
			{
				errno = 0;
				double d = std::strtod(t.text.c_str(), nullptr);
				if (errno == ERANGE)
					throw syntax_error(t.line, t.column, "float is out of range: " + t.text);
				t.kind = tok::FLOAT;
				t.fvalue = (float)d;
			}
			else
			{
				errno = 0;
				long n = std::strtol(t.text.c_str(), nullptr, 10);
				if (!(INT_MIN <= n && n <= INT_MAX && errno != ERANGE))
					throw syntax_error(t.line, t.column, "integer is out of range: " + t.text);
				t.kind = tok::NUMBER;
				t.ivalue = (int)n;
			}
			advance(j - i);
			out.push_back(std::move(t));
			continue;
		}
		if (is_alpha(c) || ((c == '$' || c == '@') && i + 1 < s.size() && is_alpha(s[i + 1])))
		{
			size_t j = i + 1;
			while (j < s.size() && is_idchar(s[j]))
				j++;
			t.text = s.substr(i, j - i);
			if (c == '$')
				t.kind = tok::VARIABLE;
			else if (c == '@')
				t.kind = tok::ALIAS;
			else if (ieq(t.text, "AND"))
				t.kind = tok::AND;
			else if (ieq(t.text, "OR"))
				t.kind = tok::OR;
			else if (ieq(t.text, "XOR"))
				t.kind = tok::XOR;
			else if (ieq(t.text, "NOT"))
				t.kind = tok::NOT;
			else if (ieq(t.text, "TRUE") || ieq(t.text, "FALSE"))
			{
				t.kind = tok::NUMBER;
				t.ivalue = ieq(t.text, "TRUE") ? 1 : 0;
			}
			else
				t.kind = tok::IDENTIFIER;
			advance(j - i);
			out.push_back(std::move(t));
			continue;
		}
		auto two = [&](char a, char b) { return c == a && i + 1 < s.size() && s[i + 1] == b; };
		size_t len = 1;
		if (two('&', '&'))
			t.kind = tok::AND, len = 2;
		else if (two('|', '|'))
			t.kind = tok::OR, len = 2;
		else if (two('=', '='))
			t.kind = tok::EQ, len = 2;
		else if (two('!', '='))
			t.kind = tok::NE, len = 2;
		else if (two('<', '='))
			t.kind = tok::LE, len = 2;
		else if (two('>', '='))
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
				default: throw syntax_error(t.line, t.column, std::string("invalid character: ") + c);
			}
		}
		t.text = s.substr(i, len);
		advance(len);
		out.push_back(std::move(t));
	}
	token e;
	e.kind = tok::END;
	e.line = line;
	e.column = col;
	out.push_back(e);
	return out;
}

class rd_parser
{
	driver& drv_;
	std::vector<token> toks_;
	size_t p_ = 0;

	const token& peek() const { return toks_[p_]; }
	token take() { return toks_[p_++]; }
	[[noreturn]] void fail(const token& t, const std::string& what) const
	{
		throw syntax_error(t.line, t.column, what + " near '" + t.text + "'");
	}
	token expect(tok k, const char* what)
	{
		if (peek().kind != k)
			fail(peek(), std::string("syntax error, expected ") + what);
		return take();
	}

	// binary precedence, higher binds tighter (parser.yy:133-141); 0 = not a binary operator
	static int prec(tok k)
	{
		switch (k)
		{
			case tok::XOR: return 2;
			case tok::OR: return 3;
			case tok::AND: return 4;
			case tok::EQ:
			case tok::NE: return 5;
			case tok::LT:
			case tok::LE:
			case tok::GT:
			case tok::GE: return 6;
			case tok::PLUS:
			case tok::MINUS: return 7;
			case tok::STAR:
			case tok::SLASH: return 8;
			default: return 0;
		}
	}
	static operation op_of(tok k)
	{
		switch (k)
		{
			case tok::XOR: return operation::XOR;
			case tok::OR: return operation::OR;
			case tok::AND: return operation::AND;
			case tok::EQ: return operation::EQ;
			case tok::NE: return operation::NE;
			case tok::LT: return operation::LT;
			case tok::LE: return operation::LE;
			case tok::GT: return operation::GT;
			case tok::GE: return operation::GE;
			case tok::PLUS: return operation::PLUS;
			case tok::MINUS: return operation::MINUS;
			case tok::STAR: return operation::STAR;
			default: return operation::SLASH;
		}
	}

	expr_ptr unary()
	{
		const token& t = peek();
		switch (t.kind)
		{
			case tok::MINUS: take(); return std::make_unique<unary_expression>(operation::MINUS, unary());
			case tok::PLUS: take(); return std::make_unique<unary_expression>(operation::PLUS, unary());
			case tok::NOT: take(); return std::make_unique<unary_expression>(operation::NOT, unary());
			case tok::FLOAT: return std::make_unique<literal_expression>(take().fvalue);
			case tok::NUMBER: return std::make_unique<literal_expression>((float)take().ivalue);
			case tok::IDENTIFIER: return std::make_unique<identifier_expression>(take().text);
			case tok::VARIABLE: return std::make_unique<variable_expression>(take().text);
			case tok::ALIAS: return std::make_unique<alias_expression>(take().text);
			case tok::LPAREN:
			{
				take();
				auto e = exp();
				expect(tok::RPAREN, "')'");
				return std::make_unique<parenthesis_expression>(std::move(e));
			}
			default: fail(t, "syntax error, unexpected token in expression");
		}
	}

	// precedence climbing over the left-associative binary levels
	expr_ptr binary(int min_prec)
	{
		auto lhs = unary();
		while (true)
		{
			int p = prec(peek().kind);
			if (p == 0 || p < min_prec)
				return lhs;
			tok op = take().kind;
			auto rhs = binary(p + 1);
			lhs = std::make_unique<binary_expression>(op_of(op), std::move(lhs), std::move(rhs));
		}
	}

public:
	// exp: binary, optionally followed by `? exp : exp` (right-associative, lowest precedence)
	expr_ptr exp()
	{
		auto cond = binary(1);
		if (peek().kind != tok::TERNARY)
			return cond;
		take();
		auto mid = exp();
		expect(tok::COLON, "':'");
		auto right = exp();
		return std::make_unique<ternary_expression>(std::move(cond), std::move(mid), std::move(right));
	}

	rd_parser(driver& drv, std::vector<token> toks) : drv_(drv), toks_(std::move(toks)) {}

	void cfg_program()
	{
		while (peek().kind != tok::END)
		{
			const token& t = peek();
			if (t.kind == tok::VARIABLE)
			{
				std::string name = take().text;
				expect(tok::ASSIGN, "'='");
				auto e = exp();
				expect(tok::SEMICOLON, "';'");
				drv_.register_variable(std::move(name), std::move(e));
			}
			else if (t.kind == tok::IDENTIFIER)
			{
				std::string name = take().text;
				if (peek().kind == tok::DOT)
				{
					take();
					std::string attr = expect(tok::IDENTIFIER, "identifier").text;
					expect(tok::ASSIGN, "'='");
					auto e = exp();
					expect(tok::SEMICOLON, "';'");
					drv_.register_node_attribute(std::move(name), std::move(attr), std::move(e));
				}
				else
				{
					expect(tok::ASSIGN, "'='");
					auto e = exp();
					expect(tok::SEMICOLON, "';'");
					drv_.register_constant(std::move(name), std::move(e));
				}
			}
			else
				fail(t, "syntax error, unexpected token in .cfg declaration");
		}
	}

	void bnd_program()
	{
		while (peek().kind != tok::END)
		{
			token kw = expect(tok::IDENTIFIER, "'node'");
			std::string name = expect(tok::IDENTIFIER, "node name").text;
			expect(tok::LBRACE, "'{'");
			node_attr_list_t attrs;
			do
			{
				std::string attr = expect(tok::IDENTIFIER, "attribute name").text;
				expect(tok::ASSIGN, "'='");
				auto e = exp();
				expect(tok::SEMICOLON, "';'");
				attrs.emplace_back(std::move(attr), std::move(e));
			} while (peek().kind != tok::RBRACE);
			take();
			if (!ieq(kw.text, "node"))
				throw syntax_error(kw.line, kw.column, "expected 'node' keyword");
			drv_.register_node(std::move(name), std::move(attrs));
		}
	}
};
} // namespace

// The reference's scanner opens drv.file in scan_begin (scanner.ll:118-128) and closes it in
// scan_end; here the parser reads the whole file itself.
void driver::scan_begin()
{
	if (file.empty() || file == "-")
		return;
	std::ifstream probe(file);
	if (!probe)
	{
		std::cerr << "cannot open " << file << ": " << std::strerror(errno) << '\n';
		std::exit(EXIT_FAILURE);
	}
}

void driver::scan_end() {}

int yy::parser::operator()()
{
	std::stringstream ss;
	if (drv_.file.empty() || drv_.file == "-")
		ss << std::cin.rdbuf();
	else
	{
		std::ifstream in(drv_.file);
		ss << in.rdbuf();
	}
	auto start = drv_.start;
	drv_.start = driver::start_type::none;
	try
	{
		rd_parser p(drv_, lex(ss.str()));
		if (start == driver::start_type::cfg)
			p.cfg_program();
		else if (start == driver::start_type::bnd)
			p.bnd_program();
		else
			throw syntax_error(1, 1, "no start symbol");
	}
	catch (const syntax_error& e)
	{
		std::cerr << drv_.file << ":" << e.line << "." << e.column << ": " << e.what() << '\n';
		return 1;
	}
	return 0;
}
