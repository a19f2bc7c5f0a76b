// Model front-end: .bnd/.cfg parsing, constant evaluation and per-node code emission.
//
// Mirrors the semantics of the reference front-end (src/parser/driver.{h,cpp},
// src/parser/expressions.{h,cpp}, src/parser/parse_types.{h,cpp}, grammar in
// src/parser/parser.yy and tokens in src/parser/scanner.ll) with a hand-written
// recursive-descent parser, because the reference's flex/bison toolchain is not a
// dependency of this library.
#pragma once

#include <map>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mb {

// Error raised for malformed input or semantic errors; `what()` is "file:line.col: message"
// like the reference's bison error reporter (parser.yy:161-165).
struct model_error : std::runtime_error
{
	explicit model_error(const std::string& m) : std::runtime_error(m) {}
};

// Operators of the expression language (expressions.h:11-27).
enum class op_t
{
	PLUS,
	MINUS,
	STAR,
	SLASH,
	AND,
	OR,
	XOR,
	NOT,
	LE,
	LT,
	GE,
	GT,
	EQ,
	NE
};

struct expr;
using expr_ptr = std::shared_ptr<const expr>;

// Expression tree node (expressions.h:37-120 has one class per kind).
struct expr
{
	enum class kind_t
	{
		literal,
		identifier,
		variable,
		alias,
		unary,
		binary,
		ternary,
		paren
	};
	kind_t kind = kind_t::literal;
	float value = 0.f; // literal: stored as float like literal_expression (expressions.h:82-90)
	std::string name;  // identifier, "$var" (with '$'), "@alias" (with '@')
	op_t op = op_t::PLUS;
	expr_ptr a, b, c;
};

using node_attr_t = std::pair<std::string, expr_ptr>;

// One Boolean node (parse_types.h:16-29). Attributes keep declaration order and the
// FIRST attribute of a given name wins on lookup (parse_types.cpp:6-13).
struct node_t
{
	std::string name;
	std::vector<node_attr_t> attrs;
	float istate = 0.5f; // parse_types.cpp:3

	const expr* find_attr(const std::string& attr) const;
	const expr& get_attr(const std::string& attr) const; // throws like parse_types.cpp:11
};

// The parsed model: the reference's `driver` fields (driver.h:39-43).
struct model_t
{
	std::map<std::string, float> variables;
	std::map<std::string, float> constants;
	std::vector<node_t> nodes;

	model_t(); // constant defaults as in driver.cpp:7-14

	int node_index(const std::string& name) const; // -1 if absent
	bool is_internal(size_t i) const;				// parse_types.cpp:20-23
	float constant(const std::string& name) const;	// 0 when missing (std::map operator[] in main.cpp)
	int noninternal_count() const;
};

// Parse the .bnd text then the .cfg text (driver.cpp:16-31). `file` names are only
// used in error messages.
void parse_bnd(model_t& m, const std::string& text, const std::string& file);
void parse_cfg(model_t& m, const std::string& text, const std::string& file);
void parse_model_files(model_t& m, const std::string& bnd_path, const std::string& cfg_path);

// Opt-in: every node attribute defined more than once (in the .bnd and again in the .cfg, say) takes
// its last definition, at the position of its first. The reference keeps the first one
// (driver.cpp:65-77 appends a .cfg attribute, parse_types.cpp:6-13 returns the first match), so a
// .cfg cannot change a rate or a logic defined in the .bnd; MaBoSS users expect the .cfg to win.
void apply_cfg_overrides(model_t& m);

// Float evaluation used for $variables, constants, istate and is_internal
// (expressions.cpp: every `evaluate` method).
float evaluate(const model_t& m, const expr& e);

// True when `e` can be evaluated without touching node state (no identifier/alias).
bool is_constant_expr(const model_t& m, const expr& e);

// CUDA source emission for an expression (expressions.cpp: every `generate_code`).
// Literals and $variables are printed with the default ostream precision (6 significant
// digits), which decides the C++ type (int vs double literal) of the emitted text.
void emit_code(const model_t& m, const expr& e, const std::string& current_node, std::ostream& os);

// `std::ostream << float` with default flags and precision 6.
std::string print_float(float v);

} // namespace mb
