// Stand-in for the bison-generated "generated/parser.h" that the reference's
// src/parser/driver.h includes (the reference generates it from src/parser/parser.yy with
// bison; flex and bison are not installed here).
//
// TEST INFRASTRUCTURE: part of the reference build under oracle/ (the checker), never part of
// the engine. It declares only what the reference's own driver.cpp uses:
//   * yy::location with initialize(std::string*)            (driver.cpp: parse_one)
//   * yy::parser(driver&), set_debug_level(), operator()()   (driver.cpp: parse_one)
//   * yy::parser::symbol_type, named by the YY_DECL declaration in driver.h (never called here)
// The parser itself is the hand-written recursive-descent parser in ../parser_shim.cpp, which
// accepts the grammar of src/parser/parser.yy with the tokens of src/parser/scanner.ll and
// performs the same semantic actions (driver::register_*).
#pragma once

// The bison header pulls these in, and the reference's parser sources rely on them
// (expressions.cpp uses std::ostream and assert without including them).
#include <cassert>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "parse_types.h"

class driver;

namespace yy
{
class location
{
public:
	std::string* file = nullptr;
	int line = 1;
	int column = 1;

	void initialize(std::string* f = nullptr, int l = 1, int c = 1)
	{
		file = f;
		line = l;
		column = c;
	}
};

class parser
{
public:
	// Only named by the yylex declaration in driver.h; no scanner function exists in this build.
	struct symbol_type;
	using location_type = location;

	explicit parser(driver& drv) : drv_(drv) {}

	void set_debug_level(int) {}

	// Parses drv.file as a .bnd or .cfg file according to drv.start; 0 on success, 1 on a
	// syntax error (reported on stderr as "file:line.column: message"). Exceptions thrown by
	// the driver's semantic actions (unknown node, duplicate node, ...) propagate, as they do
	// out of the bison parser.
	int operator()();
	int parse() { return (*this)(); }

private:
	driver& drv_;
};
} // namespace yy
