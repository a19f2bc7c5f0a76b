// driver (src/parser/driver.h:14-56): parses a .bnd and a .cfg file. The grammar and the model are
// held behind the C ABI (mb_model); the driver exposes the reference's public data members, filled
// after parse(). Expression trees are not exposed (node_t has no attrs).
#pragma once

#include <map>
#include <string>
#include <vector>

#include "maboss_b200.h"

class driver;

// node_t (src/parser/parse_types.h:16-29) without its attribute expressions.
struct node_t
{
	std::string name;
	float istate = 0.5f;
	bool internal = false;

	bool is_internal(const driver&) const { return internal; }
};

class driver
{
public:
	driver();
	~driver();
	driver(const driver&) = delete;
	driver& operator=(const driver&) = delete;

	std::string file; // the file being parsed (for messages)

	std::map<std::string, float> variables;
	std::map<std::string, float> constants;
	std::vector<node_t> nodes;

	// Returns 0 on success; otherwise prints the error to std::cerr and returns 1 (the reference
	// returns the bison parser's result and throws std::runtime_error on semantic errors). The
	// public members are replaced by the parsed model's.
	int parse(std::string bnd_file, std::string cfg_file);

	// The parsed model with the public members written back (variables, constants, istate).
	mb_model model();

	// Opt-in (no counterpart in the reference): node attributes defined again in the .cfg replace
	// the .bnd's (mb_model_apply_cfg_overrides); the reference keeps the first definition.
	void apply_cfg_overrides();

private:
	mb_model model_ = nullptr;
	void load_members();
};
