#include "driver.h"

#include <iostream>

#include "../maboss_b200_mirror.h"
#include "../timer.h"

namespace {

template <typename F>
std::string read_name(F&& get)
{
	size_t len = 0;
	mirror::check(get(nullptr, 0, &len), "driver");
	std::string s(len + 1, '\0');
	mirror::check(get(s.data(), s.size(), &len), "driver");
	s.resize(len);
	return s;
}

} // namespace

driver::driver()
{
	// defaults of src/parser/driver.cpp:7-14
	constants["discrete_time"] = 0;
	constants["sample_count"] = 1'000'000;
	constants["max_time"] = 10;
	constants["time_tick"] = 0.1f;
	constants["seed_pseudorandom"] = 0;
}

driver::~driver()
{
	if (model_)
		mb_model_free(model_);
}

int driver::parse(std::string bnd_file, std::string cfg_file)
{
	timer_stats t("parser> parse");
	file = bnd_file;
	mb_model m = nullptr;
	if (mb_model_parse_files(bnd_file.c_str(), cfg_file.c_str(), &m) != MB_OK)
	{
		std::cerr << mb_last_error() << std::endl;
		return 1;
	}
	if (model_)
		mb_model_free(model_);
	model_ = m;
	file = cfg_file;
	load_members();
	return 0;
}

void driver::load_members()
{
	int n = 0;
	mirror::check(mb_model_num_nodes(model_, &n), "driver");
	nodes.clear();
	for (int i = 0; i < n; i++)
	{
		node_t node;
		node.name = read_name([&](char* b, size_t c, size_t* l) { return mb_model_node_name(model_, i, b, c, l); });
		int internal = 0;
		mirror::check(mb_model_node_info(model_, i, &node.istate, &internal), "driver");
		node.internal = internal != 0;
		nodes.push_back(std::move(node));
	}
	variables.clear();
	mirror::check(mb_model_num_variables(model_, &n), "driver");
	for (int i = 0; i < n; i++)
	{
		auto name = read_name([&](char* b, size_t c, size_t* l) { return mb_model_variable_name(model_, i, b, c, l); });
		mirror::check(mb_model_get_variable(model_, name.c_str(), &variables[name]), "driver");
	}
	constants.clear();
	mirror::check(mb_model_num_constants(model_, &n), "driver");
	for (int i = 0; i < n; i++)
	{
		auto name = read_name([&](char* b, size_t c, size_t* l) { return mb_model_constant_name(model_, i, b, c, l); });
		mirror::check(mb_model_get_constant(model_, name.c_str(), &constants[name]), "driver");
	}
}

mb_model driver::model()
{
	if (!model_)
		throw std::runtime_error("driver: no model has been parsed");
	for (auto& [name, value] : variables)
		mirror::check(mb_model_set_variable(model_, name.c_str(), value), "driver variables");
	for (auto& [name, value] : constants)
		mirror::check(mb_model_set_constant(model_, name.c_str(), value), "driver constants");
	for (size_t i = 0; i < nodes.size(); i++)
		mirror::check(mb_model_set_istate(model_, (int)i, nodes[i].istate), "driver nodes");
	return model_;
}

void driver::apply_cfg_overrides()
{
	if (!model_)
		throw std::runtime_error("driver: no model has been parsed");
	mirror::check(mb_model_apply_cfg_overrides(model_), "driver");
	load_members(); // is_internal may have changed
}
