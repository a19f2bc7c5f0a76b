#include "kernel_compiler.h"

#include <iostream>

#include "maboss_b200_mirror.h"
#include "timer.h"

kernel_compiler::kernel_compiler() : kernel_compiler(0) {}

kernel_compiler::kernel_compiler(int device)
{
	timer_stats t("kernel_compiler> context");
	mirror::check(mb_context_create(device, &context_), "kernel_compiler");
}

kernel_compiler::~kernel_compiler()
{
	if (module_)
		mb_module_free(module_);
	if (context_)
		mb_context_free(context_);
}

int kernel_compiler::compile_simulation(const std::string& code, bool)
{
	timer_stats t("kernel_compiler> compile_simulation");
	mb_module m = nullptr;
	const mb_status s = mb_module_compile(context_, code.c_str(), &m);
	if (s == MB_ERR_COMPILE)
	{
		std::cerr << mb_last_error() << std::endl;
		return 1;
	}
	mirror::check(s, "compile_simulation");
	if (module_)
		mb_module_free(module_);
	module_ = m;
	initialize_random = { module_, "initialize_random" };
	initialize_initial_state = { module_, "initialize_initial_state" };
	simulate = { module_, "simulate" };
	window_average_small = { module_, "window_average_small" };
	final_states = { module_, "final_states" };
	return 0;
}
