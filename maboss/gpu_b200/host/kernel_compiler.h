// kernel_compiler (src/kernel_compiler.h:8-20): a CUDA context on a device and the module compiled
// from generated code. The reference creates a private context on device 0 and exits the process on
// CUDA errors; this one binds the device's primary context and throws std::runtime_error.
#pragma once

#include <string>

#include "kernel.h"

class kernel_compiler
{
	mb_context context_ = nullptr;
	mb_module module_ = nullptr;

public:
	kernel_wrapper initialize_random, initialize_initial_state, simulate, window_average_small, final_states;

	kernel_compiler();
	explicit kernel_compiler(int device);
	~kernel_compiler();
	kernel_compiler(const kernel_compiler&) = delete;
	kernel_compiler& operator=(const kernel_compiler&) = delete;

	// NVRTC compilation for sm_100a (src/kernel_compiler.cpp:61-164): 0 on success, 1 on a
	// compilation failure, whose log goes to std::cerr. `discrete_time` is part of the generated
	// code here; the argument is kept for the reference's signature.
	int compile_simulation(const std::string& code, bool discrete_time);

	mb_context context() const { return context_; }
	mb_module module() const { return module_; }
};
