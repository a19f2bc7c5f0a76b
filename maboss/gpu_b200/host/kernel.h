// kernel_wrapper (src/kernel.h:5-23): one named entry point of a compiled model. The reference
// launches its CUfunction with cuLaunchKernel on stream 0 and caller-chosen grid sizes; here the
// launches go through the C ABI (mb_launch_*), which chooses the grid for the B200, takes SoA
// buffers and the context's stream, and reports errors as status codes.
#pragma once

#include "maboss_b200.h"

struct kernel_wrapper
{
	mb_module module = nullptr;
	const char* name = "";
};
