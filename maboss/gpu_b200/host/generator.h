// generator (src/generator.h:7-23): CUDA source of a parsed model (rate functions, transition
// entropy, non-internal index and the engine's model tables), from the C ABI's code generator.
#pragma once

#include <string>

#include "parser/driver.h"

class generator
{
	driver& drv_;

public:
	explicit generator(driver& drv);

	// Writes the driver's variables, constants and initial states back into the model first, so
	// that edits of drv.variables / drv.constants / node_t::istate are generated (as the reference,
	// which reads them while generating).
	std::string generate_code() const;
};
