// trajectory_status (src/trajectory_status.h:3-8): one byte per trajectory after an epoch.
#pragma once

#include <cstdint>

enum class trajectory_status : uint8_t
{
	CONTINUE,
	FINISHED,
	FIXED_POINT
};
