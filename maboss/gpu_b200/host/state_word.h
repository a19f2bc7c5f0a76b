// state_word_t (src/state_word.h:3): one 32-bit word of a network state; node i is bit i % 32 of
// word i / 32.
#pragma once

#include <cstdint>

using state_word_t = uint32_t;
