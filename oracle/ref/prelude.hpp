// Test infrastructure only: force-included (g++ -include) in front of every
// reference translation unit that the oracle recipe compiles in place.
//
// The reference draws all of its random numbers from one inline function,
// get_random_float() (global.hpp:35-50): a thread_local SplitMix64 whose state
// is seeded from std::random_device, so no two runs agree. For parity runs the
// oracle needs every path to consume a known stream. This prelude renames the
// reference's definition while global.hpp is parsed once, then declares a
// replacement with the same signature that the harness defines. Because
// global.hpp is `#pragma once`, later `#include "global.hpp"` lines in the
// reference sources are skipped and every call site binds to the replacement.
#pragma once
#define get_random_float get_random_float__reference_splitmix
#include "global.hpp"
#undef get_random_float

#include <cstdint>

// Defined in harness.cpp: SplitMix64 over a thread-local state that the
// harness sets per path with prr_ref_rng_set_path().
float get_random_float();
