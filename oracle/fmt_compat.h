/* Compatibility shim for building the reference app against fmt 12 (the only fmt on this image):
   fmt 12 removed fmt::localtime, which the reference app calls once to timestamp its result file.
   TEST INFRASTRUCTURE ONLY (used by oracle/Makefile). */
#pragma once
#ifdef __cplusplus
#include <ctime>
#include <fmt/chrono.h>
namespace fmt {
inline std::tm localtime(std::time_t t) { std::tm r{}; localtime_r(&t, &r); return r; }
}
#endif
