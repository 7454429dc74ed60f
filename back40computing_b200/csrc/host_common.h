// Host-side error reporting shared by every translation unit of libb40c_bfs.
//
// Mirrors b40c's B40CPerror (b40c/util/error_utils.cuh:44-103): a failing call
// returns its cudaError_t value and a "[file, line] message (CUDA error N: str)"
// text is kept; here the text goes to a thread-local buffer readable through
// b40c_last_error_string() and, when B40C_VERBOSE_ERRORS is set in the
// environment, to stderr as the reference does.
#pragma once

#include <cstdarg>
#include <cstdint>

namespace b40c_b200 {

int set_error(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();
const char *last_error();

}  // namespace b40c_b200
