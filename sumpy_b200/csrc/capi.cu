// Library-level entry points of the C-ABI (include/sumpy_b200.h).
#include <string>

#include "common.cuh"

namespace sumpy {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

}  // namespace sumpy

extern "C" {

int sumpy_version(void) { return 1; }

const char *sumpy_last_error(void) { return sumpy::g_last_error.c_str(); }

}  // extern "C"
