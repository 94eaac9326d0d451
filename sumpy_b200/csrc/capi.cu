// Library-level entry points of the C-ABI (include/sumpy_b200.h).
#include <atomic>
#include <string>

#include "common.cuh"

namespace sumpy {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

static std::atomic<long long> g_wait_cycles{DEFAULT_WAIT_CYCLES};

long long wait_cycles_budget() { return g_wait_cycles.load(std::memory_order_relaxed); }

}  // namespace sumpy

extern "C" {

int sumpy_version(void) { return 1; }

const char *sumpy_last_error(void) { return sumpy::g_last_error.c_str(); }

int sumpy_set_tc_wait_cycles(int64_t cycles)
{
    sumpy::g_wait_cycles.store(cycles > 0 ? (long long)cycles : sumpy::DEFAULT_WAIT_CYCLES,
                               std::memory_order_relaxed);
    return SUMPY_OK;
}

int64_t sumpy_get_tc_wait_cycles(void)
{
    return sumpy::g_wait_cycles.load(std::memory_order_relaxed);
}

}  // extern "C"
