// Shared helpers for the sm_100a FMM kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/sumpy_b200.h"

namespace sumpy {

void set_last_error(const std::string &msg);

// Budget, in SM clock cycles (clock64), of every bounded wait in the
// kernels that wait (tensor-core barrier waits, level-chained GEMM steps);
// default 4e9 (~2 s), process-wide, set by sumpy_set_tc_wait_cycles.
constexpr long long DEFAULT_WAIT_CYCLES = 4000000000LL;
long long wait_cycles_budget();

inline int check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
        return SUMPY_ELAUNCH;
    }
    return SUMPY_OK;
}

inline int bad_arg(const char *msg)
{
    set_last_error(msg);
    return SUMPY_EINVAL;
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// stored index of multi-index (i, j, k), i in {0, 1}: degree-lexicographic
// order (|mi|, mi0, mi1, mi2) of the compressed Laplace set.
__host__ __device__ inline int stored_index(int i, int j, int k)
{
    int deg = i + j + k;
    return deg * deg + i * (deg + 1) + j;
}

__host__ __device__ inline int ncoeff_of(int p) { return (p + 1) * (p + 1); }

// dense cube index for full multi-indices of order <= p
__host__ __device__ inline int cube_index(int p, int i, int j, int k)
{
    return (i * (p + 1) + j) * (p + 1) + k;
}

}  // namespace sumpy
