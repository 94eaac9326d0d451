// Multi-index helpers shared by the Taylor-expansion kernels (Laplace and
// Helmholtz): sumpy's coefficient orders (sumpy/expansion/__init__.py:643-752)
// and launch helpers.
#pragma once

#include <string>

#include "common.cuh"

namespace sumpy {

__device__ inline int nfull_of(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }

// f-th multi-index of the full set in sumpy's order (|mi|, mi0, mi1, mi2)
__device__ inline void full_mi(int f, int &i, int &j, int &k)
{
    int deg = 0;
    while ((deg + 1) * (deg + 2) * (deg + 3) / 6 <= f) ++deg;
    int r = f - deg * (deg + 1) * (deg + 2) / 6;
    i = 0;
    while (r >= deg - i + 1) { r -= deg - i + 1; ++i; }
    j = r;
    k = deg - i - j;
}

// s-th multi-index of the stored set (inverse of stored_index)
__device__ inline void stored_mi(int s, int &i, int &j, int &k)
{
    int deg = (int)sqrtf((float)s);
    while (deg * deg > s) --deg;
    while ((deg + 1) * (deg + 1) <= s) ++deg;
    int r = s - deg * deg;
    if (r <= deg) { i = 0; j = r; }
    else { i = 1; j = r - (deg + 1); }
    k = deg - i - j;
}

// t-th pair (J, K) with J + K <= m
__device__ inline void tri_pair(int t, int m, int &J, int &K)
{
    J = 0;
    while (t > m - J) { t -= m - J + 1; ++J; }
    K = t;
}

// Full coefficients of one box in the layout [(j, k) pairs, j-major][i]:
// the x-run of pair (j, k) holds i = 0..P-j-k contiguously.
// (closed form of: the pairs (j', k') before (j, k) times their run lengths)
template <int P>
__host__ __device__ constexpr int jki_offset(int j, int k)
{
    constexpr int A = P + 1;
    return A * (A + 1) * (A + 2) / 6 - (A - j) * (A - j + 1) * (A - j + 2) / 6 + k * (A - j) -
           k * (k - 1) / 2;
}

__device__ inline double ipow(double x, int n)
{
    double r = 1.0;
    for (int q = 0; q < n; ++q) r *= x;
    return r;
}

// Index of (i, j, k) in sumpy's full order (|mi|, mi0, mi1, mi2):
// tetra(deg) + sum_{i' < i} (deg - i' + 1) + j.
__device__ __forceinline__ int full_index(int i, int j, int k)
{
    const int deg = i + j + k;
    return deg * (deg + 1) * (deg + 2) / 6 + i * (deg + 1) - i * (i - 1) / 2 + j;
}

inline bool order_ok(int p) { return p >= 0 && p <= SUMPY_MAX_ORDER; }

template <typename K>
int prepare_smem(K kernel, size_t bytes)
{
    if (bytes > 227 * 1024) return bad_arg("shared memory request exceeds 227 KB");
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)bytes);
        if (e != cudaSuccess) {
            set_last_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
            return SUMPY_ELAUNCH;
        }
    }
    return SUMPY_OK;
}

}  // namespace sumpy

// dispatch a runtime order to a template instantiation CALL(P), P = 0..16
#define SUMPY_ORDER_SWITCH(p, CALL)                                                             \
    switch (p) {                                                                               \
    case 0: return CALL(0); case 1: return CALL(1); case 2: return CALL(2);                    \
    case 3: return CALL(3); case 4: return CALL(4); case 5: return CALL(5);                    \
    case 6: return CALL(6); case 7: return CALL(7); case 8: return CALL(8);                    \
    case 9: return CALL(9); case 10: return CALL(10); case 11: return CALL(11);                \
    case 12: return CALL(12); case 13: return CALL(13); case 14: return CALL(14);              \
    case 15: return CALL(15); case 16: return CALL(16);                                        \
    default: set_last_error("unsupported order"); return SUMPY_EUNSUPPORTED;                   \
    }

