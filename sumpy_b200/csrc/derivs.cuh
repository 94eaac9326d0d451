// Scaled Laplace derivatives rscale^|mi| d^mi (1/|x|) over the stored
// multi-index set (mi0 < 2) of order P, in registers.
//
// Same recurrence as LaplaceDerivativeTaker.diff (sumpy/derivative_taker.py:
// 211-262), evaluated degree by degree: degree-d entries need only the
// degree d-1 and d-2 entries, so three register "layers" of 2P+1 values
// suffice. With P a template parameter every loop unrolls and every index
// is a compile-time constant. Within a layer the entry e = i*(deg+1) + j is
// (i, j, deg-i-j); its stored index is deg^2 + e. visit(s, i, j, k, value)
// is called for every entry in stored order. T is the arithmetic type
// (double; float for the mixed-precision M2P/P2L, whose offsets are
// differences taken in FP64 and then rounded).
#pragma once

namespace sumpy {

__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }

template <int P, typename T = double, class Visit>
__device__ __forceinline__ void laplace_layers(T x, T y, T z, T R, T Rinv, Visit &&visit)
{
    const T r2 = x * x + y * y + z * z;
    const T rinv = rsqrt_t(r2);
    const T rinv2 = rinv * rinv;
    const T xs0 = x * Rinv, xs1 = y * Rinv, xs2 = z * Rinv;
    const T irs2 = R * R * rinv2;
    T L2[2 * P + 1], L1[2 * P + 1], L0[2 * P + 1];
#pragma unroll
    for (int e = 0; e < 2 * P + 1; ++e) L2[e] = L1[e] = L0[e] = T(0);
#pragma unroll
    for (int deg = 0; deg <= P; ++deg) {
#pragma unroll
        for (int e = 0; e < 2 * deg + 1; ++e) {
            const int i = (e <= deg) ? 0 : 1;
            const int j = (i == 0) ? e : e - (deg + 1);
            const int k = deg - i - j;
            T v;
            if (j <= 1 && k <= 1) {
                if (deg == 0) {
                    v = rinv;
                } else if (deg == 1) {
                    const T c = i ? x : (j ? y : z);
                    v = -R * c * rinv * rinv2;
                } else if (deg == 2) {
                    const T c1 = i ? x : y;
                    const T c2 = k ? z : y;
                    v = T(3) * R * R * c1 * c2 * rinv * rinv2 * rinv2;
                } else {
                    v = T(-15) * R * R * R * x * y * z * rinv * rinv2 * rinv2 * rinv2;
                }
            } else {
                // layer-local index of (ii, jj) on degree dd: ii*(dd+1) + jj
                T t = T(0);
                if (i == 1) t -= T(2) * xs0 * L1[j];  // (0, j, k) on deg-1
                if (j >= 1) {
                    const T t1 = L1[i * deg + (j - 1)];
                    const T t2 = (j >= 2) ? L2[i * (deg - 1) + (j - 2)] : T(0);
                    if (j >= 2) t -= T(2 * j - 1) * xs1 * t1 + T((j - 1) * (j - 1)) * t2;
                    else t -= T(2 * j) * xs1 * t1 + T(j * (j - 1)) * t2;
                }
                if (k >= 1) {
                    const T t1 = L1[i * deg + j];
                    const T t2 = (k >= 2) ? L2[i * (deg - 1) + j] : T(0);
                    if (j < 2) t -= T(2 * k - 1) * xs2 * t1 + T((k - 1) * (k - 1)) * t2;
                    else t -= T(2 * k) * xs2 * t1 + T(k * (k - 1)) * t2;
                }
                v = t * irs2;
            }
            L0[e] = v;
            visit(deg * deg + e, i, j, k, v);
        }
#pragma unroll
        for (int e = 0; e < 2 * P + 1; ++e) {
            L2[e] = L1[e];
            L1[e] = L0[e];
        }
    }
}

}  // namespace sumpy
