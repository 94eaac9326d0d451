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

// The same recurrence for two evaluation points at once on packed FP32
// pairs (sm_100 FADD2 / FMUL2 / FFMA2: one instruction for both points),
// written with explicit fused multiply-adds: visit(s, i, j, k, value) with
// value.x for the first point and value.y for the second. Same terms as
// laplace_layers<P, float>, summed in the same order; each subtraction
// t -= c1 x t1 + c2 t2 is taken as two fused steps, so results may differ
// from the scalar form in the last bits.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

template <int P, class Visit>
__device__ __forceinline__ void laplace_layers_x2(float2 x, float2 y, float2 z, float R,
                                                  float Rinv, Visit &&visit)
{
    const float2 r2 = __ffma2_rn(x, x, __ffma2_rn(y, y, __fmul2_rn(z, z)));
    const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    const float2 rinv2 = __fmul2_rn(rinv, rinv);
    const float2 xs0 = __fmul2_rn(x, f2(Rinv)), xs1 = __fmul2_rn(y, f2(Rinv));
    const float2 xs2 = __fmul2_rn(z, f2(Rinv));
    const float2 irs2 = __fmul2_rn(f2(R * R), rinv2);
    float2 L2[2 * P + 1], L1[2 * P + 1], L0[2 * P + 1];
#pragma unroll
    for (int e = 0; e < 2 * P + 1; ++e) L2[e] = L1[e] = L0[e] = f2(0.f);
#pragma unroll
    for (int deg = 0; deg <= P; ++deg) {
#pragma unroll
        for (int e = 0; e < 2 * deg + 1; ++e) {
            const int i = (e <= deg) ? 0 : 1;
            const int j = (i == 0) ? e : e - (deg + 1);
            const int k = deg - i - j;
            float2 v;
            if (j <= 1 && k <= 1) {
                if (deg == 0) {
                    v = rinv;
                } else if (deg == 1) {
                    const float2 c = i ? x : (j ? y : z);
                    v = __fmul2_rn(__fmul2_rn(__fmul2_rn(f2(-R), c), rinv), rinv2);
                } else if (deg == 2) {
                    const float2 c1 = i ? x : y;
                    const float2 c2 = k ? z : y;
                    v = __fmul2_rn(__fmul2_rn(__fmul2_rn(__fmul2_rn(f2(3.f * R * R), c1), c2),
                                              __fmul2_rn(rinv, rinv2)),
                                   rinv2);
                } else {
                    v = __fmul2_rn(
                        __fmul2_rn(__fmul2_rn(__fmul2_rn(f2(-15.f * R * R * R), x), y), z),
                        __fmul2_rn(__fmul2_rn(rinv, rinv2), __fmul2_rn(rinv2, rinv2)));
                }
            } else {
                float2 t = f2(0.f);
                if (i == 1) t = __ffma2_rn(__fmul2_rn(f2(-2.f), xs0), L1[j], t);
                if (j >= 1) {
                    const float2 t1 = L1[i * deg + (j - 1)];
                    if (j >= 2) {
                        const float2 t2 = L2[i * (deg - 1) + (j - 2)];
                        t = __ffma2_rn(__fmul2_rn(f2(-(float)(2 * j - 1)), xs1), t1, t);
                        t = __ffma2_rn(f2(-(float)((j - 1) * (j - 1))), t2, t);
                    } else {
                        t = __ffma2_rn(__fmul2_rn(f2(-(float)(2 * j)), xs1), t1, t);
                    }
                }
                if (k >= 1) {
                    const float2 t1 = L1[i * deg + j];
                    const float ck = j < 2 ? (float)(2 * k - 1) : (float)(2 * k);
                    const float dk = j < 2 ? (float)((k - 1) * (k - 1)) : (float)(k * (k - 1));
                    t = __ffma2_rn(__fmul2_rn(f2(-ck), xs2), t1, t);
                    if (k >= 2) t = __ffma2_rn(f2(-dk), L2[i * (deg - 1) + j], t);
                }
                v = __fmul2_rn(t, irs2);
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
