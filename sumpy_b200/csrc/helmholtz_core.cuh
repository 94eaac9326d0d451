// Device helpers shared by the Helmholtz kernels (helmholtz.cu,
// helmholtz_items.cu): complex arithmetic on interleaved (re, im) pairs and
// the derivatives D(mi) = rs^|mi| d^mi (e^{ikr}/r) of the stored
// multi-indices from the closed form of Tausch's recursion (the derivation
// is at the top of helmholtz.cu).
#pragma once

#include <utility>

#include "common.cuh"
#include "taylor.cuh"

namespace sumpy {
namespace {

using z2 = double2;

__device__ __forceinline__ z2 zmk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ z2 zadd(z2 a, z2 b) { return zmk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ z2 zscal(double s, z2 a) { return zmk(s * a.x, s * a.y); }
__device__ __forceinline__ z2 zmul(z2 a, z2 b)
{
    return zmk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// acc + s * a (s real)
__device__ __forceinline__ z2 zaxpy(double s, z2 a, z2 acc)
{
    return zmk(fma(s, a.x, acc.x), fma(s, a.y, acc.y));
}
// acc + a * b
__device__ __forceinline__ z2 zfma(z2 a, z2 b, z2 acc)
{
    return zmk(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}

// C[m][q] of the closed form above; m is one axis of a stored multi-index,
// so m <= SUMPY_MAX_ORDER.
constexpr int CM = SUMPY_MAX_ORDER + 1;
struct FaaTable {
    double v[CM][CM];
};
constexpr FaaTable make_faa_table()
{
    FaaTable t{};
    double f[CM] = {};
    f[0] = 1.0;
    for (int i = 1; i < CM; ++i) f[i] = f[i - 1] * i;
    for (int m = 0; m < CM; ++m)
        for (int q = 0; q < CM; ++q) {
            const int a = 2 * q - m, b = m - q;
            double v = 0.0;
            if (a >= 0 && b >= 0) {
                double p2 = 1.0;
                for (int i = 0; i < b; ++i) p2 *= 2.0;
                v = f[m] / (f[a] * f[b] * p2);
            }
            t.v[m][q] = v;
        }
    return t;
}

// stored index s -> (degree, i, j): s = d^2 + i (d + 1) + j
__host__ __device__ constexpr int stored_deg(int s)
{
    int d = 0;
    while ((d + 1) * (d + 1) <= s) ++d;
    return d;
}
__host__ __device__ constexpr int stored_i(int s) { return s - stored_deg(s) * stored_deg(s) <= stored_deg(s) ? 0 : 1; }
__host__ __device__ constexpr int stored_j(int s)
{
    return s - stored_deg(s) * stored_deg(s) - stored_i(s) * (stored_deg(s) + 1);
}

// Scaled form used by the kernels below: with v = x / rs and
// gt_Q = rs^(2Q) g_Q (= rho^(2Q) gamma_Q),
//     D(i, j, l) = sum_{q1, q2} C[j][q1] C[l][q2] v1^(2q1-j) v2^(2q2-l) v0^i gt_{q1+q2+i},
//     gt_0 = e^{ikr}/r, gt_1 = u (ikr - 1) gt_0,
//     gt_Q = -(2Q - 1) u gt_{Q-1} - (k rs)^2 u gt_{Q-2},  u = (rs/r)^2,
// so the live state per evaluation point is v and gt_0..P.
template <int P>
struct HelmTables {
    double v0, v1, v2, v1s, v2s;   // v, v1^2, v2^2
    double gr[P + 1], gi[P + 1];
};

// a * b that the compiler may neither merge with an identical product of
// another term nor move: keeps the per-axis factors out of the live
// register set (merged across all terms they would stay live and spill).
__device__ __forceinline__ double opaque_mul(double a, double b)
{
    double r;
    asm volatile("mul.rn.f64 %0, %1, %2;" : "=d"(r) : "d"(a), "d"(b));
    return r;
}

// The coefficients as compile-time constants (immediates in the code, which
// the compiler rematerialises instead of keeping loaded values live).
constexpr FaaTable kFaa = make_faa_table();

// one (q1, q2) product of a term: tr/ti += C[L][Q2] v2^(2 Q2 - L) gt_{Q1+Q2+I}
template <int P, int I, int L, int Q1, int Q2>
__device__ __forceinline__ void helm_q2(const HelmTables<P> &t, double &tr, double &ti, double &p2)
{
    constexpr double c = kFaa.v[L][Q2];
    const double a2 = c * p2;
    tr = fma(a2, t.gr[Q1 + Q2 + I], tr);
    ti = fma(a2, t.gi[Q1 + Q2 + I], ti);
    if constexpr (Q2 < L) p2 = opaque_mul(p2, t.v2s);
}

// the q1 = Q1 slice of a term: sr/si += C[J][Q1] v1^(2 Q1 - J) sum_q2 (...)
template <int P, int I, int J, int L, int Q1, int... K2>
__device__ __forceinline__ void helm_q1(const HelmTables<P> &t, double &sr, double &si, double &p1,
                                        std::integer_sequence<int, K2...>)
{
    double tr = 0.0, ti = 0.0;
    double p2 = opaque_mul((L & 1) ? t.v2 : 1.0, 1.0);
    (helm_q2<P, I, L, Q1, (L + 1) / 2 + K2>(t, tr, ti, p2), ...);
    constexpr double c = kFaa.v[J][Q1];
    const double a1 = c * p1;
    sr = fma(a1, tr, sr);
    si = fma(a1, ti, si);
    if constexpr (Q1 < J) p1 = opaque_mul(p1, t.v1s);
}

template <int P, int I, int J, int L, int... K1>
__device__ __forceinline__ z2 helm_term_impl(const HelmTables<P> &t,
                                             std::integer_sequence<int, K1...>)
{
    double sr = 0.0, si = 0.0;
    // running power v1^(2 q1 - J) (and v2^(2 q2 - L) in helm_q1), produced
    // by opaque products so that no power is shared across terms
    double p1 = opaque_mul((J & 1) ? t.v1 : 1.0, 1.0);
    (helm_q1<P, I, J, L, (J + 1) / 2 + K1>(t, sr, si, p1,
                                            std::make_integer_sequence<int, L / 2 + 1>{}),
     ...);
    return I ? zmk(t.v0 * sr, t.v0 * si) : zmk(sr, si);
}

// D of the stored coefficient S (compile-time), from the tables
template <int P, int S>
__device__ __forceinline__ z2 helm_term(const HelmTables<P> &t)
{
    constexpr int d = stored_deg(S), i = stored_i(S), j = stored_j(S), l = d - i - j;
    return helm_term_impl<P, i, j, l>(t, std::make_integer_sequence<int, j / 2 + 1>{});
}

// the terms of one degree D (stored indices D^2 .. (D+1)^2 - 1)
template <int P, int S, typename F>
__device__ __forceinline__ void helm_step(const HelmTables<P> &t, F &f)
{
    f(std::integral_constant<int, S>{}, helm_term<P, S>(t));
    // ordered after the term's own volatile products: the next term starts
    // only once this one has been consumed (f fences its registers too)
    asm volatile("" ::: "memory");
}

template <int P, int D, typename F, int... R>
__device__ __forceinline__ void helm_degree(const HelmTables<P> &t, F &f,
                                            std::integer_sequence<int, R...>)
{
    (helm_step<P, D * D + R>(t, f), ...);
}

// run degree d (a runtime value) with the degree-D code: each degree is its
// own block, so the scheduler never interleaves more than one degree's
// 2D + 1 terms (all (P+1)^2 at once would not fit in registers)
template <int P, typename F, int... D>
__device__ __forceinline__ void helm_dispatch(int d, const HelmTables<P> &t, F &f,
                                              std::integer_sequence<int, D...>)
{
    ((d == D ? helm_degree<P, D>(t, f, std::make_integer_sequence<int, 2 * D + 1>{})
             : void()),
     ...);
}

// D(mi) = rs^|mi| d^mi (e^{ikr}/r) at x for every stored mi of order <= P,
// in stored order s = 0, 1, ..., (P+1)^2 - 1: f(std::integral_constant<int, s>, D).
template <int P, typename F>
__device__ __forceinline__ void helm_layers(double x0, double x1, double x2, double rs, double k,
                                            F &&f)
{
    HelmTables<P> t;
    const double r2 = x0 * x0 + x1 * x1 + x2 * x2;
    const double ri = rsqrt(r2);
    const double r = r2 * ri;
    const double rsi = 1.0 / rs;
    t.v0 = x0 * rsi;
    t.v1 = x1 * rsi;
    t.v2 = x2 * rsi;
    t.v1s = t.v1 * t.v1;
    t.v2s = t.v2 * t.v2;
    const double u = rs * rs * ri * ri;
    double sn, cs;
    sincos(k * r, &sn, &cs);
    t.gr[0] = cs * ri;
    t.gi[0] = sn * ri;
    if constexpr (P >= 1) {
        const double kr = k * r;
        t.gr[1] = u * (-t.gr[0] - kr * t.gi[0]);
        t.gi[1] = u * (-t.gi[0] + kr * t.gr[0]);
        const double ku = (k * rs) * (k * rs) * u;
#pragma unroll
        for (int q = 2; q <= P; ++q) {
            t.gr[q] = -(2.0 * q - 1.0) * u * t.gr[q - 1] - ku * t.gr[q - 2];
            t.gi[q] = -(2.0 * q - 1.0) * u * t.gi[q - 1] - ku * t.gi[q - 2];
        }
    }
#pragma unroll 1
    for (int d = 0; d <= P; ++d)
        helm_dispatch<P>(d, t, f, std::make_integer_sequence<int, P + 1>{});
}

// read-only 16-byte load of p[S], kept in program order and addressed with
// an immediate offset (plain loads of the multipole would be hoisted above
// all terms, with one live address each)
template <int S>
__device__ __forceinline__ z2 ordered_load(const z2 *p)
{
    z2 v;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2+%3];"
                 : "=d"(v.x), "=d"(v.y)
                 : "l"(p), "n"(S * 16));
    return v;
}

}  // namespace
}  // namespace sumpy
