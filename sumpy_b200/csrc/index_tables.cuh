// Compile-time index tables of the Taylor-expansion kernels (Laplace and
// Helmholtz): the P2M kernels' pair order and transposed-projection sweep,
// and the packed L2P kernels' decompression sweep, so that no kernel decodes
// multi-indices with loops at run time. Each table is a constexpr object per
// order P, placed in device memory and read through the read-only cache.
#pragma once

#include "taylor.cuh"

namespace sumpy {
namespace {

// a source's row of power-table entries in the P2M kernel: P + 1 rounded up
// to an even count, so that 16-byte loads read two powers at a time
__host__ __device__ constexpr int p2m_row(int p) { return (p + 2) & ~1; }

// The P2M kernels' transposed projection as tables, per order P: for the
// planes i = P..2 in turn, the entries F[i-2, J, K] -= F[i, J-2, K] +
// F[i, J, K-2] (+ kappa F[i, J, K] for Helmholtz) (J + K <= P - i + 2) as
// full-index quadruples {dst, a, b, c} (-1: term absent), and the full
// index of each stored coefficient.
__host__ __device__ constexpr int full_index_c(int i, int j, int k)
{
    return (i + j + k) * (i + j + k + 1) * (i + j + k + 2) / 6 + i * (i + j + k + 1) -
           i * (i - 1) / 2 + j;
}

template <int P>
struct alignas(16) P2mSweep {
    static constexpr int ne()
    {
        int n = 0;
        for (int i = P; i >= 2; --i) n += (P - i + 3) * (P - i + 4) / 2;
        return n;
    }
    static constexpr int NE = ne() > 0 ? ne() : 1;
    int e[4 * NE];
    int start[P + 2];
    int stored[(P + 1) * (P + 1)];
    constexpr P2mSweep() : e(), start(), stored()
    {
        int n = 0, pl = 0;
        for (int i = P; i >= 2; --i, ++pl) {
            start[pl] = n;
            const int m = P - i + 2;
            for (int J = 0; J <= m; ++J)
                for (int K = 0; J + K <= m; ++K) {
                    e[4 * n] = full_index_c(i - 2, J, K);
                    e[4 * n + 1] = J >= 2 ? full_index_c(i, J - 2, K) : -1;
                    e[4 * n + 2] = K >= 2 ? full_index_c(i, J, K - 2) : -1;
                    e[4 * n + 3] = J + K <= P - i ? full_index_c(i, J, K) : -1;
                    ++n;
                }
        }
        for (; pl < P + 2; ++pl) start[pl] = n;
        // stored coefficients: degree d = 0..P, (0, j, d - j) for j = 0..d,
        // then (1, j, d - 1 - j) for j = 0..d-1 (sumpy's order)
        int s = 0;
        for (int d = 0; d <= P; ++d) {
            for (int j = 0; j <= d; ++j) stored[s++] = full_index_c(0, j, d - j);
            for (int j = 0; j < d; ++j) stored[s++] = full_index_c(1, j, d - 1 - j);
        }
    }
};

template <int P>
__device__ constexpr P2mSweep<P> p2m_sweep{};

// (i, j) pair t of the P2M kernel, in increasing degree d = i + j (and
// increasing i within a degree): the pairs of row set u = t / 32 have
// column lengths P - d + 1 of at most p2m_kmax(u) + 1
__host__ __device__ constexpr int p2m_pair_degree(int t)
{
    int d = 0;
    while ((d + 1) * (d + 2) / 2 <= t) ++d;
    return d;
}

template <int P>
__host__ __device__ constexpr int p2m_kmax(int u)
{
    return P - p2m_pair_degree(32 * u);
}

// The packed L2P's decompression as tables, per order P, in the cube
// layout of jki_offset: for the planes i = 2..P in turn, the entries
// c[i, J, K] = -c[i-2, J+2, K] - c[i-2, J, K+2] (J + K <= P - i) as offset
// triples {dst, a, b, 0}, and the cube offset of each stored coefficient.
template <int P>
struct alignas(16) L2pDecomp {
    static constexpr int ne()
    {
        int n = 0;
        for (int i = 2; i <= P; ++i) n += (P - i + 1) * (P - i + 2) / 2;
        return n;
    }
    static constexpr int NE = ne() > 0 ? ne() : 1;
    int e[4 * NE];
    int start[P + 2];
    int stored[(P + 1) * (P + 1)];
    constexpr L2pDecomp() : e(), start(), stored()
    {
        int n = 0, pl = 0;
        for (int i = 2; i <= P; ++i, ++pl) {
            start[pl] = n;
            const int m = P - i;
            for (int J = 0; J <= m; ++J)
                for (int K = 0; J + K <= m; ++K) {
                    e[4 * n] = jki_offset<P>(J, K) + i;
                    e[4 * n + 1] = jki_offset<P>(J + 2, K) + i - 2;
                    e[4 * n + 2] = jki_offset<P>(J, K + 2) + i - 2;
                    e[4 * n + 3] = 0;
                    ++n;
                }
        }
        for (; pl < P + 2; ++pl) start[pl] = n;
        int s = 0;
        for (int d = 0; d <= P; ++d) {
            for (int j = 0; j <= d; ++j) stored[s++] = jki_offset<P>(j, d - j);
            for (int j = 0; j < d; ++j) stored[s++] = jki_offset<P>(j, d - 1 - j) + 1;
        }
    }
};

template <int P>
__device__ constexpr L2pDecomp<P> l2p_decomp{};

// Taylor shifts and the PDE decompression in the compact full-index
// layout (sumpy's order |mi|, mi0, mi1), per order P: for the planes
// i = 2..P in turn, {dst, a, b, c} with u_dst = -u_a - u_b - kappa u_c
// (dst = (i, J, K), a = (i-2, J+2, K), b = (i-2, J, K+2), c = (i-2, J, K));
// and for each axis d and full coefficient f = m, the full indices of
// m + q e_d, q = 0..P-|m|, at terms start[f] .. start[f + 1] - 1.
template <int P>
struct alignas(16) FullShift {
    static constexpr int NFULL = (P + 1) * (P + 2) * (P + 3) / 6;
    static constexpr int NT = (P + 1) * (P + 2) * (P + 3) * (P + 4) / 24;
    static constexpr int ne()
    {
        int n = 0;
        for (int i = 2; i <= P; ++i) n += (P - i + 1) * (P - i + 2) / 2;
        return n;
    }
    static constexpr int NE = ne() > 0 ? ne() : 1;
    int e[4 * NE];      // first member: read as int4
    int start[NFULL + 1];
    short idx[3][NT];
    int dstart[P + 2];
    unsigned char sdeg[(P + 1) * (P + 1)];   // degree of each stored coefficient
    constexpr FullShift() : e(), start(), idx(), dstart(), sdeg()
    {
        for (int d = 0, s = 0; d <= P; ++d)
            for (int r = 0; r < 2 * d + 1; ++r) sdeg[s++] = (unsigned char)d;
        int f = 0, t = 0;
        for (int deg = 0; deg <= P; ++deg)
            for (int i = 0; i <= deg; ++i)
                for (int j = 0; i + j <= deg; ++j, ++f) {
                    const int m[3] = {i, j, deg - i - j};
                    start[f] = t;
                    for (int q = 0; q <= P - deg; ++q, ++t)
                        for (int d = 0; d < 3; ++d) {
                            const int a = m[0] + (d == 0 ? q : 0);
                            const int b = m[1] + (d == 1 ? q : 0);
                            const int c = m[2] + (d == 2 ? q : 0);
                            idx[d][t] = (short)full_index_c(a, b, c);
                        }
                }
        start[NFULL] = t;
        int n = 0, pl = 0;
        for (int i = 2; i <= P; ++i, ++pl) {
            dstart[pl] = n;
            const int m = P - i;
            for (int J = 0; J <= m; ++J)
                for (int K = 0; J + K <= m; ++K, ++n) {
                    e[4 * n] = full_index_c(i, J, K);
                    e[4 * n + 1] = full_index_c(i - 2, J + 2, K);
                    e[4 * n + 2] = full_index_c(i - 2, J, K + 2);
                    e[4 * n + 3] = full_index_c(i - 2, J, K);
                }
        }
        for (; pl < P + 2; ++pl) dstart[pl] = n;
    }
};

template <int P>
__device__ constexpr FullShift<P> full_shift{};

}  // namespace
}  // namespace sumpy
