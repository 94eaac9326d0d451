// P2M, P2L, M2M, L2L, L2P and M2P for the compressed 3D Laplace Taylor
// expansions (sumpy's LinearPDEConformingVolumeTaylor{Multipole,Local}
// Expansion; stored set mi0 < 2, sumpy/expansion/__init__.py:563-886).
//
// Full coefficient sets live in shared memory as dense cubes
// [i][j][k] (i + j + k <= p). The Laplace projection between stored and
// full sets (u_mi = -u_{mi-2e0+2e1} - u_{mi-2e0+2e2}) runs as p-1 parallel
// sweeps over the mi0 planes:
//   decompress (local -> full, CSEMatVecOperator.matvec,
//     __init__.py:510-531):           plane i from plane i-2, i = 2..p
//   compress (full multipole -> stored, transpose_matvec, __init__.py:533-548):
//                                     plane i-2 gathers from plane i, i = p..2
//
// Derivatives of 1/r (P2L, M2P) use LaplaceDerivativeTaker's recurrence
// (sumpy/derivative_taker.py:211-262) restricted to the stored set, which is
// closed under it (mi0 never grows).
#include <algorithm>

#include "common.cuh"
#include "derivs.cuh"
#include "taylor.cuh"
#include "index_tables.cuh"

namespace sumpy {
namespace {

// same, one warp
__device__ void decompress_cube_warp(double *cube, int p, int lane)
{
    for (int i = 2; i <= p; ++i) {
        const int m = p - i;
        const int npairs = (m + 1) * (m + 2) / 2;
        for (int t = lane; t < npairs; t += 32) {
            int J, K;
            tri_pair(t, m, J, K);
            cube[cube_index(p, i, J, K)] =
                -cube[cube_index(p, i - 2, J + 2, K)] - cube[cube_index(p, i - 2, J, K + 2)];
        }
        __syncwarp();
    }
}

// {{{ P2M

// warps per CTA: four while their static tables fit in 48 KB, else two
template <int P>
__host__ __device__ constexpr int p2m_warps()
{
    return (3 * 32 * p2m_row(P) + (P + 1) * (P + 2) * (P + 3) / 6) * 8 * 4 <= 48 * 1024 ? 4 : 2;
}

// P2M with one warp per box and the full coefficients in registers: lane l
// owns the (i, j) pairs l, l + 32, ... (pairs in increasing i + j) and
// accumulates the column k = 0..P-i-j of each, so a (source, coefficient)
// term costs one FMA with the source's power z[k] = (a_z/r)^k/k!, read once
// per source two at a time; per source t = (q (a_x/r)^i/i!) (a_y/r)^j/j! is
// formed once per pair. The pair order bounds the k loop of the second and
// later row sets at compile time (order 10: 11 + 4 + 1 FMAs per source
// instead of 3 x 11); the entries past a pair's last column are computed
// and never stored. Sources go 32 at a time, one per lane for the power
// tables (a source's row of each table contiguous). The columns are then
// written to a per-warp compact full-index buffer, compressed by the p-1
// plane sweeps (warp-synchronous) and stored. Same arithmetic as p2m_kernel
// (multipole.py:77-114 and the transposed projection), ordered differently.
template <int P>
__global__ void __launch_bounds__(32 * p2m_warps<P>())
p2m_warp_kernel(double rscale, int32_t nboxes, const int32_t *__restrict__ boxes,
                const double *__restrict__ centers, int64_t cstride,
                const int32_t *__restrict__ bss, const int32_t *__restrict__ bsc,
                const double *__restrict__ sources, int64_t sstride,
                const double *__restrict__ q, int32_t base, double *__restrict__ out,
                const int32_t *__restrict__ box_level = nullptr,
                const double *__restrict__ level_rscale = nullptr)
{
    constexpr int P1 = P + 1;
    constexpr int RW = p2m_row(P);
    constexpr int NPAIR = P1 * (P1 + 1) / 2;
    constexpr int NU = (NPAIR + 31) / 32;
    constexpr int NFULL = P1 * (P1 + 1) * (P1 + 2) / 6;
    constexpr int N = P1 * P1;
    constexpr int W = p2m_warps<P>();
    // [axis][source][power]; the x powers carry the strength
    __shared__ __align__(16) double w[W][3][32][RW];
    __shared__ double full[W][NFULL];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * W + warp;
    if (ib >= nboxes) return;
    const int32_t b = boxes[ib];
    const double c[3] = {centers[b], centers[cstride + b], centers[2 * cstride + b]};
    const int32_t s0 = bss[b], ns = bsc[b];
    // all levels in one launch: the box's own level's rscale
    const double rinv = 1.0 / (level_rscale ? level_rscale[box_level[ib]] : rscale);

    // the (i, j) pairs of this lane and their last column
    int pi[NU], pj[NU], pk[NU];
#pragma unroll
    for (int u = 0; u < NU; ++u) {
        const int t = lane + 32 * u;
        const int d = p2m_pair_degree(t < NPAIR ? t : 0);
        pi[u] = t < NPAIR ? t - d * (d + 1) / 2 : 0;
        pj[u] = t < NPAIR ? d - pi[u] : 0;
        pk[u] = t < NPAIR ? P - d : -1;     // -1: idle slot, never stored
    }
    double acc[NU][P1];
#pragma unroll
    for (int u = 0; u < NU; ++u)
#pragma unroll
        for (int k = 0; k < P1; ++k) acc[u][k] = 0.0;

    for (int32_t sc = 0; sc < ns; sc += 32) {
        const int nsc = min(32, ns - sc);
        if (lane < nsc) {
            const int32_t s = s0 + sc + lane;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double a = (c[d] - sources[d * sstride + s]) * rinv;
                double v = d == 0 ? q[s] : 1.0;
                w[warp][d][lane][0] = v;
#pragma unroll
                for (int k = 1; k < P1; ++k) {
                    v = v * a * (1.0 / k);    // a compile-time reciprocal: no division
                    w[warp][d][lane][k] = v;
                }
            }
        }
        __syncwarp();
        for (int so = 0; so < nsc; ++so) {
            double z[RW];
            const double2 *zr = reinterpret_cast<const double2 *>(w[warp][2][so]);
#pragma unroll
            for (int k = 0; k < RW / 2; ++k) {
                const double2 v = zr[k];
                z[2 * k] = v.x;
                z[2 * k + 1] = v.y;
            }
#pragma unroll
            for (int u = 0; u < NU; ++u) {
                const double t = w[warp][0][so][pi[u]] * w[warp][1][so][pj[u]];
#pragma unroll
                for (int k = 0; k <= p2m_kmax<P>(u); ++k) acc[u][k] = fma(t, z[k], acc[u][k]);
            }
        }
        __syncwarp();
    }
    double *F = full[warp];
#pragma unroll
    for (int u = 0; u < NU; ++u) {
#pragma unroll
        for (int k = 0; k <= p2m_kmax<P>(u); ++k)
            if (k <= pk[u]) F[full_index(pi[u], pj[u], k)] = acc[u][k];
    }
    __syncwarp();
    // transposed projection: plane i-2 gathers from plane i, i = P..2, by
    // the precomputed full-index triples of each plane
    const int4 *sweep = reinterpret_cast<const int4 *>(p2m_sweep<P>.e);
    for (int pl = 0; pl + 2 <= P; ++pl) {
        for (int t = p2m_sweep<P>.start[pl] + lane; t < p2m_sweep<P>.start[pl + 1]; t += 32) {
            const int4 e = __ldg(sweep + t);
            double v = 0.0;
            if (e.y >= 0) v += F[e.y];
            if (e.z >= 0) v += F[e.z];
            F[e.x] -= v;
        }
        __syncwarp();
    }
    double *o = out + (int64_t)(b - base) * N;
    for (int st = lane; st < N; st += 32) o[st] = F[__ldg(p2m_sweep<P>.stored + st)];
}

// }}}

// {{{ M2M / L2L (axis-by-axis shifts)

constexpr int M2M_THREADS = 256;

// M2M with the eight children shifted concurrently: threads run over
// (child, full coefficient) pairs, each child's full coefficients in a
// compact buffer of nfull values, so one parent costs three parallel shift
// passes, one sum over children and one compression.
__global__ void __launch_bounds__(M2M_THREADS)
m2m_children_kernel(int ps, int pt, double rsrc, double rtgt, const int32_t *__restrict__ boxes,
                    const int32_t *__restrict__ child_ids, int64_t child_stride,
                    const double *__restrict__ centers, int64_t cstride, int32_t sbase,
                    const double *__restrict__ src, int32_t tbase, double *__restrict__ tgt)
{
    extern __shared__ double sm[];
    const int P1 = pt + 1;
    const int nfull = nfull_of(pt);
    double *A = sm;                         // [8][nfull]
    double *B = A + 8 * nfull;              // [8][nfull]
    double *pw = B + 8 * nfull;             // [8][3][P1]
    uint32_t *tab = reinterpret_cast<uint32_t *>(pw + 8 * 3 * P1);  // [nfull] packed (i,j,k)
    __shared__ int32_t kids[8];
    __shared__ int nkids;

    const int32_t b = boxes[blockIdx.x];
    const int ns = ncoeff_of(ps), nt = ncoeff_of(pt);
    const double ratio = rsrc / rtgt;
    if (threadIdx.x == 0) {
        int c = 0;
        for (int slot = 0; slot < 8; ++slot) {
            const int32_t ch = child_ids[slot * child_stride + b];
            if (ch != 0) kids[c++] = ch;
        }
        nkids = c;
    }
    for (int f = threadIdx.x; f < nfull; f += blockDim.x) {
        int i, j, k;
        full_mi(f, i, j, k);
        tab[f] = (uint32_t)i | ((uint32_t)j << 8) | ((uint32_t)k << 16);
    }
    __syncthreads();
    const int nk = nkids;
    for (int t = threadIdx.x; t < nk * 3; t += blockDim.x) {
        const int c = t / 3, d = t % 3;
        const int32_t ch = kids[c];
        const double dd = (centers[d * cstride + b] - centers[d * cstride + ch]) / rtgt;
        double *w = pw + (c * 3 + d) * P1;
        w[0] = 1.0;
        for (int q = 1; q <= pt; ++q) w[q] = w[q - 1] * dd / q;
    }
    for (int t = threadIdx.x; t < nk * nfull; t += blockDim.x) {
        const int c = t / nfull, f = t % nfull;
        const uint32_t e = tab[f];
        const int i = e & 0xff, j = (e >> 8) & 0xff, k = e >> 16;
        const int deg = i + j + k;
        double v = 0.0;
        if (i < 2 && deg <= ps)
            v = src[(int64_t)(kids[c] - sbase) * ns + stored_index(i, j, k)] * ipow(ratio, deg);
        A[c * nfull + f] = v;
    }
    __syncthreads();
    // axes in the order 1, 2, 0: sumpy/expansion/multipole.py:329 for the axis-0
    // hyperplanes of the Laplace stored set
    const int axes[3] = {1, 2, 0};
    double *in = A, *out = B;
#pragma unroll 1
    for (int a = 0; a < 3; ++a) {
        const int d = axes[a];
        for (int t = threadIdx.x; t < nk * nfull; t += blockDim.x) {
            const int c = t / nfull, f = t % nfull;
            const uint32_t e = tab[f];
            int m[3] = {(int)(e & 0xff), (int)((e >> 8) & 0xff), (int)(e >> 16)};
            const double *w = pw + (c * 3 + d) * P1;
            const double *inc = in + c * nfull;
            const int md = m[d];
            double acc = 0.0;
            for (int q = 0; q <= md; ++q) {
                m[d] = q;
                acc += inc[full_index(m[0], m[1], m[2])] * w[md - q];
            }
            out[c * nfull + f] = acc;
        }
        __syncthreads();
        double *sw = in; in = out; out = sw;
    }
    // sum over children into out[0..nfull) then compress in place
    double *accv = out;
    for (int f = threadIdx.x; f < nfull; f += blockDim.x) {
        double v = 0.0;
        for (int c = 0; c < nk; ++c) v += in[c * nfull + f];
        accv[f] = v;
    }
    __syncthreads();
    for (int i = pt; i >= 2; --i) {
        const int m = pt - i + 2;
        const int npairs = (m + 1) * (m + 2) / 2;
        for (int t = threadIdx.x; t < npairs; t += blockDim.x) {
            int J, K;
            tri_pair(t, m, J, K);
            double v = 0.0;
            if (J >= 2) v += accv[full_index(i, J - 2, K)];
            if (K >= 2) v += accv[full_index(i, J, K - 2)];
            accv[full_index(i - 2, J, K)] -= v;
        }
        __syncthreads();
    }
    double *o = tgt + (int64_t)(b - tbase) * nt;
    for (int s2 = threadIdx.x; s2 < nt; s2 += blockDim.x) {
        int i, j, k;
        stored_mi(s2, i, j, k);
        o[s2] += accv[full_index(i, j, k)];
    }
}

constexpr int L2L_BOXES = 8;

// L2L for up to eight target boxes per CTA, concurrently: each box's parent
// local is decompressed into the box's own compact buffer (p-1 sweeps over
// the mi0 planes, all boxes at once), then shifted one axis at a time
// (axes 0, 1, 2) and accumulated into the box's local.
__global__ void __launch_bounds__(M2M_THREADS)
l2l_boxes_kernel(int ps, int pt, double rsrc, double rtgt, int32_t nboxes,
                 const int32_t *__restrict__ boxes, const int32_t *__restrict__ parent_ids,
                 const double *__restrict__ centers, int64_t cstride, int32_t sbase,
                 const double *__restrict__ src, int32_t tbase, double *__restrict__ tgt)
{
    extern __shared__ double sm[];
    const int P1 = ps + 1;
    const int nfull = nfull_of(ps);
    double *A = sm;                                   // [8][nfull]
    double *B = A + L2L_BOXES * nfull;                // [8][nfull]
    double *pw = B + L2L_BOXES * nfull;               // [8][3][P1]
    uint32_t *tab = reinterpret_cast<uint32_t *>(pw + L2L_BOXES * 3 * P1);
    const int b0 = blockIdx.x * L2L_BOXES;
    const int nk = min(L2L_BOXES, nboxes - b0);
    const int ns = ncoeff_of(ps), nt = ncoeff_of(pt);

    for (int f = threadIdx.x; f < nfull; f += blockDim.x) {
        int i, j, k;
        full_mi(f, i, j, k);
        tab[f] = (uint32_t)i | ((uint32_t)j << 8) | ((uint32_t)k << 16);
    }
    for (int t = threadIdx.x; t < nk * 3; t += blockDim.x) {
        const int c = t / 3, d = t % 3;
        const int32_t b = boxes[b0 + c];
        const int32_t par = parent_ids[b];
        const double dd = (centers[d * cstride + b] - centers[d * cstride + par]) / rsrc;
        double *w = pw + (c * 3 + d) * P1;
        w[0] = 1.0;
        for (int q = 1; q <= ps; ++q) w[q] = w[q - 1] * dd / q;
    }
    for (int t = threadIdx.x; t < nk * ns; t += blockDim.x) {
        const int c = t / ns, s2 = t % ns;
        const int32_t par = parent_ids[boxes[b0 + c]];
        int i, j, k;
        stored_mi(s2, i, j, k);
        A[c * nfull + full_index(i, j, k)] = src[(int64_t)(par - sbase) * ns + s2];
    }
    __syncthreads();
    for (int i = 2; i <= ps; ++i) {
        const int m = ps - i;
        const int npairs = (m + 1) * (m + 2) / 2;
        for (int t = threadIdx.x; t < nk * npairs; t += blockDim.x) {
            const int c = t / npairs;
            int J, K;
            tri_pair(t % npairs, m, J, K);
            double *a = A + c * nfull;
            a[full_index(i, J, K)] = -a[full_index(i - 2, J + 2, K)] - a[full_index(i - 2, J, K + 2)];
        }
        __syncthreads();
    }
    double *in = A, *out = B;
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
        for (int t = threadIdx.x; t < nk * nfull; t += blockDim.x) {
            const int c = t / nfull, f = t % nfull;
            const uint32_t e = tab[f];
            int m[3] = {(int)(e & 0xff), (int)((e >> 8) & 0xff), (int)(e >> 16)};
            const int deg = m[0] + m[1] + m[2];
            const double *w = pw + (c * 3 + d) * P1;
            const double *inc = in + c * nfull;
            const int md = m[d];
            double acc = 0.0;
            for (int q = 0; q <= ps - deg; ++q) {
                m[d] = md + q;
                acc += inc[full_index(m[0], m[1], m[2])] * w[q];
            }
            out[c * nfull + f] = acc;
        }
        __syncthreads();
        double *sw = in; in = out; out = sw;
    }
    const double ratio = rtgt / rsrc;
    for (int t = threadIdx.x; t < nk * nt; t += blockDim.x) {
        const int c = t / nt, s2 = t % nt;
        int i, j, k;
        stored_mi(s2, i, j, k);
        const int deg = i + j + k;
        if (deg <= ps)
            tgt[(int64_t)(boxes[b0 + c] - tbase) * nt + s2] +=
                in[c * nfull + full_index(i, j, k)] * ipow(ratio, deg);
    }
}

// }}}

// {{{ L2P

constexpr int L2P_MAX_WARPS = 4;

// sum over |mi| <= p - sh of cube[i+di][j+dj][k+dk] x^i y^j z^k / (i! j! k!),
// nested Horner with inv[n] = 1/n (sh = di + dj + dk)
__device__ __forceinline__ double horner_cube(const double *cube, const double *inv, int p, int di,
                                              int dj, int dk, double x, double y, double z)
{
    const int q = p - di - dj - dk;
    double tot = 0.0;
    for (int i = q; i >= 0; --i) {
        double sy = 0.0;
        for (int j = q - i; j >= 0; --j) {
            double sz = 0.0;
            const double *row = cube + cube_index(p, i + di, j + dj, dk);
            for (int k = q - i - j; k >= 0; --k) sz = row[k] + sz * z * inv[k + 1];
            sy = sz + sy * y * inv[j + 1];
        }
        tot = sy + tot * x * inv[i + 1];
    }
    return tot;
}

// sum over j + k <= p - i of cube[i][j][k] y^j z^k / (j! k!) (one x-plane)
__device__ __forceinline__ double horner_plane(const double *cube, const double *inv, int p,
                                               int i, double y, double z)
{
    const int q = p - i;
    double sy = 0.0;
    for (int j = q; j >= 0; --j) {
        double sz = 0.0;
        const double *row = cube + cube_index(p, i, j, 0);
        for (int k = q - j; k >= 0; --k) sz = row[k] + sz * z * inv[k + 1];
        sy = sz + sy * y * inv[j + 1];
    }
    return sy;
}

template <bool GRAD>
__global__ void l2p_kernel(int p, double rscale, int32_t nboxes, const int32_t *__restrict__ boxes,
                           const double *__restrict__ centers, int64_t cstride, int32_t sbase,
                           const double *__restrict__ src, const int32_t *__restrict__ bts,
                           const int32_t *__restrict__ btc, const double *__restrict__ targets,
                           int64_t tstride, double scale, double *__restrict__ result,
                           double *__restrict__ grad)
{
    extern __shared__ double sm[];
    const int P1 = p + 1, C = P1 * P1 * P1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    const int ib = blockIdx.x * nwarps + warp;
    if (ib >= nboxes) return;
    double *cube = sm + warp * (C + P1 + 1);
    double *inv = cube + C;  // inv[n] = 1/n, n = 1..p+1

    const int32_t b = boxes[ib];
    const int n = ncoeff_of(p);
    const double *cs = src + (int64_t)(b - sbase) * n;
    for (int s = lane; s < n; s += 32) {
        int i, j, k;
        stored_mi(s, i, j, k);
        cube[cube_index(p, i, j, k)] = cs[s];
    }
    for (int q = lane; q <= p + 1; q += 32) inv[q] = q ? 1.0 / q : 0.0;
    __syncwarp();
    decompress_cube_warp(cube, p, lane);

    const double c[3] = {centers[b], centers[cstride + b], centers[2 * cstride + b]};
    const double rinv = 1.0 / rscale;
    const int32_t t0 = bts[b], nt = btc[b];
    if (!GRAD && result) {
        // values: the box's targets on g = next_pow2(nt) lanes, the 32/g lane
        // groups split the x-planes i = ph, ph + nph, ... of each target's
        // polynomial; shuffle-xor sum over the groups
        for (int32_t tc = 0; tc < nt; tc += 32) {
            const int ntc = min(32, nt - tc);
            int g = 1;
            while (g < ntc) g <<= 1;
            const int nph = 32 / g;
            const int tl = lane & (g - 1), ph = lane / g;
            const bool active = tl < ntc;
            const int32_t t = t0 + tc + tl;
            double v = 0.0;
            // groups beyond the last plane (ph > p: few targets, many groups)
            // have nothing to sum; inv[] holds 1/n for n <= p + 1 only
            if (active && ph <= p) {
                const double x = (targets[t] - c[0]) * rinv;
                const double y = (targets[tstride + t] - c[1]) * rinv;
                const double z = (targets[2 * tstride + t] - c[2]) * rinv;
                // x^i / i! for i = ph, ph + nph, ... (indices of inv[] stay <= p)
                double xi = 1.0;
                for (int i = 1; i <= ph; ++i) xi *= x * inv[i];
                for (int i = ph; i <= p; i += nph) {
                    v += xi * horner_plane(cube, inv, p, i, y, z);
                    for (int q = i + 1; q <= i + nph && q <= p; ++q) xi *= x * inv[q];
                }
            }
            for (int off = g; off < 32; off <<= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if (active && ph == 0) result[t] = scale * v;
        }
        return;
    }
    for (int32_t tt = lane; tt < nt; tt += 32) {
        const int32_t t = t0 + tt;
        const double x = (targets[t] - c[0]) * rinv;
        const double y = (targets[tstride + t] - c[1]) * rinv;
        const double z = (targets[2 * tstride + t] - c[2]) * rinv;
        if (result) result[t] = scale * horner_cube(cube, inv, p, 0, 0, 0, x, y, z);
        if (GRAD) {
            // d/dt of sum L[mi] (b/r)^mi / mi! = (1/r) sum L[mi + e_d] (b/r)^mi / mi!
            const double gs = scale * rinv;
            grad[t] = p > 0 ? gs * horner_cube(cube, inv, p, 1, 0, 0, x, y, z) : 0.0;
            grad[tstride + t] = p > 0 ? gs * horner_cube(cube, inv, p, 0, 1, 0, x, y, z) : 0.0;
            grad[2 * tstride + t] = p > 0 ? gs * horner_cube(cube, inv, p, 0, 0, 1, x, y, z) : 0.0;
        }
    }
}

// }}}

constexpr int DSTRIDE = 33;  // lanes per coefficient row + 1 (bank spread)

// {{{ M2P / P2L with register-resident derivative layers

constexpr int E2P_WARPS = 4;

// M2P: one warp per target box; the box's targets occupy g = next_pow2(nt)
// lanes and the 32/g lane groups stride over the List-3 boxes; a
// shuffle-xor tree sums the groups.
template <int P, bool GRAD>
__global__ void __launch_bounds__(32 * E2P_WARPS)
m2p_reg_kernel(double rscale, int32_t ntgt_boxes, const int32_t *__restrict__ target_boxes,
               const int32_t *__restrict__ src_starts, const int32_t *__restrict__ src_lists,
               const double *__restrict__ centers, int64_t cstride, int32_t sbase,
               const double *__restrict__ src, const int32_t *__restrict__ bts,
               const int32_t *__restrict__ btc, const double *__restrict__ targets,
               int64_t tstride, double scale, double *__restrict__ result,
               double *__restrict__ grad)
{
    constexpr int N = (P + 1) * (P + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * E2P_WARPS + warp;
    if (ib >= ntgt_boxes) return;
    const int32_t tb = target_boxes[ib];
    const int32_t t0 = bts[tb], nt = btc[tb];
    const int32_t ls = src_starts[ib], le = src_starts[ib + 1];
    const double Rinv = 1.0 / rscale;
    for (int32_t tc = 0; tc < nt; tc += 32) {
        const int ntc = min(32, nt - tc);
        int g = 1;
        while (g < ntc) g <<= 1;
        const int nph = 32 / g;
        const int tl = lane & (g - 1), ph = lane / g;
        const bool active = tl < ntc;
        const int32_t t = t0 + tc + tl;
        double tx = 0, ty = 0, tz = 0;
        if (active) { tx = targets[t]; ty = targets[tstride + t]; tz = targets[2 * tstride + t]; }
        double acc = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        if (active) {
            for (int32_t l = ls + ph; l < le; l += nph) {
                const int32_t sb = src_lists[l];
                const double *M = src + (int64_t)(sb - sbase) * N;
                // value: degrees <= P; gradient: d/dt D[mi] = D[mi + e_d] / rscale,
                // with D on (2, j, k) = -D(0, j+2, k) - D(0, j, k+2)
                laplace_layers<GRAD ? P + 1 : P>(
                    tx - centers[sb], ty - centers[cstride + sb], tz - centers[2 * cstride + sb],
                    rscale, Rinv, [&](int s, int i, int j, int k, double v) {
                        const int deg = i + j + k;
                        if (deg <= P) acc += __ldg(M + s) * v;
                        if (GRAD && deg >= 1) {
                            if (j >= 1) gy += __ldg(M + stored_index(i, j - 1, k)) * v;
                            if (k >= 1) gz += __ldg(M + stored_index(i, j, k - 1)) * v;
                            if (i == 1) {
                                gx += __ldg(M + stored_index(0, j, k)) * v;
                            } else {
                                if (j >= 2) gx -= __ldg(M + stored_index(1, j - 2, k)) * v;
                                if (k >= 2) gx -= __ldg(M + stored_index(1, j, k - 2)) * v;
                            }
                        }
                    });
            }
        }
        for (int off = g; off < 32; off <<= 1) {
            acc += __shfl_xor_sync(0xffffffffu, acc, off);
            if (GRAD) {
                gx += __shfl_xor_sync(0xffffffffu, gx, off);
                gy += __shfl_xor_sync(0xffffffffu, gy, off);
                gz += __shfl_xor_sync(0xffffffffu, gz, off);
            }
        }
        if (active && ph == 0) {
            if (result) result[t] += scale * acc;
            if (GRAD) {
                const double gs = scale * Rinv;
                grad[t] += gs * gx;
                grad[tstride + t] += gs * gy;
                grad[2 * tstride + t] += gs * gz;
            }
        }
    }
}

constexpr int P2L_WARPS = 2;

// P2L: one warp per target box; the sources of all its List-4 boxes are
// enumerated flat, 32 per round, one per lane; each lane writes q * D of its
// source into a per-warp shared transpose (stride 33) and every lane then
// sums its coefficients over the round's sources.
template <int P>
__global__ void __launch_bounds__(32 * P2L_WARPS)
p2l_reg_kernel(double rscale, int32_t ntgt_boxes, const int32_t *__restrict__ target_boxes,
               const int32_t *__restrict__ src_starts, const int32_t *__restrict__ src_lists,
               const double *__restrict__ centers, int64_t cstride,
               const int32_t *__restrict__ bss, const int32_t *__restrict__ bsc,
               const double *__restrict__ sources, int64_t sstride, const double *__restrict__ q,
               int32_t tbase, double *__restrict__ out)
{
    constexpr int N = (P + 1) * (P + 1);
    constexpr int NPL = (N + 31) / 32;
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * P2L_WARPS + warp;
    if (ib >= ntgt_boxes) return;
    double *D = sm + warp * (N * DSTRIDE);
    const int32_t tb = target_boxes[ib];
    const double c0 = centers[tb], c1 = centers[cstride + tb], c2 = centers[2 * cstride + tb];
    const int32_t ls = src_starts[ib], le = src_starts[ib + 1];
    const double Rinv = 1.0 / rscale;
    int32_t total = 0;
    for (int32_t l = ls; l < le; ++l) total += bsc[src_lists[l]];
    double acc[NPL];
#pragma unroll
    for (int m = 0; m < NPL; ++m) acc[m] = 0.0;
    for (int32_t base = 0; base < total; base += 32) {
        const int nsc = min(32, total - base);
        if (lane < nsc) {
            // locate flat source index base + lane
            int32_t f = base + lane, l = ls, sb = src_lists[ls];
            while (f >= bsc[sb]) { f -= bsc[sb]; ++l; sb = src_lists[l]; }
            const int32_t s = bss[sb] + f;
            const double qq = q[s];
            laplace_layers<P>(c0 - sources[s], c1 - sources[sstride + s],
                              c2 - sources[2 * sstride + s], rscale, Rinv,
                              [&](int k, int, int, int, double v) { D[k * DSTRIDE + lane] = qq * v; });
        }
        __syncwarp();
#pragma unroll
        for (int m = 0; m < NPL; ++m) {
            const int k = lane + 32 * m;
            if (k < N) {
                double sum = 0.0;
                for (int l2 = 0; l2 < nsc; ++l2) sum += D[k * DSTRIDE + l2];
                acc[m] += sum;
            }
        }
        __syncwarp();
    }
    double *o = out + (int64_t)(tb - tbase) * N;
#pragma unroll
    for (int m = 0; m < NPL; ++m) {
        const int k = lane + 32 * m;
        if (k < N) o[k] = acc[m];
    }
}

// Mixed-precision M2P / P2L: the FP64 offset (target - center,
// center - source) rounded to FP32, the derivative layers and the products
// with the coefficients in FP32, per List-3 box / per source; sums over
// boxes (M2P) and sources (P2L) in FP64.
constexpr int M2P_GROUPS = 8;   // lane groups (List-3 boxes in flight) per warp, mixed M2P

template <int P>
__global__ void __launch_bounds__(32 * E2P_WARPS)
m2p_mixed_kernel(double rscale, int32_t ntgt_boxes, const int32_t *__restrict__ target_boxes,
                 const int32_t *__restrict__ src_starts, const int32_t *__restrict__ src_lists,
                 const double *__restrict__ centers, int64_t cstride, int32_t sbase,
                 const double *__restrict__ src, const int32_t *__restrict__ bts,
                 const int32_t *__restrict__ btc, const double *__restrict__ targets,
                 int64_t tstride, double scale, double *__restrict__ result)
{
    constexpr int N = (P + 1) * (P + 1);
    // per warp: the multipoles of the (up to M2P_GROUPS) List-3 boxes of one
    // round, one per lane group, as FP32 (read back as broadcasts within a
    // group); lane groups have at least 32 / M2P_GROUPS lanes
    extern __shared__ float smm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * E2P_WARPS + warp;
    if (ib >= ntgt_boxes) return;
    float *Ms = smm + warp * (M2P_GROUPS * N);
    const int32_t tb = target_boxes[ib];
    const int32_t t0 = bts[tb], nt = btc[tb];
    const int32_t ls = src_starts[ib], le = src_starts[ib + 1];
    const float R = (float)rscale, Rinv = (float)(1.0 / rscale);
    for (int32_t tc = 0; tc < nt; tc += 32) {
        const int ntc = min(32, nt - tc);
        int g = 32 / M2P_GROUPS;
        while (g < ntc) g <<= 1;
        const int nph = 32 / g;
        const int tl = lane & (g - 1), ph = lane / g;
        const bool active = tl < ntc;
        const int32_t t = t0 + tc + tl;
        double tx = 0, ty = 0, tz = 0;
        if (active) { tx = targets[t]; ty = targets[tstride + t]; tz = targets[2 * tstride + t]; }
        double acc = 0.0;
        for (int32_t l0 = ls; l0 < le; l0 += nph) {
            const int nb = min(nph, le - l0);
            // stage the round's boxes: box r's coefficients at Ms[r * N ...]
            __syncwarp();
            for (int e = lane; e < nb * N; e += 32) {
                const int r = e / N, s = e - r * N;
                Ms[r * N + s] = (float)src[(int64_t)(src_lists[l0 + r] - sbase) * N + s];
            }
            __syncwarp();
            if (active && ph < nb) {
                const int32_t sb = src_lists[l0 + ph];
                const float *M = Ms + ph * N;
                float accf = 0.f;
                laplace_layers<P, float>(
                    (float)(tx - centers[sb]), (float)(ty - centers[cstride + sb]),
                    (float)(tz - centers[2 * cstride + sb]), R, Rinv,
                    [&](int s, int, int, int, float v) { accf = fmaf(M[s], v, accf); });
                acc += (double)accf;
            }
        }
        for (int off = g; off < 32; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (active && ph == 0) result[t] += scale * acc;
    }
}

template <int P>
__global__ void __launch_bounds__(32 * P2L_WARPS)
p2l_mixed_kernel(double rscale, int32_t ntgt_boxes, const int32_t *__restrict__ target_boxes,
                 const int32_t *__restrict__ src_starts, const int32_t *__restrict__ src_lists,
                 const double *__restrict__ centers, int64_t cstride,
                 const int32_t *__restrict__ bss, const int32_t *__restrict__ bsc,
                 const double *__restrict__ sources, int64_t sstride, const double *__restrict__ q,
                 int32_t tbase, double *__restrict__ out)
{
    constexpr int N = (P + 1) * (P + 1);
    constexpr int NPL = (N + 31) / 32;
    extern __shared__ float smf[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * P2L_WARPS + warp;
    if (ib >= ntgt_boxes) return;
    float *D = smf + warp * (N * DSTRIDE);
    const int32_t tb = target_boxes[ib];
    const double c0 = centers[tb], c1 = centers[cstride + tb], c2 = centers[2 * cstride + tb];
    const int32_t ls = src_starts[ib], le = src_starts[ib + 1];
    const float R = (float)rscale, Rinv = (float)(1.0 / rscale);
    int32_t total = 0;
    for (int32_t l = ls; l < le; ++l) total += bsc[src_lists[l]];
    double acc[NPL];
#pragma unroll
    for (int m = 0; m < NPL; ++m) acc[m] = 0.0;
    for (int32_t base = 0; base < total; base += 32) {
        const int nsc = min(32, total - base);
        if (lane < nsc) {
            int32_t f = base + lane, l = ls, sb = src_lists[ls];
            while (f >= bsc[sb]) { f -= bsc[sb]; ++l; sb = src_lists[l]; }
            const int32_t s = bss[sb] + f;
            const float qq = (float)q[s];
            laplace_layers<P, float>((float)(c0 - sources[s]), (float)(c1 - sources[sstride + s]),
                                     (float)(c2 - sources[2 * sstride + s]), R, Rinv,
                                     [&](int k, int, int, int, float v) { D[k * DSTRIDE + lane] = qq * v; });
        }
        __syncwarp();
#pragma unroll
        for (int m = 0; m < NPL; ++m) {
            const int k = lane + 32 * m;
            if (k < N) {
                float sum = 0.f;
                for (int l2 = 0; l2 < nsc; ++l2) sum += D[k * DSTRIDE + l2];
                acc[m] += (double)sum;
            }
        }
        __syncwarp();
    }
    double *o = out + (int64_t)(tb - tbase) * N;
#pragma unroll
    for (int m = 0; m < NPL; ++m) {
        const int k = lane + 32 * m;
        if (k < N) o[k] = acc[m];
    }
}

// {{{ L2P over packed items (all levels in one launch)

// (coefficients in the [(j, k)][i] layout of jki_offset, taylor.cuh)

// boxes per warp item (the host's L2P_ITEM_SLOTS): 4 (measured at 1M points,
// order 10: 0.144 ms against 0.235 ms with 8, whose shared memory leaves
// 12 warps per SM; most items of a 96-point-leaf tree hold one box)
#ifndef SUMPY_L2PK_SLOTS
#define SUMPY_L2PK_SLOTS 4
#endif
constexpr int L2PK_SLOTS = SUMPY_L2PK_SLOTS;

// warps per CTA: four while the slots' coefficients fit in 200 KB, else two
template <int P>
__host__ __device__ constexpr int l2pk_warps()
{
    return 8 * L2PK_SLOTS * (P + 1) * (P + 2) * (P + 3) / 6 * 4 <= 200 * 1024 ? 4 : 2;
}

// One warp evaluates up to 32 targets taken from up to L2PK_SLOTS boxes (slots; a
// box with more than 32 targets spans several items). The slots' locals
// are decompressed together (p - 1 plane sweeps, sumpy's
// CSEMatVecOperator.matvec), then lane l evaluates its target as
//   sum_(j,k) y^j z^k / (j! k!) * sum_i c[i][j][k] x^i / i!
// with x, y, z scaled by the box's rscale and the power tables in
// registers: 286 FMAs at p = 10 with compile-time indices, the x-runs of
// its own box read from shared memory (at p = 10 the eight slot bases,
// 2288 bytes apart, fall on distinct banks).
// item = {first slot, number of slots}; slot = {box, first target,
// number of targets, level}; results are assigned. GRAD: also the three
// target-coordinate derivatives, from the same x-runs shifted by one in i
// (d/dx) or taken from the neighbouring (j + 1, k) / (j, k + 1) runs.
template <int P, bool GRAD = false>
__global__ void __launch_bounds__(32 * l2pk_warps<P>())
l2p_packed_kernel(int32_t nitems, const int2 *__restrict__ items, const int4 *__restrict__ slots,
                  const double *__restrict__ level_rscale, const double *__restrict__ centers,
                  int64_t cstride, const double *__restrict__ loc,
                  const double *__restrict__ targets, int64_t tstride, double scale,
                  double *__restrict__ result, double *__restrict__ grad = nullptr)
{
    constexpr int P1 = P + 1;
    constexpr int N = P1 * P1;
    constexpr int NF = P1 * (P1 + 1) * (P1 + 2) / 6;
    extern __shared__ __align__(16) double sml[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * l2pk_warps<P>() + warp;
    if (it >= nitems) return;
    double *cubes = sml + warp * (L2PK_SLOTS * NF);
    const int2 item = items[it];
    const int nsl = item.y;
    // the warp's shared memory holds L2PK_SLOTS slots: an item with more is
    // skipped rather than written past it (the host builds at most that many)
    if (nsl < 0 || nsl > L2PK_SLOTS) return;

    // this lane's slot and target
    int my = -1, off = lane;
    int4 sl = make_int4(0, 0, 0, 0);
    for (int q = 0; q < nsl; ++q) {
        const int4 v = slots[item.x + q];
        if (my < 0) {
            if (off < v.z) { my = q; sl = v; } else { off -= v.z; }
        }
    }
    // this lane's target, its box center and rscale: loaded before the
    // locals are staged, so that their latency overlaps the staging
    double tx = 0.0, ty = 0.0, tz = 0.0, cx = 0.0, cy = 0.0, cz = 0.0, rs = 1.0;
    if (my >= 0) {
        const int32_t bb = sl.x, tt = sl.y + off;
        tx = targets[tt];
        ty = targets[tstride + tt];
        tz = targets[2 * tstride + tt];
        cx = centers[bb];
        cy = centers[cstride + bb];
        cz = centers[2 * cstride + bb];
        rs = level_rscale[sl.w];
    }
    // stored -> full layout, all slots
    for (int e = lane; e < nsl * N; e += 32) {
        const int q = e / N, st = e - q * N;
        const int32_t b = slots[item.x + q].x;
        cubes[q * NF + __ldg(l2p_decomp<P>.stored + st)] = loc[(int64_t)b * N + st];
    }
    __syncwarp();
    // decompress: plane i from plane i - 2, i = 2..P (all slots per sweep),
    // by the precomputed offset triples of each plane
    const int4 *tri = reinterpret_cast<const int4 *>(l2p_decomp<P>.e);
    for (int pl = 0; pl + 2 <= P; ++pl) {
        const int e0 = l2p_decomp<P>.start[pl];
        const int npairs = l2p_decomp<P>.start[pl + 1] - e0;
        for (int e = lane; e < nsl * npairs; e += 32) {
            int q = 0, r = e;
            while (r >= npairs) { r -= npairs; ++q; }
            const int4 o = __ldg(tri + e0 + r);
            double *c = cubes + q * NF;
            c[o.x] = -c[o.y] - c[o.z];
        }
        __syncwarp();
    }
    if (my < 0) return;
    const int32_t t = sl.y + off;
    const double rinv = 1.0 / rs;
    const double x = (tx - cx) * rinv;
    const double y = (ty - cy) * rinv;
    const double z = (tz - cz) * rinv;
    double xp[P1], yp[P1], zp[P1];
    xp[0] = yp[0] = zp[0] = 1.0;
#pragma unroll
    for (int n = 1; n <= P; ++n) {
        const double inv_n = 1.0 / n;   // compile-time constant
        xp[n] = xp[n - 1] * x * inv_n;
        yp[n] = yp[n - 1] * y * inv_n;
        zp[n] = zp[n - 1] * z * inv_n;
    }
    const double *c = cubes + my * NF;
    double pot = 0.0;
#pragma unroll
    for (int j = 0; j <= P; ++j) {
        double pj = 0.0;
#pragma unroll
        for (int k = 0; k <= P - j; ++k) {
            const double *run = c + jki_offset<P>(j, k);
            double r = 0.0;
#pragma unroll
            for (int i = P - j - k; i >= 0; --i) r = fma(run[i], xp[i], r);
            pj = fma(zp[k], r, pj);
        }
        pot = fma(yp[j], pj, pot);
    }
    if (result) result[t] = scale * pot;
    if constexpr (GRAD) {
        double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
        for (int j = 0; j < P; ++j) {
            double px = 0.0, py = 0.0, pz = 0.0;
#pragma unroll
            for (int k = 0; k < P - j; ++k) {
                const double *r0 = c + jki_offset<P>(j, k);
                const double *ry = c + jki_offset<P>(j + 1, k);
                const double *rz = c + jki_offset<P>(j, k + 1);
                double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
                for (int i = P - 1 - j - k; i >= 0; --i) {
                    sx = fma(r0[i + 1], xp[i], sx);
                    sy = fma(ry[i], xp[i], sy);
                    sz = fma(rz[i], xp[i], sz);
                }
                px = fma(zp[k], sx, px);
                py = fma(zp[k], sy, py);
                pz = fma(zp[k], sz, pz);
            }
            gx = fma(yp[j], px, gx);
            gy = fma(yp[j], py, gy);
            gz = fma(yp[j], pz, gz);
        }
        const double gs = scale * rinv;   // d/dt = (1/rscale) d/d(scaled offset)
        grad[t] = gs * gx;
        grad[tstride + t] = gs * gy;
        grad[2 * tstride + t] = gs * gz;
    }
}

// }}}

// {{{ mixed M2P / P2L over flat work items (all levels in one launch)

// The per-level launches above give one warp a whole target box: a box
// with a long List 3 (up to ~300 rounds at 1M points) runs alone at the end
// of its level while the rest of the GPU idles, and the levels run one after
// another. Here the host cuts the work into items of a few rounds each,
// over all levels, longest first; items of one target box add their partial
// sums with FP64 atomics.

__device__ __forceinline__ void cpa16(void *dst, const void *src)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cpa_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory");
}

// stored coefficients per box in the FP32 multipole copy: N rounded up to a
// multiple of 4 (16-byte rows for cp.async)
__host__ __device__ constexpr int npad_of(int p) { return (((p + 1) * (p + 1)) + 3) & ~3; }

constexpr int ITEM_WARPS = 4;
#ifndef SUMPY_P2L_REG_MAX_N
#define SUMPY_P2L_REG_MAX_N 128   // P2L items keep per-lane sums in registers up to this N
#endif
constexpr int M2PI_GROUPS = 8;   // max lane groups (List-3 boxes in flight) per warp

// FP64 multipoles [nboxes][N] -> FP32 [nboxes][NP], zero padded
__global__ void mpole_f32_kernel(int n, int np, int64_t nboxes, const double *__restrict__ src,
                                 float *__restrict__ dst)
{
    const int64_t total = nboxes * np;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = e / np;
        const int s = (int)(e - b * np);
        dst[e] = s < n ? (float)src[b * n + s] : 0.f;
    }
}

// item = {first target, first List-3 entry, number of List-3 boxes,
//         targets (1..32) | source level << 8}
// GRAD: also the potential's target-coordinate derivatives, d/dt D[mi] =
// D[mi + e_d] / rscale, from derivative layers one degree higher (the
// D(2, j, k) entries reduced by the Laplace identity to mi0 < 2).
template <int P, bool GRAD = false>
__global__ void __launch_bounds__(32 * ITEM_WARPS)
m2p_items_kernel(int32_t nitems, const int4 *__restrict__ items,
                 const double *__restrict__ level_rscale, const int32_t *__restrict__ src_lists,
                 const double *__restrict__ centers, int64_t cstride,
                 const float *__restrict__ mp32, const double *__restrict__ targets,
                 int64_t tstride, double scale, double *__restrict__ result,
                 double *__restrict__ grad = nullptr)
{
    constexpr int NP = npad_of(P);
    constexpr int C = NP / 4;
    extern __shared__ __align__(16) float smi[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * ITEM_WARPS + warp;
    if (it >= nitems) return;
    float *buf = smi + warp * (2 * M2PI_GROUPS * NP);
    const int4 item = items[it];
    const int32_t t0 = item.x, l0 = item.y, nb = item.z;
    const int ntc = item.w & 0xff, lev = item.w >> 8;
    int g = 32 / M2PI_GROUPS;
    while (g < ntc) g <<= 1;
    const int nph = 32 / g;
    const int tl = lane & (g - 1), ph = lane / g;
    const bool active = tl < ntc;
    const int32_t t = t0 + tl;
    double tx = 0, ty = 0, tz = 0;
    if (active) { tx = targets[t]; ty = targets[tstride + t]; tz = targets[2 * tstride + t]; }
    const double rs = level_rscale[lev];
    const float R = (float)rs, Rinv = (float)(1.0 / rs);
    const int nrounds = (nb + nph - 1) / nph;

    // round r's boxes (nph at most) into buffer r & 1
    auto stage = [&](int r) {
        const int first = r * nph, cnt = min(nph, nb - first);
        float *dst = buf + (r & 1) * (M2PI_GROUPS * NP);
        for (int e = lane; e < cnt * C; e += 32) {
            const int k = e / C, c = e - k * C;
            const int32_t sb = src_lists[l0 + first + k];
            cpa16(dst + k * NP + 4 * c, mp32 + (int64_t)sb * NP + 4 * c);
        }
        cpa_commit();
    };
    stage(0);
    double acc = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    for (int r = 0; r < nrounds; ++r) {
        if (r + 1 < nrounds) {
            stage(r + 1);
            cpa_wait<1>();
        } else {
            cpa_wait<0>();
        }
        __syncwarp();
        const int k = r * nph + ph;
        if (active && k < nb) {
            const int32_t sb = src_lists[l0 + k];
            const float *M = buf + (r & 1) * (M2PI_GROUPS * NP) + ph * NP;
            // four partial sums: a dependent chain of N / 4 FMAs, not N
            float a4[4] = {0.f, 0.f, 0.f, 0.f};
            if constexpr (GRAD) {
                float fx = 0.f, fy = 0.f, fz = 0.f;
                laplace_layers<P + 1, float>(
                    (float)(tx - centers[sb]), (float)(ty - centers[cstride + sb]),
                    (float)(tz - centers[2 * cstride + sb]), R, Rinv,
                    [&](int s, int i, int j, int kk, float v) {
                        const int deg = i + j + kk;
                        if (deg <= P) a4[s & 3] = fmaf(M[s], v, a4[s & 3]);
                        if (deg >= 1) {
                            if (j >= 1) fy = fmaf(M[stored_index(i, j - 1, kk)], v, fy);
                            if (kk >= 1) fz = fmaf(M[stored_index(i, j, kk - 1)], v, fz);
                            if (i == 1) {
                                fx = fmaf(M[stored_index(0, j, kk)], v, fx);
                            } else {
                                if (j >= 2) fx = fmaf(-M[stored_index(1, j - 2, kk)], v, fx);
                                if (kk >= 2) fx = fmaf(-M[stored_index(1, j, kk - 2)], v, fx);
                            }
                        }
                    });
                gx += (double)fx;
                gy += (double)fy;
                gz += (double)fz;
            } else {
                laplace_layers<P, float>(
                    (float)(tx - centers[sb]), (float)(ty - centers[cstride + sb]),
                    (float)(tz - centers[2 * cstride + sb]), R, Rinv,
                    [&](int s, int, int, int, float v) { a4[s & 3] = fmaf(M[s], v, a4[s & 3]); });
            }
            acc += (double)((a4[0] + a4[1]) + (a4[2] + a4[3]));
        }
        __syncwarp();   // buffer r & 1 is refilled by round r + 2's copies
    }
    for (int off = g; off < 32; off <<= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (GRAD) {
            gx += __shfl_xor_sync(0xffffffffu, gx, off);
            gy += __shfl_xor_sync(0xffffffffu, gy, off);
            gz += __shfl_xor_sync(0xffffffffu, gz, off);
        }
    }
    if (active && ph == 0) {
        if (result) atomicAdd(result + t, scale * acc);
        if (GRAD) {
            const double gs = scale / level_rscale[lev];
            atomicAdd(grad + t, gs * gx);
            atomicAdd(grad + tstride + t, gs * gy);
            atomicAdd(grad + 2 * tstride + t, gs * gz);
        }
    }
}

// The potential-only M2P on packed FP32 pairs: each lane group takes two
// List-3 boxes per round (boxes ph and ph + nph of the round's 2 nph), so
// every recurrence and accumulation instruction serves both boxes
// (laplace_layers_x2). A round's 2 nph FP32 multipoles are double-buffered
// into shared memory by cp.async as in m2p_items_kernel; a missing second
// box repeats the first and its half of the sum is dropped.
template <int P>
__global__ void __launch_bounds__(32 * ITEM_WARPS)
m2p_items_x2_kernel(int32_t nitems, const int4 *__restrict__ items,
                    const double *__restrict__ level_rscale, const int32_t *__restrict__ src_lists,
                    const double *__restrict__ centers, int64_t cstride,
                    const float *__restrict__ mp32, const double *__restrict__ targets,
                    int64_t tstride, double scale, double *__restrict__ result)
{
    constexpr int NP = npad_of(P);
    constexpr int C = NP / 4;
    constexpr int BUF = 2 * M2PI_GROUPS * NP;   // one round: two boxes per lane group
    extern __shared__ __align__(16) float smi[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * ITEM_WARPS + warp;
    if (it >= nitems) return;
    float *buf = smi + warp * (2 * BUF);
    const int4 item = items[it];
    const int32_t t0 = item.x, l0 = item.y, nb = item.z;
    const int ntc = item.w & 0xff, lev = item.w >> 8;
    int g = 32 / M2PI_GROUPS;
    while (g < ntc) g <<= 1;
    const int nph = 32 / g;
    const int per = 2 * nph;
    const int tl = lane & (g - 1), ph = lane / g;
    const bool active = tl < ntc;
    const int32_t t = t0 + tl;
    double tx = 0, ty = 0, tz = 0;
    if (active) { tx = targets[t]; ty = targets[tstride + t]; tz = targets[2 * tstride + t]; }
    const double rs = level_rscale[lev];
    const float R = (float)rs, Rinv = (float)(1.0 / rs);
    const int nrounds = (nb + per - 1) / per;

    // round r's boxes (2 nph at most) into buffer r & 1
    auto stage = [&](int r) {
        const int first = r * per, cnt = min(per, nb - first);
        float *dst = buf + (r & 1) * BUF;
        for (int e = lane; e < cnt * C; e += 32) {
            const int k = e / C, c = e - k * C;
            const int32_t sb = src_lists[l0 + first + k];
            cpa16(dst + k * NP + 4 * c, mp32 + (int64_t)sb * NP + 4 * c);
        }
        cpa_commit();
    };
    stage(0);
    double acc = 0.0;
    for (int r = 0; r < nrounds; ++r) {
        if (r + 1 < nrounds) {
            stage(r + 1);
            cpa_wait<1>();
        } else {
            cpa_wait<0>();
        }
        __syncwarp();
        const int k1 = r * per + ph, k2 = k1 + nph;
        if (active && k1 < nb) {
            const bool two = k2 < nb;
            const int32_t sb1 = src_lists[l0 + k1];
            const int32_t sb2 = two ? src_lists[l0 + k2] : sb1;
            const float *M1 = buf + (r & 1) * BUF + ph * NP;
            const float *M2 = two ? M1 + nph * NP : M1;
            const float2 x = make_float2((float)(tx - centers[sb1]), (float)(tx - centers[sb2]));
            const float2 y = make_float2((float)(ty - centers[cstride + sb1]),
                                         (float)(ty - centers[cstride + sb2]));
            const float2 z = make_float2((float)(tz - centers[2 * cstride + sb1]),
                                         (float)(tz - centers[2 * cstride + sb2]));
            // two partial sums per box: a dependent chain of N / 2 FMAs
            float2 a2[2] = {f2(0.f), f2(0.f)};
            laplace_layers_x2<P>(x, y, z, R, Rinv, [&](int s, int, int, int, float2 v) {
                a2[s & 1] = __ffma2_rn(make_float2(M1[s], M2[s]), v, a2[s & 1]);
            });
            acc += (double)(a2[0].x + a2[1].x);
            if (two) acc += (double)(a2[0].y + a2[1].y);
        }
        __syncwarp();   // buffer r & 1 is refilled by round r + 2's copies
    }
    for (int off = g; off < 32; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (active && ph == 0 && result) atomicAdd(result + t, scale * acc);
}

// P2L item = {target box, first entry of the flat List-4 source index
// array, number of sources (<= 32 * rounds), target level}; one item per
// warp (a persistent form, each warp running up to 32 items as one software
// pipeline, measured slower: 0.443 against 0.425 ms at 1M points). Each lane keeps
// its own FP32 sums q D over its sources in registers (N <= 128) and the
// warp transposes them through shared memory once per item; higher orders
// transpose every round.
template <int P>
__global__ void __launch_bounds__(32 * ITEM_WARPS)
p2l_items_kernel(int32_t nitems, const int4 *__restrict__ items,
                 const double *__restrict__ level_rscale, const int32_t *__restrict__ src_index,
                 const double *__restrict__ centers, int64_t cstride,
                 const double *__restrict__ sources, int64_t sstride, const double *__restrict__ q,
                 double *__restrict__ out)
{
    constexpr int N = (P + 1) * (P + 1);
    constexpr int NPL = (N + 31) / 32;
    constexpr bool REG = N <= SUMPY_P2L_REG_MAX_N;
    extern __shared__ float smf[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * ITEM_WARPS + warp;
    if (it >= nitems) return;
    float *D = smf + warp * (N * DSTRIDE);
    const int4 item = items[it];
    const int32_t tb = item.x, f0 = item.y, cnt = item.z, lev = item.w;
    const double c0 = centers[tb], c1 = centers[cstride + tb], c2 = centers[2 * cstride + tb];
    const double rs = level_rscale[lev];
    const float R = (float)rs, Rinv = (float)(1.0 / rs);
    float own[REG ? N : 1];
#pragma unroll
    for (int s = 0; s < (REG ? N : 1); ++s) own[s] = 0.f;
    double acc[NPL];
#pragma unroll
    for (int m = 0; m < NPL; ++m) acc[m] = 0.0;

    auto transpose_sum = [&](int nsrc) {
        __syncwarp();
#pragma unroll
        for (int m = 0; m < NPL; ++m) {
            const int k = lane + 32 * m;
            if (k < N) {
                float sum = 0.f;
                for (int l2 = 0; l2 < nsrc; ++l2) sum += D[k * DSTRIDE + l2];
                acc[m] += (double)sum;
            }
        }
        __syncwarp();
    };
    // software pipeline over the rounds of 32 sources: a round's coordinates
    // and strength are loaded while the previous round's derivatives are
    // computed, and its source indices one round earlier still, so that
    // only the item's first round waits for memory
    auto src_at = [&](int32_t k) { return k < cnt ? src_index[f0 + k] : -1; };
    double nx = 0.0, ny = 0.0, nz = 0.0, nq = 0.0;
    auto fetch = [&](int32_t s) {
        if (s >= 0) {
            nx = sources[s];
            ny = sources[sstride + s];
            nz = sources[2 * sstride + s];
            nq = q[s];
        }
    };
    int32_t s_next = src_at(lane);
    fetch(s_next);
    s_next = src_at(32 + lane);
    for (int32_t base = 0; base < cnt; base += 32) {
        const int nsc = min(32, cnt - base);
        const float dx = (float)(c0 - nx), dy = (float)(c1 - ny), dz = (float)(c2 - nz);
        const float qq = (float)nq;
        fetch(s_next);                      // the next round
        s_next = src_at(base + 64 + lane);  // the round after it
        if (lane < nsc) {
            laplace_layers<P, float>(dx, dy, dz, R, Rinv, [&](int k, int, int, int, float v) {
                if constexpr (REG) own[k] = fmaf(qq, v, own[k]);
                else D[k * DSTRIDE + lane] = qq * v;
            });
        }
        if constexpr (!REG) transpose_sum(nsc);
    }
    if constexpr (REG) {
#pragma unroll
        for (int s = 0; s < N; ++s) D[s * DSTRIDE + lane] = own[s];
        transpose_sum(min(32, cnt));
    }
    double *o = out + (int64_t)tb * N;
#pragma unroll
    for (int m = 0; m < NPL; ++m) {
        const int k = lane + 32 * m;
        if (k < N) atomicAdd(o + k, acc[m]);
    }
}

// }}}

template <int P, bool GRAD>
int launch_m2p_reg(double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
                   const int32_t *src_starts, const int32_t *src_lists, const double *centers,
                   int64_t cstride, int32_t sbase, const double *src, const int32_t *bts,
                   const int32_t *btc, const double *targets, int64_t tstride, double scale,
                   double *result, double *grad, cudaStream_t st)
{
    const int blocks = (ntgt_boxes + E2P_WARPS - 1) / E2P_WARPS;
    m2p_reg_kernel<P, GRAD><<<blocks, 32 * E2P_WARPS, 0, st>>>(
        rscale, ntgt_boxes, target_boxes, src_starts, src_lists, centers, cstride, sbase, src, bts,
        btc, targets, tstride, scale, result, grad);
    return check_launch("m2p_reg_kernel");
}

template <int P>
int launch_p2l_reg(double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
                   const int32_t *src_starts, const int32_t *src_lists, const double *centers,
                   int64_t cstride, const int32_t *bss, const int32_t *bsc, const double *sources,
                   int64_t sstride, const double *q, int32_t tbase, double *out, cudaStream_t st)
{
    constexpr int N = (P + 1) * (P + 1);
    const size_t smem = sizeof(double) * N * DSTRIDE * P2L_WARPS;
    int rc = prepare_smem(p2l_reg_kernel<P>, smem);
    if (rc) return rc;
    const int blocks = (ntgt_boxes + P2L_WARPS - 1) / P2L_WARPS;
    p2l_reg_kernel<P><<<blocks, 32 * P2L_WARPS, smem, st>>>(rscale, ntgt_boxes, target_boxes,
                                                             src_starts, src_lists, centers, cstride,
                                                             bss, bsc, sources, sstride, q, tbase, out);
    return check_launch("p2l_reg_kernel");
}

// }}}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_p2e_from_single_box_f64(int order, double rscale, int32_t nsrc_boxes,
                                  const int32_t *source_boxes, const double *centers,
                                  int64_t center_stride, const int32_t *box_source_starts,
                                  const int32_t *box_source_counts_nonchild,
                                  const double *sources, int64_t source_stride,
                                  const double *strength, int32_t tgt_base_ibox,
                                  double *tgt_expansions, void *stream)
{
    if (!order_ok(order)) { set_last_error("p2m: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nsrc_boxes < 0) return bad_arg("p2m: nsrc_boxes < 0");
    if (nsrc_boxes == 0) return SUMPY_OK;
    if (!source_boxes || !centers || !box_source_starts || !box_source_counts_nonchild ||
        !sources || !strength || !tgt_expansions)
        return bad_arg("p2m: null pointer argument");
#define CALL_P2M(P)                                                                              \
    (p2m_warp_kernel<P><<<(nsrc_boxes + p2m_warps<P>() - 1) / p2m_warps<P>(),                    \
                          32 * p2m_warps<P>(), 0, as_stream(stream)>>>(                           \
         rscale, nsrc_boxes, source_boxes, centers, center_stride, box_source_starts,           \
         box_source_counts_nonchild, sources, source_stride, strength, tgt_base_ibox,           \
         tgt_expansions),                                                                       \
     check_launch("p2m_warp_kernel"))
    SUMPY_ORDER_SWITCH(order, CALL_P2M)
#undef CALL_P2M
}

int sumpy_e2e_from_children_f64(int src_order, int tgt_order, double src_rscale,
                                double tgt_rscale, int32_t ntgt_boxes,
                                const int32_t *target_boxes, const int32_t *box_child_ids,
                                int64_t child_stride, const double *centers,
                                int64_t center_stride, int32_t src_base_ibox,
                                const double *src_expansions, int32_t tgt_base_ibox,
                                double *tgt_expansions, void *stream)
{
    if (!order_ok(src_order) || !order_ok(tgt_order)) {
        set_last_error("m2m: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    if (ntgt_boxes < 0) return bad_arg("m2m: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !box_child_ids || !centers || !src_expansions || !tgt_expansions)
        return bad_arg("m2m: null pointer argument");
    const int P1 = tgt_order + 1;
    const int nfull = (tgt_order + 1) * (tgt_order + 2) * (tgt_order + 3) / 6;
    const size_t smem = sizeof(double) * (16 * nfull + 8 * 3 * P1) + sizeof(uint32_t) * nfull;
    int rc = prepare_smem(m2m_children_kernel, smem);
    if (rc) return rc;
    m2m_children_kernel<<<ntgt_boxes, M2M_THREADS, smem, as_stream(stream)>>>(
        src_order, tgt_order, src_rscale, tgt_rscale, target_boxes, box_child_ids, child_stride,
        centers, center_stride, src_base_ibox, src_expansions, tgt_base_ibox, tgt_expansions);
    return check_launch("m2m_children_kernel");
}

int sumpy_e2e_from_parent_f64(int src_order, int tgt_order, double src_rscale,
                              double tgt_rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
                              const int32_t *box_parent_ids, const double *centers,
                              int64_t center_stride, int32_t src_base_ibox,
                              const double *src_expansions, int32_t tgt_base_ibox,
                              double *tgt_expansions, void *stream)
{
    if (!order_ok(src_order) || !order_ok(tgt_order)) {
        set_last_error("l2l: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    if (ntgt_boxes < 0) return bad_arg("l2l: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !box_parent_ids || !centers || !src_expansions || !tgt_expansions)
        return bad_arg("l2l: null pointer argument");
    const int P1 = src_order + 1;
    const int nfull = (src_order + 1) * (src_order + 2) * (src_order + 3) / 6;
    const size_t smem = sizeof(double) * (2 * L2L_BOXES * nfull + L2L_BOXES * 3 * P1) +
                        sizeof(uint32_t) * nfull;
    int rc = prepare_smem(l2l_boxes_kernel, smem);
    if (rc) return rc;
    const int blocks = (ntgt_boxes + L2L_BOXES - 1) / L2L_BOXES;
    l2l_boxes_kernel<<<blocks, M2M_THREADS, smem, as_stream(stream)>>>(
        src_order, tgt_order, src_rscale, tgt_rscale, ntgt_boxes, target_boxes, box_parent_ids,
        centers, center_stride, src_base_ibox, src_expansions, tgt_base_ibox, tgt_expansions);
    return check_launch("l2l_boxes_kernel");
}

static int launch_l2p(bool grad_on, int order, double rscale, int32_t ntgt_boxes,
                      const int32_t *target_boxes, const double *centers, int64_t center_stride,
                      int32_t src_base_ibox, const double *src_expansions,
                      const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
                      const double *targets, int64_t target_stride, double scale, double *result,
                      double *grad, void *stream)
{
    if (!order_ok(order)) { set_last_error("l2p: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("l2p: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !centers || !src_expansions || !box_target_starts ||
        !box_target_counts_nonchild || !targets || (!result && !grad_on) || (grad_on && !grad))
        return bad_arg("l2p: null pointer argument");
    const int P1 = order + 1;
    const size_t per_warp = sizeof(double) * (P1 * P1 * P1 + P1 + 1);
    int warps = (int)std::max<size_t>(1, std::min<size_t>(L2P_MAX_WARPS, (48 * 1024) / per_warp));
    const size_t smem = per_warp * warps;
    int rc = grad_on ? prepare_smem(l2p_kernel<true>, smem) : prepare_smem(l2p_kernel<false>, smem);
    if (rc) return rc;
    const int blocks = (ntgt_boxes + warps - 1) / warps;
    if (grad_on)
        l2p_kernel<true><<<blocks, 32 * warps, smem, as_stream(stream)>>>(
            order, rscale, ntgt_boxes, target_boxes, centers, center_stride, src_base_ibox,
            src_expansions, box_target_starts, box_target_counts_nonchild, targets, target_stride,
            scale, result, grad);
    else
        l2p_kernel<false><<<blocks, 32 * warps, smem, as_stream(stream)>>>(
            order, rscale, ntgt_boxes, target_boxes, centers, center_stride, src_base_ibox,
            src_expansions, box_target_starts, box_target_counts_nonchild, targets, target_stride,
            scale, result, nullptr);
    return check_launch("l2p_kernel");
}

int sumpy_e2p_from_single_box_f64(int order, double rscale, int32_t ntgt_boxes,
                                  const int32_t *target_boxes, const double *centers,
                                  int64_t center_stride, int32_t src_base_ibox,
                                  const double *src_expansions, const int32_t *box_target_starts,
                                  const int32_t *box_target_counts_nonchild,
                                  const double *targets, int64_t target_stride, double scale,
                                  double *result, void *stream)
{
    return launch_l2p(false, order, rscale, ntgt_boxes, target_boxes, centers, center_stride,
                      src_base_ibox, src_expansions, box_target_starts,
                      box_target_counts_nonchild, targets, target_stride, scale, result, nullptr,
                      stream);
}

int sumpy_e2p_from_single_box_grad_f64(int order, double rscale, int32_t ntgt_boxes,
                                       const int32_t *target_boxes, const double *centers,
                                       int64_t center_stride, int32_t src_base_ibox,
                                       const double *src_expansions,
                                       const int32_t *box_target_starts,
                                       const int32_t *box_target_counts_nonchild,
                                       const double *targets, int64_t target_stride, double scale,
                                       double *result, double *grad, void *stream)
{
    return launch_l2p(true, order, rscale, ntgt_boxes, target_boxes, centers, center_stride,
                      src_base_ibox, src_expansions, box_target_starts,
                      box_target_counts_nonchild, targets, target_stride, scale, result, grad,
                      stream);
}

static int launch_m2p(bool grad_on, int order, double rscale, int32_t ntgt_boxes,
                      const int32_t *target_boxes, const int32_t *source_box_starts,
                      const int32_t *source_box_lists, const double *centers,
                      int64_t center_stride, int32_t src_base_ibox, const double *src_expansions,
                      const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
                      const double *targets, int64_t target_stride, double scale, double *result,
                      double *grad, void *stream)
{
    if (!order_ok(order)) { set_last_error("m2p: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("m2p: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !source_box_starts || !source_box_lists || !centers ||
        !src_expansions || !box_target_starts || !box_target_counts_nonchild || !targets ||
        (!result && !grad_on) || (grad_on && !grad))
        return bad_arg("m2p: null pointer argument");
#define CALL_M2P(P)                                                                              \
    (grad_on ? launch_m2p_reg<P, true>(rscale, ntgt_boxes, target_boxes, source_box_starts,     \
                                       source_box_lists, centers, center_stride, src_base_ibox, \
                                       src_expansions, box_target_starts,                       \
                                       box_target_counts_nonchild, targets, target_stride,      \
                                       scale, result, grad, as_stream(stream))                   \
             : launch_m2p_reg<P, false>(rscale, ntgt_boxes, target_boxes, source_box_starts,    \
                                        source_box_lists, centers, center_stride, src_base_ibox, \
                                        src_expansions, box_target_starts,                      \
                                        box_target_counts_nonchild, targets, target_stride,     \
                                        scale, result, nullptr, as_stream(stream)))
    SUMPY_ORDER_SWITCH(order, CALL_M2P)
#undef CALL_M2P
}

int sumpy_e2p_from_csr_f64(int order, double rscale, int32_t ntgt_boxes,
                           const int32_t *target_boxes, const int32_t *source_box_starts,
                           const int32_t *source_box_lists, const double *centers,
                           int64_t center_stride, int32_t src_base_ibox,
                           const double *src_expansions, const int32_t *box_target_starts,
                           const int32_t *box_target_counts_nonchild, const double *targets,
                           int64_t target_stride, double scale, double *result, void *stream)
{
    return launch_m2p(false, order, rscale, ntgt_boxes, target_boxes, source_box_starts,
                      source_box_lists, centers, center_stride, src_base_ibox, src_expansions,
                      box_target_starts, box_target_counts_nonchild, targets, target_stride,
                      scale, result, nullptr, stream);
}

int sumpy_e2p_from_csr_grad_f64(int order, double rscale, int32_t ntgt_boxes,
                                const int32_t *target_boxes, const int32_t *source_box_starts,
                                const int32_t *source_box_lists, const double *centers,
                                int64_t center_stride, int32_t src_base_ibox,
                                const double *src_expansions, const int32_t *box_target_starts,
                                const int32_t *box_target_counts_nonchild,
                                const double *targets, int64_t target_stride, double scale,
                                double *result, double *grad, void *stream)
{
    return launch_m2p(true, order, rscale, ntgt_boxes, target_boxes, source_box_starts,
                      source_box_lists, centers, center_stride, src_base_ibox, src_expansions,
                      box_target_starts, box_target_counts_nonchild, targets, target_stride,
                      scale, result, grad, stream);
}

int sumpy_p2e_from_csr_f64(int order, double rscale, int32_t ntgt_boxes,
                           const int32_t *target_boxes, const int32_t *source_box_starts,
                           const int32_t *source_box_lists, const double *centers,
                           int64_t center_stride, const int32_t *box_source_starts,
                           const int32_t *box_source_counts_nonchild, const double *sources,
                           int64_t source_stride, const double *strength, int32_t tgt_base_ibox,
                           double *tgt_expansions, void *stream)
{
    if (!order_ok(order)) { set_last_error("p2l: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("p2l: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !source_box_starts || !source_box_lists || !centers ||
        !box_source_starts || !box_source_counts_nonchild || !sources || !strength ||
        !tgt_expansions)
        return bad_arg("p2l: null pointer argument");
#define CALL_P2L(P)                                                                             \
    launch_p2l_reg<P>(rscale, ntgt_boxes, target_boxes, source_box_starts, source_box_lists,   \
                      centers, center_stride, box_source_starts, box_source_counts_nonchild,    \
                      sources, source_stride, strength, tgt_base_ibox, tgt_expansions,          \
                      as_stream(stream))
    SUMPY_ORDER_SWITCH(order, CALL_P2L)
#undef CALL_P2L
}

int sumpy_e2p_from_csr_mixed(int order, double rscale, int32_t ntgt_boxes,
                             const int32_t *target_boxes, const int32_t *source_box_starts,
                             const int32_t *source_box_lists, const double *centers,
                             int64_t center_stride, int32_t src_base_ibox,
                             const double *src_expansions, const int32_t *box_target_starts,
                             const int32_t *box_target_counts_nonchild, const double *targets,
                             int64_t target_stride, double scale, double *result, void *stream)
{
    if (!order_ok(order)) { set_last_error("m2p mixed: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("m2p mixed: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !source_box_starts || !source_box_lists || !centers ||
        !src_expansions || !box_target_starts || !box_target_counts_nonchild || !targets || !result)
        return bad_arg("m2p mixed: null pointer argument");
    const int blocks = (ntgt_boxes + E2P_WARPS - 1) / E2P_WARPS;
#define CALL_M2PM(P)                                                                             \
    (prepare_smem(m2p_mixed_kernel<P>,                                                           \
                  sizeof(float) * M2P_GROUPS * (P + 1) * (P + 1) * E2P_WARPS)                    \
         ? SUMPY_ELAUNCH                                                                         \
         : (m2p_mixed_kernel<P><<<blocks, 32 * E2P_WARPS,                                        \
                                  sizeof(float) * M2P_GROUPS * (P + 1) * (P + 1) * E2P_WARPS,    \
                                  as_stream(stream)>>>(                                          \
                rscale, ntgt_boxes, target_boxes, source_box_starts, source_box_lists, centers, \
                center_stride, src_base_ibox, src_expansions, box_target_starts,                \
                box_target_counts_nonchild, targets, target_stride, scale, result),             \
            check_launch("m2p_mixed_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_M2PM)
#undef CALL_M2PM
}

int sumpy_p2e_from_csr_mixed(int order, double rscale, int32_t ntgt_boxes,
                             const int32_t *target_boxes, const int32_t *source_box_starts,
                             const int32_t *source_box_lists, const double *centers,
                             int64_t center_stride, const int32_t *box_source_starts,
                             const int32_t *box_source_counts_nonchild, const double *sources,
                             int64_t source_stride, const double *strength,
                             int32_t tgt_base_ibox, double *tgt_expansions, void *stream)
{
    if (!order_ok(order)) { set_last_error("p2l mixed: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("p2l mixed: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !source_box_starts || !source_box_lists || !centers ||
        !box_source_starts || !box_source_counts_nonchild || !sources || !strength ||
        !tgt_expansions)
        return bad_arg("p2l mixed: null pointer argument");
    const int blocks = (ntgt_boxes + P2L_WARPS - 1) / P2L_WARPS;
#define CALL_P2LM(P)                                                                             \
    (prepare_smem(p2l_mixed_kernel<P>,                                                           \
                  sizeof(float) * (P + 1) * (P + 1) * DSTRIDE * P2L_WARPS)                       \
         ? SUMPY_ELAUNCH                                                                         \
         : (p2l_mixed_kernel<P><<<blocks, 32 * P2L_WARPS,                                        \
                                  sizeof(float) * (P + 1) * (P + 1) * DSTRIDE * P2L_WARPS,       \
                                  as_stream(stream)>>>(                                          \
                rscale, ntgt_boxes, target_boxes, source_box_starts, source_box_lists, centers, \
                center_stride, box_source_starts, box_source_counts_nonchild, sources,          \
                source_stride, strength, tgt_base_ibox, tgt_expansions),                        \
            check_launch("p2l_mixed_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_P2LM)
#undef CALL_P2LM
}

int sumpy_p2e_from_single_box_levels_f64(int order, int32_t nsrc_boxes,
                                         const int32_t *source_boxes, const int32_t *box_levels,
                                         const double *level_rscales, const double *centers,
                                         int64_t center_stride, const int32_t *box_source_starts,
                                         const int32_t *box_source_counts_nonchild,
                                         const double *sources, int64_t source_stride,
                                         const double *strength, double *expansions,
                                         void *stream)
{
    if (!order_ok(order)) { set_last_error("p2m levels: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nsrc_boxes < 0) return bad_arg("p2m levels: nsrc_boxes < 0");
    if (nsrc_boxes == 0) return SUMPY_OK;
    if (!source_boxes || !box_levels || !level_rscales || !centers || !box_source_starts ||
        !box_source_counts_nonchild || !sources || !strength || !expansions)
        return bad_arg("p2m levels: null pointer argument");
#define CALL_P2ML(P)                                                                             \
    (p2m_warp_kernel<P><<<(nsrc_boxes + p2m_warps<P>() - 1) / p2m_warps<P>(),                    \
                          32 * p2m_warps<P>(), 0, as_stream(stream)>>>(                           \
         0.0, nsrc_boxes, source_boxes, centers, center_stride, box_source_starts,              \
         box_source_counts_nonchild, sources, source_stride, strength, 0, expansions,           \
         box_levels, level_rscales),                                                            \
     check_launch("p2m_warp_kernel"))
    SUMPY_ORDER_SWITCH(order, CALL_P2ML)
#undef CALL_P2ML
}

int sumpy_e2p_from_single_box_packed_f64(int order, int32_t nitems, const int32_t *items,
                                         const int32_t *slots, const double *level_rscales,
                                         const double *centers, int64_t center_stride,
                                         const double *src_expansions, const double *targets,
                                         int64_t target_stride, double scale, double *result,
                                         void *stream)
{
    if (!order_ok(order)) { set_last_error("l2p packed: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("l2p packed: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !slots || !level_rscales || !centers || !src_expansions || !targets || !result)
        return bad_arg("l2p packed: null pointer argument");
    if ((reinterpret_cast<uintptr_t>(items) & 7) || (reinterpret_cast<uintptr_t>(slots) & 15))
        return bad_arg("l2p packed: items must be 8-byte and slots 16-byte aligned");
#define NF_OF(P) ((P + 1) * (P + 2) * (P + 3) / 6)
#define CALL_L2PK(P)                                                                             \
    (prepare_smem(l2p_packed_kernel<P>,                                                          \
                  sizeof(double) * L2PK_SLOTS * NF_OF(P) * l2pk_warps<P>())                      \
         ? SUMPY_ELAUNCH                                                                         \
         : (l2p_packed_kernel<P><<<(nitems + l2pk_warps<P>() - 1) / l2pk_warps<P>(),             \
                                   32 * l2pk_warps<P>(),                                         \
                                   sizeof(double) * L2PK_SLOTS * NF_OF(P) * l2pk_warps<P>(),    \
                                   as_stream(stream)>>>(                                         \
                nitems, reinterpret_cast<const int2 *>(items),                                  \
                reinterpret_cast<const int4 *>(slots), level_rscales, centers, center_stride,   \
                src_expansions, targets, target_stride, scale, result),                         \
            check_launch("l2p_packed_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_L2PK)
#undef CALL_L2PK
#undef NF_OF
}

int sumpy_e2p_from_single_box_packed_grad_f64(int order, int32_t nitems, const int32_t *items,
                                              const int32_t *slots, const double *level_rscales,
                                              const double *centers, int64_t center_stride,
                                              const double *src_expansions,
                                              const double *targets, int64_t target_stride,
                                              double scale, double *result, double *grad,
                                              void *stream)
{
    if (!order_ok(order)) { set_last_error("l2p packed grad: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("l2p packed grad: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !slots || !level_rscales || !centers || !src_expansions || !targets || !grad)
        return bad_arg("l2p packed grad: null pointer argument");
    if ((reinterpret_cast<uintptr_t>(items) & 7) || (reinterpret_cast<uintptr_t>(slots) & 15))
        return bad_arg("l2p packed grad: items must be 8-byte and slots 16-byte aligned");
#define NF_OF(P) ((P + 1) * (P + 2) * (P + 3) / 6)
#define CALL_L2PKG(P)                                                                            \
    (prepare_smem(l2p_packed_kernel<P, true>,                                                    \
                  sizeof(double) * L2PK_SLOTS * NF_OF(P) * l2pk_warps<P>())                      \
         ? SUMPY_ELAUNCH                                                                         \
         : (l2p_packed_kernel<P, true><<<(nitems + l2pk_warps<P>() - 1) / l2pk_warps<P>(),       \
                                         32 * l2pk_warps<P>(),                                   \
                                         sizeof(double) * L2PK_SLOTS * NF_OF(P) *                \
                                             l2pk_warps<P>(),                                    \
                                         as_stream(stream)>>>(                                   \
                nitems, reinterpret_cast<const int2 *>(items),                                  \
                reinterpret_cast<const int4 *>(slots), level_rscales, centers, center_stride,   \
                src_expansions, targets, target_stride, scale, result, grad),                   \
            check_launch("l2p_packed_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_L2PKG)
#undef CALL_L2PKG
#undef NF_OF
}

int sumpy_mpoles_to_f32(int order, int64_t nboxes, const double *src_expansions, float *dst,
                        void *stream)
{
    if (!order_ok(order)) { set_last_error("mpoles_to_f32: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nboxes < 0) return bad_arg("mpoles_to_f32: nboxes < 0");
    if (nboxes == 0) return SUMPY_OK;
    if (!src_expansions || !dst) return bad_arg("mpoles_to_f32: null pointer argument");
    const int np = npad_of(order);
    const int64_t total = nboxes * np;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
    mpole_f32_kernel<<<blocks, 256, 0, as_stream(stream)>>>(ncoeff_of(order), np, nboxes,
                                                            src_expansions, dst);
    return check_launch("mpole_f32_kernel");
}

int sumpy_e2p_from_items_mixed(int order, int32_t nitems, const int32_t *items,
                               const double *level_rscales, const int32_t *source_box_lists,
                               const double *centers, int64_t center_stride,
                               const float *src_expansions_f32, const double *targets,
                               int64_t target_stride, double scale, double *result, void *stream)
{
    if (!order_ok(order)) { set_last_error("m2p items: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("m2p items: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !level_rscales || !source_box_lists || !centers || !src_expansions_f32 ||
        !targets || !result)
        return bad_arg("m2p items: null pointer argument");
    if ((reinterpret_cast<uintptr_t>(items) | reinterpret_cast<uintptr_t>(src_expansions_f32)) & 15)
        return bad_arg("m2p items: items and FP32 expansions must be 16-byte aligned");
    const int blocks = (nitems + ITEM_WARPS - 1) / ITEM_WARPS;
#define CALL_M2PI(P)                                                                             \
    (prepare_smem(m2p_items_x2_kernel<P>,                                                        \
                  sizeof(float) * 4 * M2PI_GROUPS * npad_of(P) * ITEM_WARPS)                     \
         ? SUMPY_ELAUNCH                                                                         \
         : (m2p_items_x2_kernel<P><<<blocks, 32 * ITEM_WARPS,                                    \
                                     sizeof(float) * 4 * M2PI_GROUPS * npad_of(P) * ITEM_WARPS,  \
                                     as_stream(stream)>>>(                                       \
                nitems, reinterpret_cast<const int4 *>(items), level_rscales, source_box_lists, \
                centers, center_stride, src_expansions_f32, targets, target_stride, scale,      \
                result),                                                                         \
            check_launch("m2p_items_x2_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_M2PI)
#undef CALL_M2PI
}

int sumpy_e2p_from_items_grad_mixed(int order, int32_t nitems, const int32_t *items,
                                    const double *level_rscales,
                                    const int32_t *source_box_lists, const double *centers,
                                    int64_t center_stride, const float *src_expansions_f32,
                                    const double *targets, int64_t target_stride, double scale,
                                    double *result, double *grad, void *stream)
{
    if (!order_ok(order)) { set_last_error("m2p items grad: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("m2p items grad: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !level_rscales || !source_box_lists || !centers || !src_expansions_f32 ||
        !targets || !grad)
        return bad_arg("m2p items grad: null pointer argument");
    if ((reinterpret_cast<uintptr_t>(items) | reinterpret_cast<uintptr_t>(src_expansions_f32)) & 15)
        return bad_arg("m2p items grad: items and FP32 expansions must be 16-byte aligned");
    const int blocks = (nitems + ITEM_WARPS - 1) / ITEM_WARPS;
#define CALL_M2PIG(P)                                                                            \
    (prepare_smem(m2p_items_kernel<P, true>,                                                     \
                  sizeof(float) * 2 * M2PI_GROUPS * npad_of(P) * ITEM_WARPS)                     \
         ? SUMPY_ELAUNCH                                                                         \
         : (m2p_items_kernel<P, true><<<blocks, 32 * ITEM_WARPS,                                 \
                                        sizeof(float) * 2 * M2PI_GROUPS * npad_of(P) * ITEM_WARPS, \
                                        as_stream(stream)>>>(                                    \
                nitems, reinterpret_cast<const int4 *>(items), level_rscales, source_box_lists, \
                centers, center_stride, src_expansions_f32, targets, target_stride, scale,      \
                result, grad),                                                                   \
            check_launch("m2p_items_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_M2PIG)
#undef CALL_M2PIG
}

int sumpy_p2e_from_items_mixed(int order, int32_t nitems, const int32_t *items,
                               const double *level_rscales, const int32_t *source_index,
                               const double *centers, int64_t center_stride,
                               const double *sources, int64_t source_stride,
                               const double *strength, double *tgt_expansions, void *stream)
{
    if (!order_ok(order)) { set_last_error("p2l items: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("p2l items: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !level_rscales || !source_index || !centers || !sources || !strength ||
        !tgt_expansions)
        return bad_arg("p2l items: null pointer argument");
    if (reinterpret_cast<uintptr_t>(items) & 15)
        return bad_arg("p2l items: items must be 16-byte aligned");
    const int blocks = (nitems + ITEM_WARPS - 1) / ITEM_WARPS;
#define CALL_P2LI(P)                                                                             \
    (prepare_smem(p2l_items_kernel<P>, sizeof(float) * (P + 1) * (P + 1) * DSTRIDE * ITEM_WARPS) \
         ? SUMPY_ELAUNCH                                                                         \
         : (p2l_items_kernel<P><<<blocks, 32 * ITEM_WARPS,                                       \
                                  sizeof(float) * (P + 1) * (P + 1) * DSTRIDE * ITEM_WARPS,      \
                                  as_stream(stream)>>>(                                          \
                nitems, reinterpret_cast<const int4 *>(items), level_rscales, source_index,     \
                centers, center_stride, sources, source_stride, strength, tgt_expansions),      \
            check_launch("p2l_items_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_P2LI)
#undef CALL_P2LI
}

}  // extern "C"
