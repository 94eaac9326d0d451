// 3D Helmholtz FMM kernels: G = exp(i k r) / r (sumpy's HelmholtzKernel(3),
// sumpy/kernel.py:755-844) with the compressed Taylor expansions
// (stored set mi0 < 2). Complex values are interleaved (re, im) pairs
// (double2), which is how a complex128 array is laid out.
//
// What differs from the Laplace kernels:
//  * P2M, M2M, L2L and L2P are real-linear maps with real coefficients (k is
//    real), applied here to complex data. The PDE projection gains a term:
//    u_mi = -u_{mi-2e0+2e1} - u_{mi-2e0+2e2} - kappa u_{mi-2e0} with
//    kappa = k^2 rscale^2 (sumpy/expansion/__init__.py:754-886 for the PDE
//    Laplacian + k^2, sumpy/kernel.py:838-844).
//  * M2P and P2L need D(mi) = rs^|mi| d^mi G for the stored mi. sumpy takes
//    them with Tausch's recursion for radial functions
//    (RadialDerivativeTaker / HelmholtzDerivativeTaker,
//    sumpy/derivative_taker.py:269-389). Here the same quantities come from
//    its closed form: with u = r^2/2, G = F(u) and g_Q = F^(Q)(u) =
//    ((1/r) d/dr)^Q G, the chain rule on the separable u = sum x_a^2/2 gives
//        d^mi G = sum_{q_a} g_{q0+q1+q2} prod_a C[m_a][q_a] x_a^(2 q_a - m_a),
//        C[m][q] = m! / ((2q - m)! (m - q)! 2^(m - q)),  ceil(m/2) <= q <= m,
//    so with n = x/r, rho = rs/r and gamma_Q = r^(2Q) g_Q,
//        D(mi) = rho^|mi| sum_{q_a} gamma_{q0+q1+q2} prod_a C[m_a][q_a] n_a^(2q_a - m_a),
//    gamma_0 = e^{ikr}/r, gamma_1 = (ikr - 1) e^{ikr}/r,
//    gamma_Q = -(2Q - 1) gamma_{Q-1} - (kr)^2 gamma_{Q-2}
//    (sumpy's q >= 2 step for g_q multiplied by r^(2Q)). For stored mi,
//    m_0 <= 1 and the axis-0 factor is 1 or n_0.
//  * P2P evaluates q e^{ikr}/r with complex strengths.
//  * M2L reuses the real GEMM kernels (m2l.cu, m2l_tc.cu) on the real
//    embedding [[Re, -Im], [Im, Re]] of the complex class operators.
#include <algorithm>
#include <utility>

#include "common.cuh"
#include "helmholtz_core.cuh"
#include "taylor.cuh"
#include "index_tables.cuh"

namespace sumpy {
namespace {

// {{{ P2P

constexpr int HP2P_WARPS = 8;

struct HSrc {
    double x, y, z, qr, qi;
};

// List 1 (P2PFromCSR, sumpy/p2p.py:484-799) for G = e^{ikr}/r: one warp per
// target box, targets on g = next_pow2(nt) lanes, 32/g lane groups striding
// the staged sources, shuffle-xor sum. MIXED: FP64 coordinate difference
// rounded to FP32, FP32 distance, phase and products per source box, FP64
// totals. Results are assigned.
template <bool MIXED>
__global__ void __launch_bounds__(32 * HP2P_WARPS)
hp2p_csr_kernel(int32_t ntgt_boxes, const int32_t *__restrict__ target_boxes,
                const int32_t *__restrict__ src_box_starts, const int32_t *__restrict__ src_box_lists,
                const int32_t *__restrict__ box_src_starts, const int32_t *__restrict__ box_src_counts,
                const int32_t *__restrict__ box_tgt_starts, const int32_t *__restrict__ box_tgt_counts,
                const double *__restrict__ sources, int64_t sstride, const z2 *__restrict__ strength,
                const double *__restrict__ targets, int64_t tstride,
                const int32_t *__restrict__ target_to_source, double k, double scale,
                z2 *__restrict__ result)
{
    __shared__ HSrc buf[HP2P_WARPS][32];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int ib = blockIdx.x * HP2P_WARPS + warp;
    if (ib >= ntgt_boxes) return;
    HSrc *wb = buf[warp];
    const float kf = (float)k;

    const int32_t tb = target_boxes[ib];
    const int32_t t0 = box_tgt_starts[tb];
    const int32_t nt = box_tgt_counts[tb];
    const int32_t ls = src_box_starts[ib], le = src_box_starts[ib + 1];

    for (int32_t tc = 0; tc < nt; tc += 32) {
        const int ntc = min(32, nt - tc);
        int g = 1;
        while (g < ntc) g <<= 1;
        const int nph = 32 / g;
        const int tl = lane & (g - 1);
        const int ph = lane / g;
        const bool active = tl < ntc;
        const int32_t t = t0 + tc + tl;
        double tx = 0, ty = 0, tz = 0;
        int32_t self = -1;
        if (active) {
            tx = targets[t];
            ty = targets[tstride + t];
            tz = targets[2 * tstride + t];
            if (target_to_source) self = target_to_source[t];
        }
        double ar = 0.0, ai = 0.0;
        for (int32_t l = ls; l < le; ++l) {
            const int32_t sb = src_box_lists[l];
            const int32_t s0 = box_src_starts[sb];
            const int32_t ns = box_src_counts[sb];
            float arf = 0.f, aif = 0.f;
            for (int32_t sc = 0; sc < ns; sc += 32) {
                const int nsc = min(32, ns - sc);
                if (lane < nsc) {
                    const int32_t s = s0 + sc + lane;
                    const z2 q = strength[s];
                    wb[lane].x = sources[s];
                    wb[lane].y = sources[sstride + s];
                    wb[lane].z = sources[2 * sstride + s];
                    wb[lane].qr = q.x;
                    wb[lane].qi = q.y;
                }
                __syncwarp();
                if (active) {
                    for (int j = ph; j < nsc; j += nph) {
                        if (s0 + sc + j == self) continue;
                        const HSrc sp = wb[j];
                        if (MIXED) {
                            const float dx = (float)(tx - sp.x);
                            const float dy = (float)(ty - sp.y);
                            const float dz = (float)(tz - sp.z);
                            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            const float ri = rsqrtf(r2);
                            float sn, cs;
                            sincosf(kf * (r2 * ri), &sn, &cs);
                            const float wr = cs * ri, wi = sn * ri;
                            const float qr = (float)sp.qr, qi = (float)sp.qi;
                            arf = fmaf(qr, wr, fmaf(-qi, wi, arf));
                            aif = fmaf(qr, wi, fmaf(qi, wr, aif));
                        } else {
                            const double dx = tx - sp.x, dy = ty - sp.y, dz = tz - sp.z;
                            const double r2 = dx * dx + dy * dy + dz * dz;
                            const double ri = rsqrt(r2);
                            double sn, cs;
                            sincos(k * (r2 * ri), &sn, &cs);
                            const double wr = cs * ri, wi = sn * ri;
                            ar = fma(sp.qr, wr, fma(-sp.qi, wi, ar));
                            ai = fma(sp.qr, wi, fma(sp.qi, wr, ai));
                        }
                    }
                }
                __syncwarp();
            }
            if (MIXED) {
                ar += (double)arf;
                ai += (double)aif;
            }
        }
        for (int off = g; off < 32; off <<= 1) {
            ar += __shfl_xor_sync(0xffffffffu, ar, off);
            ai += __shfl_xor_sync(0xffffffffu, ai, off);
        }
        if (active && ph == 0) result[t] = zmk(scale * ar, scale * ai);
    }
}

constexpr int HDIRECT_THREADS = 256;

// all pairs, FP64 (sumpy/p2p.py:215-285)
__global__ void __launch_bounds__(HDIRECT_THREADS)
hp2p_direct_kernel(int64_t ntgt, const double *__restrict__ targets, int64_t tstride, int64_t nsrc,
                   const double *__restrict__ sources, int64_t sstride,
                   const z2 *__restrict__ strength, const int32_t *__restrict__ target_to_source,
                   double k, double scale, z2 *__restrict__ result)
{
    __shared__ HSrc tile[HDIRECT_THREADS];
    const int64_t t = (int64_t)blockIdx.x * HDIRECT_THREADS + threadIdx.x;
    const bool active = t < ntgt;
    double tx = 0, ty = 0, tz = 0;
    int64_t self = -1;
    if (active) {
        tx = targets[t];
        ty = targets[tstride + t];
        tz = targets[2 * tstride + t];
        if (target_to_source) self = target_to_source[t];
    }
    double ar = 0.0, ai = 0.0;
    for (int64_t s0 = 0; s0 < nsrc; s0 += HDIRECT_THREADS) {
        const int64_t s = s0 + threadIdx.x;
        if (s < nsrc) {
            const z2 q = strength[s];
            tile[threadIdx.x] = HSrc{sources[s], sources[sstride + s], sources[2 * sstride + s],
                                     q.x, q.y};
        }
        __syncthreads();
        const int n = (int)min((int64_t)HDIRECT_THREADS, nsrc - s0);
        if (active) {
            for (int j = 0; j < n; ++j) {
                if (s0 + j == self) continue;
                const double dx = tx - tile[j].x, dy = ty - tile[j].y, dz = tz - tile[j].z;
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double ri = rsqrt(r2);
                double sn, cs;
                sincos(k * (r2 * ri), &sn, &cs);
                const double wr = cs * ri, wi = sn * ri;
                ar = fma(tile[j].qr, wr, fma(-tile[j].qi, wi, ar));
                ai = fma(tile[j].qr, wi, fma(tile[j].qi, wr, ai));
            }
        }
        __syncthreads();
    }
    if (active) result[t] = zmk(scale * ar, scale * ai);
}

// }}}

// {{{ P2M

// P2M with one warp per box, the Laplace P2M's schedule on complex
// strengths (p2m_warp_kernel, expansions.cu): lane l owns the (i, j) pairs
// l, l + 32, ... in increasing i + j and accumulates the real and imaginary
// parts of their columns k = 0..P-i-j in registers; per source the z powers
// are read once, two at a time, and t = (a_x/r)^i/i! (a_y/r)^j/j! is formed
// once per pair and scaled by the strength's two parts. The columns go to a
// per-warp compact full-index buffer, compressed by the transposed
// Helmholtz projection, planes P..2 in turn (the sweep table's fourth index
// is the kappa term), and stored (sumpy/p2e.py:155-261,
// multipole.py:77-114; sumpy/expansion/__init__.py:754-886).
template <int P>
__host__ __device__ constexpr int hp2m_warps()
{
    return (3 * 32 * p2m_row(P) + 2 * 32 + 2 * (P + 1) * (P + 2) * (P + 3) / 6) * 8 * 2 <=
                   48 * 1024
               ? 2
               : 1;
}

template <int P>
__global__ void __launch_bounds__(32 * hp2m_warps<P>())
hp2m_warp_kernel(double rscale, double k, int32_t nboxes, const int32_t *__restrict__ boxes,
                 const double *__restrict__ centers, int64_t cstride,
                 const int32_t *__restrict__ bss, const int32_t *__restrict__ bsc,
                 const double *__restrict__ sources, int64_t sstride, const z2 *__restrict__ q,
                 int32_t base, z2 *__restrict__ out, const int32_t *__restrict__ box_level,
                 const double *__restrict__ level_rscale)
{
    constexpr int P1 = P + 1;
    constexpr int RW = p2m_row(P);
    constexpr int NPAIR = P1 * (P1 + 1) / 2;
    constexpr int NU = (NPAIR + 31) / 32;
    constexpr int NFULL = P1 * (P1 + 1) * (P1 + 2) / 6;
    constexpr int N = P1 * P1;
    constexpr int W = hp2m_warps<P>();
    __shared__ __align__(16) double w[W][3][32][RW];   // [axis][source][power]
    __shared__ z2 qs[W][32];
    __shared__ z2 full[W][NFULL];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * W + warp;
    if (ib >= nboxes) return;
    const int32_t b = boxes[ib];
    const double c[3] = {centers[b], centers[cstride + b], centers[2 * cstride + b]};
    const int32_t s0 = bss[b], ns = bsc[b];
    // all levels in one launch: the box's own level's rscale
    const double rs = level_rscale ? level_rscale[box_level[ib]] : rscale;
    const double rinv = 1.0 / rs, kappa = k * k * rs * rs;

    int pi[NU], pj[NU], pk[NU];
#pragma unroll
    for (int u = 0; u < NU; ++u) {
        const int t = lane + 32 * u;
        const int d = p2m_pair_degree(t < NPAIR ? t : 0);
        pi[u] = t < NPAIR ? t - d * (d + 1) / 2 : 0;
        pj[u] = t < NPAIR ? d - pi[u] : 0;
        pk[u] = t < NPAIR ? P - d : -1;     // -1: idle slot, never stored
    }
    double ar[NU][P1], ai[NU][P1];
#pragma unroll
    for (int u = 0; u < NU; ++u)
#pragma unroll
        for (int kk = 0; kk < P1; ++kk) ar[u][kk] = ai[u][kk] = 0.0;

    for (int32_t sc = 0; sc < ns; sc += 32) {
        const int nsc = min(32, ns - sc);
        if (lane < nsc) {
            const int32_t s = s0 + sc + lane;
            qs[warp][lane] = q[s];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double a = (c[d] - sources[d * sstride + s]) * rinv;
                double v = 1.0;
                w[warp][d][lane][0] = v;
#pragma unroll
                for (int kk = 1; kk < P1; ++kk) {
                    v = v * a * (1.0 / kk);    // a compile-time reciprocal: no division
                    w[warp][d][lane][kk] = v;
                }
            }
        }
        __syncwarp();
        for (int so = 0; so < nsc; ++so) {
            double z[RW];
            const double2 *zr = reinterpret_cast<const double2 *>(w[warp][2][so]);
#pragma unroll
            for (int kk = 0; kk < RW / 2; ++kk) {
                const double2 v = zr[kk];
                z[2 * kk] = v.x;
                z[2 * kk + 1] = v.y;
            }
            const z2 qq = qs[warp][so];
#pragma unroll
            for (int u = 0; u < NU; ++u) {
                const double t = w[warp][0][so][pi[u]] * w[warp][1][so][pj[u]];
                const double tr = t * qq.x, ti = t * qq.y;
#pragma unroll
                for (int kk = 0; kk <= p2m_kmax<P>(u); ++kk) {
                    ar[u][kk] = fma(tr, z[kk], ar[u][kk]);
                    ai[u][kk] = fma(ti, z[kk], ai[u][kk]);
                }
            }
        }
        __syncwarp();
    }
    z2 *F = full[warp];
#pragma unroll
    for (int u = 0; u < NU; ++u) {
#pragma unroll
        for (int kk = 0; kk <= p2m_kmax<P>(u); ++kk)
            if (kk <= pk[u]) F[full_index(pi[u], pj[u], kk)] = zmk(ar[u][kk], ai[u][kk]);
    }
    __syncwarp();
    // transposed projection: plane i-2 gathers from plane i, i = P..2
    const int4 *sweep = reinterpret_cast<const int4 *>(p2m_sweep<P>.e);
    for (int pl = 0; pl + 2 <= P; ++pl) {
        for (int t = p2m_sweep<P>.start[pl] + lane; t < p2m_sweep<P>.start[pl + 1]; t += 32) {
            const int4 e = __ldg(sweep + t);
            z2 v = zmk(0.0, 0.0);
            if (e.y >= 0) v = zadd(v, F[e.y]);
            if (e.z >= 0) v = zadd(v, F[e.z]);
            if (e.w >= 0) v = zaxpy(kappa, F[e.w], v);
            F[e.x] = zmk(F[e.x].x - v.x, F[e.x].y - v.y);
        }
        __syncwarp();
    }
    z2 *o = out + (int64_t)(b - base) * N;
    for (int st = lane; st < N; st += 32) o[st] = F[__ldg(p2m_sweep<P>.stored + st)];
}

// }}}

// {{{ M2M / L2L

constexpr int HE2E_THREADS = 256;

// E2EFromChildren (sumpy/e2e.py:866-978; multipole.py:159-407): the
// children's stored coefficients in the parent's full slots times
// (r_child/r_parent)^|mi|, shifted along axes 1, 2, 0 (all children of the
// parent concurrently), summed, compressed with kappa_parent; accumulated.
__global__ void __launch_bounds__(HE2E_THREADS)
hm2m_kernel(int ps, int pt, double rsrc, double rtgt, double kappa_t,
            const int32_t *__restrict__ boxes, const int32_t *__restrict__ child_ids,
            int64_t child_stride, const double *__restrict__ centers, int64_t cstride,
            int32_t sbase, const z2 *__restrict__ src, int32_t tbase, z2 *__restrict__ tgt)
{
    extern __shared__ __align__(16) double sm[];
    const int P1 = pt + 1;
    const int nfull = nfull_of(pt);
    z2 *A = reinterpret_cast<z2 *>(sm);     // [8][nfull]
    z2 *B = A + 8 * nfull;                  // [8][nfull]
    double *pw = reinterpret_cast<double *>(B + 8 * nfull);        // [8][3][P1]
    uint32_t *tab = reinterpret_cast<uint32_t *>(pw + 8 * 3 * P1);  // [nfull]
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
        z2 v = zmk(0.0, 0.0);
        if (i < 2 && deg <= ps)
            v = zscal(ipow(ratio, deg), src[(int64_t)(kids[c] - sbase) * ns + stored_index(i, j, k)]);
        A[c * nfull + f] = v;
    }
    __syncthreads();
    const int axes[3] = {1, 2, 0};
    z2 *in = A, *out = B;
#pragma unroll 1
    for (int a = 0; a < 3; ++a) {
        const int d = axes[a];
        for (int t = threadIdx.x; t < nk * nfull; t += blockDim.x) {
            const int c = t / nfull, f = t % nfull;
            const uint32_t e = tab[f];
            int m[3] = {(int)(e & 0xff), (int)((e >> 8) & 0xff), (int)(e >> 16)};
            const double *w = pw + (c * 3 + d) * P1;
            const z2 *inc = in + c * nfull;
            const int md = m[d];
            z2 acc = zmk(0.0, 0.0);
            for (int q = 0; q <= md; ++q) {
                m[d] = q;
                acc = zaxpy(w[md - q], inc[full_index(m[0], m[1], m[2])], acc);
            }
            out[c * nfull + f] = acc;
        }
        __syncthreads();
        z2 *sw = in; in = out; out = sw;
    }
    z2 *accv = out;
    for (int f = threadIdx.x; f < nfull; f += blockDim.x) {
        z2 v = zmk(0.0, 0.0);
        for (int c = 0; c < nk; ++c) v = zadd(v, in[c * nfull + f]);
        accv[f] = v;
    }
    __syncthreads();
    for (int i = pt; i >= 2; --i) {
        const int m = pt - i + 2;
        const int npairs = (m + 1) * (m + 2) / 2;
        for (int t = threadIdx.x; t < npairs; t += blockDim.x) {
            int J, K;
            tri_pair(t, m, J, K);
            z2 v = zmk(0.0, 0.0);
            if (J >= 2) v = zadd(v, accv[full_index(i, J - 2, K)]);
            if (K >= 2) v = zadd(v, accv[full_index(i, J, K - 2)]);
            if (J + K <= pt - i) v = zaxpy(kappa_t, accv[full_index(i, J, K)], v);
            z2 &o = accv[full_index(i - 2, J, K)];
            o = zmk(o.x - v.x, o.y - v.y);
        }
        __syncthreads();
    }
    z2 *o = tgt + (int64_t)(b - tbase) * nt;
    for (int s2 = threadIdx.x; s2 < nt; s2 += blockDim.x) {
        int i, j, k;
        stored_mi(s2, i, j, k);
        o[s2] = zadd(o[s2], accv[full_index(i, j, k)]);
    }
}

constexpr int HL2L_BOXES = 4;

// E2EFromParent (sumpy/e2e.py:985-1083; local.py:346-464): parent local
// decompressed with kappa_parent, Taylor-shifted along axes 0, 1, 2
// (truncated at the parent's order P), times (r_child/r_parent)^|mi|,
// accumulated into the child; HL2L_BOXES children per CTA. Every multi-index
// step comes from the compile-time tables of full_shift<P> (the shift terms
// m + q e_d and the decompression planes in the compact full layout).
template <int P>
__global__ void __launch_bounds__(HE2E_THREADS)
hl2l_kernel(int pt, double rsrc, double rtgt, double kappa_s, int32_t nboxes,
            const int32_t *__restrict__ boxes, const int32_t *__restrict__ parent_ids,
            const double *__restrict__ centers, int64_t cstride, int32_t sbase,
            const z2 *__restrict__ src, int32_t tbase, z2 *__restrict__ tgt)
{
    constexpr int P1 = P + 1;
    constexpr int NF = FullShift<P>::NFULL;
    constexpr int NS = P1 * P1;
    const FullShift<P> &T = full_shift<P>;
    extern __shared__ __align__(16) double sm[];
    z2 *A = reinterpret_cast<z2 *>(sm);
    z2 *B = A + HL2L_BOXES * NF;
    double *pw = reinterpret_cast<double *>(B + HL2L_BOXES * NF);   // [box][axis][P1]
    const int b0 = blockIdx.x * HL2L_BOXES;
    const int nk = min(HL2L_BOXES, nboxes - b0);

    for (int t = threadIdx.x; t < nk * 3; t += blockDim.x) {
        const int c = t / 3, d = t % 3;
        const int32_t b = boxes[b0 + c];
        const int32_t par = parent_ids[b];
        const double dd = (centers[d * cstride + b] - centers[d * cstride + par]) / rsrc;
        double *w = pw + (c * 3 + d) * P1;
        double v = 1.0;
        w[0] = v;
#pragma unroll
        for (int q = 1; q <= P; ++q) {
            v = v * dd * (1.0 / q);    // a compile-time reciprocal: no division
            w[q] = v;
        }
    }
    for (int t = threadIdx.x; t < nk * NS; t += blockDim.x) {
        const int c = t / NS, s2 = t - c * NS;
        const int32_t par = parent_ids[boxes[b0 + c]];
        A[c * NF + __ldg(p2m_sweep<P>.stored + s2)] = src[(int64_t)(par - sbase) * NS + s2];
    }
    __syncthreads();
    const int4 *de = reinterpret_cast<const int4 *>(T.e);
    for (int pl = 0; pl + 2 <= P; ++pl) {
        const int e0 = T.dstart[pl], npairs = T.dstart[pl + 1] - e0;
        for (int t = threadIdx.x; t < nk * npairs; t += blockDim.x) {
            int c = 0, r = t;
            while (r >= npairs) { r -= npairs; ++c; }
            const int4 o = __ldg(de + e0 + r);
            z2 *a = A + c * NF;
            const z2 u1 = a[o.y], u2 = a[o.z], u0 = a[o.w];
            a[o.x] = zmk(-u1.x - u2.x - kappa_s * u0.x, -u1.y - u2.y - kappa_s * u0.y);
        }
        __syncthreads();
    }
    z2 *in = A, *out = B;
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
        const short *ix = T.idx[d];
        for (int t = threadIdx.x; t < nk * NF; t += blockDim.x) {
            const int c = t / NF, f = t - c * NF;
            const int s0 = __ldg(T.start + f), s1 = __ldg(T.start + f + 1);
            const double *w = pw + (c * 3 + d) * P1;
            const z2 *inc = in + c * NF;
            z2 acc = zmk(0.0, 0.0);
            for (int s = s0; s < s1; ++s) acc = zaxpy(w[s - s0], inc[__ldg(ix + s)], acc);
            out[c * NF + f] = acc;
        }
        __syncthreads();
        z2 *sw = in; in = out; out = sw;
    }
    __shared__ double rpow[P1];
    if (threadIdx.x == 0) {
        const double ratio = rtgt / rsrc;
        double v = 1.0;
        for (int q = 0; q <= P; ++q, v *= ratio) rpow[q] = v;
    }
    __syncthreads();
    const int nt = ncoeff_of(pt);
    for (int t = threadIdx.x; t < nk * nt; t += blockDim.x) {
        const int c = t / nt, s2 = t - c * nt;
        int f, deg;
        if (pt == P) {
            f = __ldg(p2m_sweep<P>.stored + s2);
            deg = T.sdeg[s2];
        } else {
            int i, j, k;
            stored_mi(s2, i, j, k);
            deg = i + j + k;
            f = deg <= P ? full_index(i, j, k) : 0;
        }
        if (deg <= P) {
            z2 &o = tgt[(int64_t)(boxes[b0 + c] - tbase) * nt + s2];
            o = zaxpy(rpow[deg], in[c * NF + f], o);
        }
    }
}

// }}}

// {{{ L2P

constexpr int HL2P_WARPS = 2;

__device__ __forceinline__ z2 h_horner_cube(const z2 *cube, const double *inv, int p, double x,
                                            double y, double z)
{
    z2 tot = zmk(0.0, 0.0);
    for (int i = p; i >= 0; --i) {
        z2 sy = zmk(0.0, 0.0);
        for (int j = p - i; j >= 0; --j) {
            z2 sz = zmk(0.0, 0.0);
            const z2 *row = cube + cube_index(p, i, j, 0);
            for (int k = p - i - j; k >= 0; --k) sz = zaxpy(z * inv[k + 1], sz, row[k]);
            sy = zaxpy(y * inv[j + 1], sy, sz);
        }
        tot = zaxpy(x * inv[i + 1], tot, sy);
    }
    return tot;
}

// E2PFromSingleBox (sumpy/e2p.py:123-226; local.py:284-309): one warp per
// leaf, decompressed cube in shared memory, nested Horner per target;
// result assigned (times the kernel scaling).
__global__ void __launch_bounds__(32 * HL2P_WARPS)
hl2p_kernel(int p, double rscale, double kappa, int32_t nboxes, const int32_t *__restrict__ boxes,
            const double *__restrict__ centers, int64_t cstride, int32_t sbase,
            const z2 *__restrict__ src, const int32_t *__restrict__ bts,
            const int32_t *__restrict__ btc, const double *__restrict__ targets, int64_t tstride,
            double scale, z2 *__restrict__ result, const int32_t *__restrict__ box_level = nullptr,
            const double *__restrict__ level_rscale = nullptr, double k = 0.0)
{
    extern __shared__ __align__(16) double sm[];
    const int P1 = p + 1, C = P1 * P1 * P1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * HL2P_WARPS + warp;
    if (ib >= nboxes) return;
    if (level_rscale) {   // all levels in one launch: the box's own level
        rscale = level_rscale[box_level[ib]];
        kappa = k * k * rscale * rscale;
    }
    z2 *cube = reinterpret_cast<z2 *>(sm) + warp * C;
    double *inv = reinterpret_cast<double *>(reinterpret_cast<z2 *>(sm) + HL2P_WARPS * C) +
                  warp * (P1 + 1);

    const int32_t b = boxes[ib];
    const int n = ncoeff_of(p);
    const z2 *cs = src + (int64_t)(b - sbase) * n;
    for (int s = lane; s < n; s += 32) {
        int i, j, k;
        stored_mi(s, i, j, k);
        cube[cube_index(p, i, j, k)] = cs[s];
    }
    for (int q = lane; q <= p + 1; q += 32) inv[q] = q ? 1.0 / q : 0.0;
    __syncwarp();
    for (int i = 2; i <= p; ++i) {
        const int m = p - i;
        const int npairs = (m + 1) * (m + 2) / 2;
        for (int t = lane; t < npairs; t += 32) {
            int J, K;
            tri_pair(t, m, J, K);
            const z2 u1 = cube[cube_index(p, i - 2, J + 2, K)];
            const z2 u2 = cube[cube_index(p, i - 2, J, K + 2)];
            const z2 u0 = cube[cube_index(p, i - 2, J, K)];
            cube[cube_index(p, i, J, K)] =
                zmk(-u1.x - u2.x - kappa * u0.x, -u1.y - u2.y - kappa * u0.y);
        }
        __syncwarp();
    }
    const double c[3] = {centers[b], centers[cstride + b], centers[2 * cstride + b]};
    const double rinv = 1.0 / rscale;
    const int32_t t0 = bts[b], nt = btc[b];
    for (int32_t tt = lane; tt < nt; tt += 32) {
        const int32_t t = t0 + tt;
        const double x = (targets[t] - c[0]) * rinv;
        const double y = (targets[tstride + t] - c[1]) * rinv;
        const double z = (targets[2 * tstride + t] - c[2]) * rinv;
        result[t] = zscal(scale, h_horner_cube(cube, inv, p, x, y, z));
    }
}

// }}}

// {{{ M2P / P2L (derivatives from the closed form, in registers)

constexpr int HM2P_WARPS = 4;

// E2PFromCSR (List 3; sumpy/e2p.py:233-343, multipole.py:131-157): one warp
// per target box; the box's targets occupy g = next_pow2(nt) lanes and the
// 32/g lane groups stride over the List-3 boxes; each lane sums M[s] D(s)
// with D from helm_layers; shuffle-xor sum; accumulated into result.
template <int P>
__global__ void __launch_bounds__(32 * HM2P_WARPS)
hm2p_reg_kernel(double rscale, double k, int32_t ntgt_boxes,
                const int32_t *__restrict__ target_boxes, const int32_t *__restrict__ src_starts,
                const int32_t *__restrict__ src_lists, const double *__restrict__ centers,
                int64_t cstride, int32_t sbase, const z2 *__restrict__ src,
                const int32_t *__restrict__ bts, const int32_t *__restrict__ btc,
                const double *__restrict__ targets, int64_t tstride, double scale,
                z2 *__restrict__ result)
{
    constexpr int N = (P + 1) * (P + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * HM2P_WARPS + warp;
    if (ib >= ntgt_boxes) return;
    const int32_t tb = target_boxes[ib];
    const int32_t t0 = bts[tb], nt = btc[tb];
    const int32_t ls = src_starts[ib], le = src_starts[ib + 1];
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
        double ar = 0.0, ai = 0.0;
        if (active) {
            for (int32_t l = ls + ph; l < le; l += nph) {
                const int32_t sb = src_lists[l];
                const z2 *M = src + (int64_t)(sb - sbase) * N;
                helm_layers<P>(tx - centers[sb], ty - centers[cstride + sb],
                               tz - centers[2 * cstride + sb], rscale, k,
                               [&](auto sc, z2 v) {
                                   const z2 m = ordered_load<decltype(sc)::value>(M);
                                   ar = fma(m.x, v.x, fma(-m.y, v.y, ar));
                                   ai = fma(m.x, v.y, fma(m.y, v.x, ai));
                                   asm volatile("" : "+d"(ar), "+d"(ai));
                               });
            }
        }
        for (int off = g; off < 32; off <<= 1) {
            ar += __shfl_xor_sync(0xffffffffu, ar, off);
            ai += __shfl_xor_sync(0xffffffffu, ai, off);
        }
        if (active && ph == 0) {
            z2 &o = result[t];
            o = zmk(fma(scale, ar, o.x), fma(scale, ai, o.y));
        }
    }
}

constexpr int HP2L_WARPS = 2;

// P2EFromCSR (List 4; sumpy/p2e.py:268-388, local.py:225-271): one warp per
// target box; the sources of its List-4 boxes are enumerated flat, 32 per
// round, one per lane. The coefficients come out of helm_layers in stored
// order; every 32 of them pass through a per-warp shared tile
// [coefficient][source] (stride 33), where each lane sums its coefficient
// over the round's sources. Accumulated into the box's local.
template <int P>
__global__ void __launch_bounds__(32 * HP2L_WARPS)
hp2l_reg_kernel(double rscale, double k, int32_t ntgt_boxes,
                const int32_t *__restrict__ target_boxes, const int32_t *__restrict__ src_starts,
                const int32_t *__restrict__ src_lists, const double *__restrict__ centers,
                int64_t cstride, const int32_t *__restrict__ bss, const int32_t *__restrict__ bsc,
                const double *__restrict__ sources, int64_t sstride, const z2 *__restrict__ q,
                int32_t tbase, z2 *__restrict__ out)
{
    constexpr int N = (P + 1) * (P + 1);
    constexpr int NPL = (N + 31) / 32;
    __shared__ z2 tile[HP2L_WARPS][32][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * HP2L_WARPS + warp;
    if (ib >= ntgt_boxes) return;
    z2 (*T)[33] = tile[warp];
    const int32_t tb = target_boxes[ib];
    const double c0 = centers[tb], c1 = centers[cstride + tb], c2 = centers[2 * cstride + tb];
    const int32_t ls = src_starts[ib], le = src_starts[ib + 1];
    int32_t total = 0;
    for (int32_t l = ls; l < le; ++l) total += bsc[src_lists[l]];
    z2 acc[NPL];
#pragma unroll
    for (int m = 0; m < NPL; ++m) acc[m] = zmk(0.0, 0.0);
    for (int32_t base = 0; base < total; base += 32) {
        const int nsc = min(32, total - base);
        // inactive lanes evaluate at a harmless point with zero strength
        double x0 = 1.0, x1 = 0.0, x2 = 0.0;
        z2 qq = zmk(0.0, 0.0);
        if (lane < nsc) {
            int32_t f = base + lane, l = ls, sb = src_lists[ls];
            while (f >= bsc[sb]) { f -= bsc[sb]; ++l; sb = src_lists[l]; }
            const int32_t s = bss[sb] + f;
            qq = q[s];
            x0 = c0 - sources[s];
            x1 = c1 - sources[sstride + s];
            x2 = c2 - sources[2 * sstride + s];
        }
        helm_layers<P>(x0, x1, x2, rscale, k, [&](auto sc, z2 v) {
            constexpr int s = decltype(sc)::value;
            T[s & 31][lane] = zmul(qq, v);
            if ((s & 31) == 31 || s == N - 1) {
                __syncwarp();
                const int row = lane;
                if ((s & ~31) + row <= s) {
                    double sr = 0.0, si = 0.0;
                    for (int l2 = 0; l2 < nsc; ++l2) {
                        const z2 w = T[row][l2];
                        sr += w.x;
                        si += w.y;
                    }
                    acc[s >> 5] = zadd(acc[s >> 5], zmk(sr, si));
                }
                __syncwarp();
            }
        });
    }
    z2 *o = out + (int64_t)(tb - tbase) * N;
#pragma unroll
    for (int m = 0; m < NPL; ++m) {
        const int kk = lane + 32 * m;
        if (kk < N) o[kk] = zadd(o[kk], acc[m]);
    }
}

template <int P>
int launch_hm2p(double rscale, double k, int32_t ntgt_boxes, const int32_t *target_boxes,
                const int32_t *src_starts, const int32_t *src_lists, const double *centers,
                int64_t cstride, int32_t sbase, const z2 *src, const int32_t *bts,
                const int32_t *btc, const double *targets, int64_t tstride, double scale,
                z2 *result, cudaStream_t st)
{
    const int blocks = (ntgt_boxes + HM2P_WARPS - 1) / HM2P_WARPS;
    hm2p_reg_kernel<P><<<blocks, 32 * HM2P_WARPS, 0, st>>>(
        rscale, k, ntgt_boxes, target_boxes, src_starts, src_lists, centers, cstride, sbase, src,
        bts, btc, targets, tstride, scale, result);
    return check_launch("hm2p_reg_kernel");
}

template <int P>
int launch_hp2l(double rscale, double k, int32_t ntgt_boxes, const int32_t *target_boxes,
                const int32_t *src_starts, const int32_t *src_lists, const double *centers,
                int64_t cstride, const int32_t *bss, const int32_t *bsc, const double *sources,
                int64_t sstride, const z2 *q, int32_t tbase, z2 *out, cudaStream_t st)
{
    const int blocks = (ntgt_boxes + HP2L_WARPS - 1) / HP2L_WARPS;
    hp2l_reg_kernel<P><<<blocks, 32 * HP2L_WARPS, 0, st>>>(
        rscale, k, ntgt_boxes, target_boxes, src_starts, src_lists, centers, cstride, bss, bsc,
        sources, sstride, q, tbase, out);
    return check_launch("hp2l_reg_kernel");
}

// }}}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

namespace {

inline const z2 *cz(const double *p) { return reinterpret_cast<const z2 *>(p); }
inline z2 *mz(double *p) { return reinterpret_cast<z2 *>(p); }

template <bool MIXED>
int launch_hp2p(int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *ss,
                const int32_t *sl, const int32_t *bss, const int32_t *bsc, const int32_t *bts,
                const int32_t *btc, const double *sources, int64_t sstride, double k,
                const double *strength, const double *targets, int64_t tstride,
                const int32_t *tts, double scale, double *result, void *stream)
{
    if (ntgt_boxes < 0) return bad_arg("helmholtz p2p: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !ss || !sl || !bss || !bsc || !bts || !btc || !sources || !strength ||
        !targets || !result)
        return bad_arg("helmholtz p2p: null pointer argument");
    const unsigned blocks = (unsigned)((ntgt_boxes + HP2P_WARPS - 1) / HP2P_WARPS);
    hp2p_csr_kernel<MIXED><<<blocks, 32 * HP2P_WARPS, 0, as_stream(stream)>>>(
        ntgt_boxes, target_boxes, ss, sl, bss, bsc, bts, btc, sources, sstride, cz(strength),
        targets, tstride, tts, k, scale, mz(result));
    return check_launch("hp2p_csr_kernel");
}

}  // namespace

extern "C" {

int sumpy_helmholtz_p2p_from_csr_f64(int32_t ntgt_boxes, const int32_t *target_boxes,
                                     const int32_t *source_box_starts,
                                     const int32_t *source_box_lists,
                                     const int32_t *box_source_starts,
                                     const int32_t *box_source_counts_nonchild,
                                     const int32_t *box_target_starts,
                                     const int32_t *box_target_counts_nonchild,
                                     const double *sources, int64_t source_stride, double k,
                                     const double *strength, const double *targets,
                                     int64_t target_stride, const int32_t *target_to_source,
                                     double scale, double *result, void *stream)
{
    return launch_hp2p<false>(ntgt_boxes, target_boxes, source_box_starts, source_box_lists,
                              box_source_starts, box_source_counts_nonchild, box_target_starts,
                              box_target_counts_nonchild, sources, source_stride, k, strength,
                              targets, target_stride, target_to_source, scale, result, stream);
}

int sumpy_helmholtz_p2p_from_csr_mixed(int32_t ntgt_boxes, const int32_t *target_boxes,
                                       const int32_t *source_box_starts,
                                       const int32_t *source_box_lists,
                                       const int32_t *box_source_starts,
                                       const int32_t *box_source_counts_nonchild,
                                       const int32_t *box_target_starts,
                                       const int32_t *box_target_counts_nonchild,
                                       const double *sources, int64_t source_stride, double k,
                                       const double *strength, const double *targets,
                                       int64_t target_stride, const int32_t *target_to_source,
                                       double scale, double *result, void *stream)
{
    return launch_hp2p<true>(ntgt_boxes, target_boxes, source_box_starts, source_box_lists,
                             box_source_starts, box_source_counts_nonchild, box_target_starts,
                             box_target_counts_nonchild, sources, source_stride, k, strength,
                             targets, target_stride, target_to_source, scale, result, stream);
}

int sumpy_helmholtz_p2p_direct_f64(int64_t ntargets, const double *targets, int64_t target_stride,
                                   int64_t nsources, const double *sources,
                                   int64_t source_stride, double k, const double *strength,
                                   const int32_t *target_to_source, double scale, double *result,
                                   void *stream)
{
    if (ntargets < 0 || nsources < 0) return bad_arg("helmholtz p2p_direct: negative size");
    if (ntargets == 0) return SUMPY_OK;
    if (!targets || !result || (nsources > 0 && (!sources || !strength)))
        return bad_arg("helmholtz p2p_direct: null pointer argument");
    const unsigned blocks = (unsigned)((ntargets + HDIRECT_THREADS - 1) / HDIRECT_THREADS);
    hp2p_direct_kernel<<<blocks, HDIRECT_THREADS, 0, as_stream(stream)>>>(
        ntargets, targets, target_stride, nsources, sources, source_stride, cz(strength),
        target_to_source, k, scale, mz(result));
    return check_launch("hp2p_direct_kernel");
}

int sumpy_helmholtz_p2e_from_single_box_f64(int order, double rscale, double k,
                                            int32_t nsrc_boxes, const int32_t *source_boxes,
                                            const double *centers, int64_t center_stride,
                                            const int32_t *box_source_starts,
                                            const int32_t *box_source_counts_nonchild,
                                            const double *sources, int64_t source_stride,
                                            const double *strength, int32_t tgt_base_ibox,
                                            double *tgt_expansions, void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz p2m: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nsrc_boxes < 0) return bad_arg("helmholtz p2m: nsrc_boxes < 0");
    if (nsrc_boxes == 0) return SUMPY_OK;
    if (!source_boxes || !centers || !box_source_starts || !box_source_counts_nonchild ||
        !sources || !strength || !tgt_expansions)
        return bad_arg("helmholtz p2m: null pointer argument");
#define CALL_HP2M(P)                                                                             \
    (hp2m_warp_kernel<P><<<(nsrc_boxes + hp2m_warps<P>() - 1) / hp2m_warps<P>(),                   \
                           32 * hp2m_warps<P>(), 0, as_stream(stream)>>>(                          \
         rscale, k, nsrc_boxes, source_boxes, centers, center_stride, box_source_starts,         \
         box_source_counts_nonchild, sources, source_stride, cz(strength), tgt_base_ibox,        \
         mz(tgt_expansions), nullptr, nullptr),                                                  \
     check_launch("hp2m_warp_kernel"))
    SUMPY_ORDER_SWITCH(order, CALL_HP2M)
#undef CALL_HP2M
}

int sumpy_helmholtz_e2e_from_children_f64(int src_order, int tgt_order, double src_rscale,
                                          double tgt_rscale, double k, int32_t ntgt_boxes,
                                          const int32_t *target_boxes,
                                          const int32_t *box_child_ids, int64_t child_stride,
                                          const double *centers, int64_t center_stride,
                                          int32_t src_base_ibox, const double *src_expansions,
                                          int32_t tgt_base_ibox, double *tgt_expansions,
                                          void *stream)
{
    if (!order_ok(src_order) || !order_ok(tgt_order)) {
        set_last_error("helmholtz m2m: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    if (ntgt_boxes < 0) return bad_arg("helmholtz m2m: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !box_child_ids || !centers || !src_expansions || !tgt_expansions)
        return bad_arg("helmholtz m2m: null pointer argument");
    const int nfull = (tgt_order + 1) * (tgt_order + 2) * (tgt_order + 3) / 6;
    const size_t smem = sizeof(z2) * 16 * nfull + sizeof(double) * 8 * 3 * (tgt_order + 1) +
                        sizeof(uint32_t) * nfull;
    int rc = prepare_smem(hm2m_kernel, smem);
    if (rc) return rc;
    hm2m_kernel<<<ntgt_boxes, HE2E_THREADS, smem, as_stream(stream)>>>(
        src_order, tgt_order, src_rscale, tgt_rscale, k * k * tgt_rscale * tgt_rscale,
        target_boxes, box_child_ids, child_stride, centers, center_stride, src_base_ibox,
        cz(src_expansions), tgt_base_ibox, mz(tgt_expansions));
    return check_launch("hm2m_kernel");
}

int sumpy_helmholtz_e2e_from_parent_f64(int src_order, int tgt_order, double src_rscale,
                                        double tgt_rscale, double k, int32_t ntgt_boxes,
                                        const int32_t *target_boxes, const int32_t *box_parent_ids,
                                        const double *centers, int64_t center_stride,
                                        int32_t src_base_ibox, const double *src_expansions,
                                        int32_t tgt_base_ibox, double *tgt_expansions,
                                        void *stream)
{
    if (!order_ok(src_order) || !order_ok(tgt_order)) {
        set_last_error("helmholtz l2l: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    if (ntgt_boxes < 0) return bad_arg("helmholtz l2l: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !box_parent_ids || !centers || !src_expansions || !tgt_expansions)
        return bad_arg("helmholtz l2l: null pointer argument");
    const unsigned blocks = (unsigned)((ntgt_boxes + HL2L_BOXES - 1) / HL2L_BOXES);
#define CALL_HL2L(P)                                                                             \
    (prepare_smem(hl2l_kernel<P>, sizeof(z2) * 2 * HL2L_BOXES * FullShift<P>::NFULL +            \
                                      sizeof(double) * HL2L_BOXES * 3 * (P + 1))                 \
         ? SUMPY_ELAUNCH                                                                         \
         : (hl2l_kernel<P><<<blocks, HE2E_THREADS,                                               \
                             sizeof(z2) * 2 * HL2L_BOXES * FullShift<P>::NFULL +                 \
                                 sizeof(double) * HL2L_BOXES * 3 * (P + 1),                      \
                             as_stream(stream)>>>(                                               \
                tgt_order, src_rscale, tgt_rscale, k * k * src_rscale * src_rscale, ntgt_boxes, \
                target_boxes, box_parent_ids, centers, center_stride, src_base_ibox,            \
                cz(src_expansions), tgt_base_ibox, mz(tgt_expansions)),                         \
            check_launch("hl2l_kernel")))
    SUMPY_ORDER_SWITCH(src_order, CALL_HL2L)
#undef CALL_HL2L
}

int sumpy_helmholtz_e2p_from_single_box_f64(int order, double rscale, double k,
                                            int32_t ntgt_boxes, const int32_t *target_boxes,
                                            const double *centers, int64_t center_stride,
                                            int32_t src_base_ibox, const double *src_expansions,
                                            const int32_t *box_target_starts,
                                            const int32_t *box_target_counts_nonchild,
                                            const double *targets, int64_t target_stride,
                                            double scale, double *result, void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz l2p: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("helmholtz l2p: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !centers || !src_expansions || !box_target_starts ||
        !box_target_counts_nonchild || !targets || !result)
        return bad_arg("helmholtz l2p: null pointer argument");
    const int P1 = order + 1;
    const size_t smem = (sizeof(z2) * P1 * P1 * P1 + sizeof(double) * (P1 + 1)) * HL2P_WARPS;
    int rc = prepare_smem(hl2p_kernel, smem);
    if (rc) return rc;
    const unsigned blocks = (unsigned)((ntgt_boxes + HL2P_WARPS - 1) / HL2P_WARPS);
    hl2p_kernel<<<blocks, 32 * HL2P_WARPS, smem, as_stream(stream)>>>(
        order, rscale, k * k * rscale * rscale, ntgt_boxes, target_boxes, centers, center_stride,
        src_base_ibox, cz(src_expansions), box_target_starts, box_target_counts_nonchild, targets,
        target_stride, scale, mz(result));
    return check_launch("hl2p_kernel");
}

int sumpy_helmholtz_p2e_from_single_box_levels_f64(
    int order, double k, int32_t nsrc_boxes, const int32_t *source_boxes, const int32_t *box_levels,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength, double *expansions,
    void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz p2m levels: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nsrc_boxes < 0) return bad_arg("helmholtz p2m levels: nsrc_boxes < 0");
    if (nsrc_boxes == 0) return SUMPY_OK;
    if (!source_boxes || !box_levels || !level_rscales || !centers || !box_source_starts ||
        !box_source_counts_nonchild || !sources || !strength || !expansions)
        return bad_arg("helmholtz p2m levels: null pointer argument");
#define CALL_HP2M(P)                                                                             \
    (hp2m_warp_kernel<P><<<(nsrc_boxes + hp2m_warps<P>() - 1) / hp2m_warps<P>(),                   \
                           32 * hp2m_warps<P>(), 0, as_stream(stream)>>>(                          \
         1.0, k, nsrc_boxes, source_boxes, centers, center_stride, box_source_starts,            \
         box_source_counts_nonchild, sources, source_stride, cz(strength), 0, mz(expansions),    \
         box_levels, level_rscales),                                                             \
     check_launch("hp2m_warp_kernel"))
    SUMPY_ORDER_SWITCH(order, CALL_HP2M)
#undef CALL_HP2M
}

int sumpy_helmholtz_e2p_from_single_box_levels_f64(
    int order, double k, int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *box_levels,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const double *src_expansions, const int32_t *box_target_starts,
    const int32_t *box_target_counts_nonchild, const double *targets, int64_t target_stride,
    double scale, double *result, void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz l2p levels: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("helmholtz l2p levels: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !box_levels || !level_rscales || !centers || !src_expansions ||
        !box_target_starts || !box_target_counts_nonchild || !targets || !result)
        return bad_arg("helmholtz l2p levels: null pointer argument");
    const int P1 = order + 1;
    const size_t smem = (sizeof(z2) * P1 * P1 * P1 + sizeof(double) * (P1 + 1)) * HL2P_WARPS;
    int rc = prepare_smem(hl2p_kernel, smem);
    if (rc) return rc;
    const unsigned blocks = (unsigned)((ntgt_boxes + HL2P_WARPS - 1) / HL2P_WARPS);
    hl2p_kernel<<<blocks, 32 * HL2P_WARPS, smem, as_stream(stream)>>>(
        order, 1.0, 0.0, ntgt_boxes, target_boxes, centers, center_stride, 0, cz(src_expansions),
        box_target_starts, box_target_counts_nonchild, targets, target_stride, scale, mz(result),
        box_levels, level_rscales, k);
    return check_launch("hl2p_kernel");
}

int sumpy_helmholtz_e2p_from_csr_f64(int order, double rscale, double k, int32_t ntgt_boxes,
                                     const int32_t *target_boxes, const int32_t *source_box_starts,
                                     const int32_t *source_box_lists, const double *centers,
                                     int64_t center_stride, int32_t src_base_ibox,
                                     const double *src_expansions,
                                     const int32_t *box_target_starts,
                                     const int32_t *box_target_counts_nonchild,
                                     const double *targets, int64_t target_stride, double scale,
                                     double *result, void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz m2p: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("helmholtz m2p: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !source_box_starts || !source_box_lists || !centers ||
        !src_expansions || !box_target_starts || !box_target_counts_nonchild || !targets ||
        !result)
        return bad_arg("helmholtz m2p: null pointer argument");
#define CALL_HM2P(P)                                                                             \
    launch_hm2p<P>(rscale, k, ntgt_boxes, target_boxes, source_box_starts, source_box_lists,     \
                   centers, center_stride, src_base_ibox, cz(src_expansions), box_target_starts, \
                   box_target_counts_nonchild, targets, target_stride, scale, mz(result),        \
                   as_stream(stream))
    SUMPY_ORDER_SWITCH(order, CALL_HM2P)
#undef CALL_HM2P
}

int sumpy_helmholtz_p2e_from_csr_f64(int order, double rscale, double k, int32_t ntgt_boxes,
                                     const int32_t *target_boxes, const int32_t *source_box_starts,
                                     const int32_t *source_box_lists, const double *centers,
                                     int64_t center_stride, const int32_t *box_source_starts,
                                     const int32_t *box_source_counts_nonchild,
                                     const double *sources, int64_t source_stride,
                                     const double *strength, int32_t tgt_base_ibox,
                                     double *tgt_expansions, void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz p2l: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (ntgt_boxes < 0) return bad_arg("helmholtz p2l: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !source_box_starts || !source_box_lists || !centers ||
        !box_source_starts || !box_source_counts_nonchild || !sources || !strength ||
        !tgt_expansions)
        return bad_arg("helmholtz p2l: null pointer argument");
#define CALL_HP2L(P)                                                                             \
    launch_hp2l<P>(rscale, k, ntgt_boxes, target_boxes, source_box_starts, source_box_lists,     \
                   centers, center_stride, box_source_starts, box_source_counts_nonchild,        \
                   sources, source_stride, cz(strength), tgt_base_ibox, mz(tgt_expansions),      \
                   as_stream(stream))
    SUMPY_ORDER_SWITCH(order, CALL_HP2L)
#undef CALL_HP2L
}

}  // extern "C"
