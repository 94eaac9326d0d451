// Helmholtz L2P (E2PFromSingleBox, sumpy/e2p.py:123-226; local.py:284-309)
// of all levels in one launch over packed work items: the complex-data
// form of the Laplace l2p_packed_kernel (expansions.cu). Up to 32 targets
// of up to HL2PK_SLOTS boxes per warp; the boxes' stored locals are
// decompressed together with the Helmholtz PDE projection
//     u_mi = -u_{mi-2e0+2e1} - u_{mi-2e0+2e2} - kappa u_{mi-2e0},
//     kappa = k^2 rscale^2 (the box's level)
// (sumpy/expansion/__init__.py:754-886) into the [(j, k)][i] layout, and
// lane l evaluates its target as sum_(j,k) y^j z^k / (j! k!) sum_i
// c[i][j][k] x^i / i! with real power tables in registers and complex
// coefficients (two FMAs per term). Results are assigned.
#include "common.cuh"
#include "helmholtz_core.cuh"
#include "taylor.cuh"
#include "index_tables.cuh"

namespace sumpy {
namespace {

constexpr int HL2PK_SLOTS = 4;   // boxes per warp item

// warps per CTA: two while the slots' coefficients fit in 200 KB, else one
template <int P>
__host__ __device__ constexpr int hl2pk_warps()
{
    return 16 * HL2PK_SLOTS * (P + 1) * (P + 2) * (P + 3) / 6 * 2 <= 200 * 1024 ? 2 : 1;
}

template <int P>
__global__ void __launch_bounds__(32 * hl2pk_warps<P>())
hl2p_packed_kernel(int32_t nitems, const int2 *__restrict__ items, const int4 *__restrict__ slots,
                   const double *__restrict__ level_rscale, double k,
                   const double *__restrict__ centers, int64_t cstride, const z2 *__restrict__ loc,
                   const double *__restrict__ targets, int64_t tstride, double scale,
                   z2 *__restrict__ result)
{
    constexpr int P1 = P + 1;
    constexpr int N = P1 * P1;
    constexpr int NF = P1 * (P1 + 1) * (P1 + 2) / 6;
    extern __shared__ __align__(16) double smh[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * hl2pk_warps<P>() + warp;
    if (it >= nitems) return;
    z2 *cubes = reinterpret_cast<z2 *>(smh) + warp * (HL2PK_SLOTS * NF);
    const int2 item = items[it];
    const int nsl = item.y;
    // the warp's shared memory holds HL2PK_SLOTS slots: an item with more is
    // skipped rather than written past it (the host builds at most that many)
    if (nsl < 0 || nsl > HL2PK_SLOTS) return;

    int my = -1, off = lane;
    int4 sl = make_int4(0, 0, 0, 0);
    for (int q = 0; q < nsl; ++q) {
        const int4 v = slots[item.x + q];
        if (my < 0) {
            if (off < v.z) { my = q; sl = v; } else { off -= v.z; }
        }
    }
    // stored -> full layout, all slots
    for (int e = lane; e < nsl * N; e += 32) {
        const int q = e / N, st = e - q * N;
        const int32_t b = slots[item.x + q].x;
        cubes[q * NF + __ldg(l2p_decomp<P>.stored + st)] = loc[(int64_t)b * N + st];
    }
    // each slot's kappa = k^2 rscale^2 of its level, in every lane
    double kap[HL2PK_SLOTS];
    {
        double mine = 0.0;
        if (lane < nsl) {
            const double rs = level_rscale[slots[item.x + lane].w];
            mine = k * k * rs * rs;
        }
#pragma unroll
        for (int q = 0; q < HL2PK_SLOTS; ++q) kap[q] = __shfl_sync(0xffffffffu, mine, q);
    }
    __syncwarp();
    // decompress: plane i from plane i - 2 (all slots per sweep), each slot
    // with its own level's kappa, by the precomputed offset triples of each
    // plane (the u_{mi-2e0} term sits two places before the destination)
    const int4 *tri = reinterpret_cast<const int4 *>(l2p_decomp<P>.e);
    for (int pl = 0; pl + 2 <= P; ++pl) {
        const int e0 = l2p_decomp<P>.start[pl];
        const int npairs = l2p_decomp<P>.start[pl + 1] - e0;
        for (int e = lane; e < nsl * npairs; e += 32) {
            int q = 0, r = e;
            while (r >= npairs) { r -= npairs; ++q; }
            const int4 o = __ldg(tri + e0 + r);
            double kappa = kap[0];
#pragma unroll
            for (int qq = 1; qq < HL2PK_SLOTS; ++qq)
                if (q == qq) kappa = kap[qq];
            z2 *c = cubes + q * NF;
            const z2 u1 = c[o.y], u2 = c[o.z], u0 = c[o.x - 2];
            c[o.x] = zmk(-u1.x - u2.x - kappa * u0.x, -u1.y - u2.y - kappa * u0.y);
        }
        __syncwarp();
    }
    if (my < 0) return;
    const int32_t b = sl.x, t = sl.y + off;
    const double rinv = 1.0 / level_rscale[sl.w];
    const double x = (targets[t] - centers[b]) * rinv;
    const double y = (targets[tstride + t] - centers[cstride + b]) * rinv;
    const double z = (targets[2 * tstride + t] - centers[2 * cstride + b]) * rinv;
    double xp[P1], yp[P1], zp[P1];
    xp[0] = yp[0] = zp[0] = 1.0;
#pragma unroll
    for (int n = 1; n <= P; ++n) {
        const double inv_n = 1.0 / n;   // compile-time constant
        xp[n] = xp[n - 1] * x * inv_n;
        yp[n] = yp[n - 1] * y * inv_n;
        zp[n] = zp[n - 1] * z * inv_n;
    }
    const z2 *c = cubes + my * NF;
    double pr = 0.0, pi = 0.0;
#pragma unroll
    for (int j = 0; j <= P; ++j) {
        double jr = 0.0, ji = 0.0;
#pragma unroll
        for (int kk = 0; kk <= P - j; ++kk) {
            const z2 *run = c + jki_offset<P>(j, kk);
            double rr = 0.0, ri = 0.0;
#pragma unroll
            for (int i = P - j - kk; i >= 0; --i) {
                const z2 v = run[i];
                rr = fma(v.x, xp[i], rr);
                ri = fma(v.y, xp[i], ri);
            }
            jr = fma(zp[kk], rr, jr);
            ji = fma(zp[kk], ri, ji);
        }
        pr = fma(yp[j], jr, pr);
        pi = fma(yp[j], ji, pi);
    }
    result[t] = zmk(scale * pr, scale * pi);
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_helmholtz_e2p_from_single_box_packed_f64(
    int order, double k, int32_t nitems, const int32_t *items, const int32_t *slots,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const double *src_expansions, const double *targets, int64_t target_stride, double scale,
    double *result, void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz l2p packed: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("helmholtz l2p packed: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !slots || !level_rscales || !centers || !src_expansions || !targets || !result)
        return bad_arg("helmholtz l2p packed: null pointer argument");
    if ((reinterpret_cast<uintptr_t>(items) & 7) || (reinterpret_cast<uintptr_t>(slots) & 15) ||
        ((reinterpret_cast<uintptr_t>(src_expansions) | reinterpret_cast<uintptr_t>(result)) & 15))
        return bad_arg("helmholtz l2p packed: misaligned argument");
#define NF_OF(P) ((P + 1) * (P + 2) * (P + 3) / 6)
#define CALL_HL2PK(P)                                                                            \
    (prepare_smem(hl2p_packed_kernel<P>, sizeof(z2) * HL2PK_SLOTS * NF_OF(P) * hl2pk_warps<P>()) \
         ? SUMPY_ELAUNCH                                                                         \
         : (hl2p_packed_kernel<P><<<(nitems + hl2pk_warps<P>() - 1) / hl2pk_warps<P>(),           \
                                    32 * hl2pk_warps<P>(),                                       \
                                    sizeof(z2) * HL2PK_SLOTS * NF_OF(P) * hl2pk_warps<P>(),      \
                                    as_stream(stream)>>>(                                        \
                nitems, reinterpret_cast<const int2 *>(items),                                  \
                reinterpret_cast<const int4 *>(slots), level_rscales, k, centers,               \
                center_stride, reinterpret_cast<const z2 *>(src_expansions), targets,           \
                target_stride, scale, reinterpret_cast<z2 *>(result)),                          \
            check_launch("hl2p_packed_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_HL2PK)
#undef CALL_HL2PK
#undef NF_OF
}

}  // extern "C"
