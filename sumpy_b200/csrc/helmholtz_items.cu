// Helmholtz List 3 (M2P) and List 4 (P2L) of all levels in one launch each,
// over work items cut by the host -- the one-launch form of the per-level
// hm2p_reg_kernel / hp2l_reg_kernel in helmholtz.cu (same arithmetic per
// (target, box) and per (box, source)): a target box with a long list no
// longer runs alone at the end of its level, and the levels do not wait for
// one another. Items of one target box add their sums with FP64 atomics.
// Expansions are the flat [nboxes][(order+1)^2] complex arrays (one order
// on every level).
#include "common.cuh"
#include "helmholtz_core.cuh"
#include "taylor.cuh"

namespace sumpy {
namespace {

constexpr int HITEM_WARPS = 4;   // M2P items per CTA
constexpr int HP2LI_WARPS = 2;   // P2L items per CTA (a 33.8 KB shared tile each)

// item = {first target, first List-3 entry, number of List-3 boxes,
//         targets (1..32) | source level << 8}; the item's targets take
// g = next_pow2(ntc) lanes and its boxes go to the 32/g lane groups in turn.
template <int P>
__global__ void __launch_bounds__(32 * HITEM_WARPS)
hm2p_items_kernel(int32_t nitems, const int4 *__restrict__ items,
                  const double *__restrict__ level_rscale, double k,
                  const int32_t *__restrict__ src_lists, const double *__restrict__ centers,
                  int64_t cstride, const z2 *__restrict__ src, const double *__restrict__ targets,
                  int64_t tstride, double scale, double *__restrict__ result)
{
    constexpr int N = (P + 1) * (P + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * HITEM_WARPS + warp;
    if (it >= nitems) return;
    const int4 item = items[it];
    const int32_t t0 = item.x, l0 = item.y, nb = item.z;
    const int ntc = item.w & 0xff, lev = item.w >> 8;
    int g = 1;
    while (g < ntc) g <<= 1;
    const int nph = 32 / g;
    const int tl = lane & (g - 1), ph = lane / g;
    const bool active = tl < ntc;
    const int32_t t = t0 + tl;
    const double rs = level_rscale[lev];
    double ar = 0.0, ai = 0.0;
    if (active) {
        const double tx = targets[t], ty = targets[tstride + t], tz = targets[2 * tstride + t];
        for (int32_t l = l0 + ph; l < l0 + nb; l += nph) {
            const int32_t sb = src_lists[l];
            const z2 *M = src + (int64_t)sb * N;
            helm_layers<P>(tx - centers[sb], ty - centers[cstride + sb],
                           tz - centers[2 * cstride + sb], rs, k, [&](auto sc, z2 v) {
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
        atomicAdd(result + 2 * (int64_t)t, scale * ar);
        atomicAdd(result + 2 * (int64_t)t + 1, scale * ai);
    }
}

// item = {target box, first entry of the flat List-4 source index array,
// number of sources, target level}: 32 sources per round, one per lane;
// each 32 coefficients of D pass through a per-warp shared tile
// [coefficient][source] (stride 33) where each lane sums its coefficient
// over the round's sources.
template <int P>
__global__ void __launch_bounds__(32 * HP2LI_WARPS)
hp2l_items_kernel(int32_t nitems, const int4 *__restrict__ items,
                  const double *__restrict__ level_rscale, double k,
                  const int32_t *__restrict__ src_index, const double *__restrict__ centers,
                  int64_t cstride, const double *__restrict__ sources, int64_t sstride,
                  const z2 *__restrict__ q, double *__restrict__ out)
{
    constexpr int N = (P + 1) * (P + 1);
    constexpr int NPL = (N + 31) / 32;
    __shared__ z2 tile[HP2LI_WARPS][32][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * HP2LI_WARPS + warp;
    if (it >= nitems) return;
    z2 (*T)[33] = tile[warp];
    const int4 item = items[it];
    const int32_t tb = item.x, f0 = item.y, cnt = item.z, lev = item.w;
    const double c0 = centers[tb], c1 = centers[cstride + tb], c2 = centers[2 * cstride + tb];
    const double rs = level_rscale[lev];
    z2 acc[NPL];
#pragma unroll
    for (int m = 0; m < NPL; ++m) acc[m] = zmk(0.0, 0.0);
    for (int32_t base = 0; base < cnt; base += 32) {
        const int nsc = min(32, cnt - base);
        // inactive lanes evaluate at a harmless point with zero strength
        double x0 = 1.0, x1 = 0.0, x2 = 0.0;
        z2 qq = zmk(0.0, 0.0);
        if (lane < nsc) {
            const int32_t s = src_index[f0 + base + lane];
            qq = q[s];
            x0 = c0 - sources[s];
            x1 = c1 - sources[sstride + s];
            x2 = c2 - sources[2 * sstride + s];
        }
        helm_layers<P>(x0, x1, x2, rs, k, [&](auto sc, z2 v) {
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
    double *o = out + 2 * (int64_t)tb * N;
#pragma unroll
    for (int m = 0; m < NPL; ++m) {
        const int kk = lane + 32 * m;
        if (kk < N) {
            atomicAdd(o + 2 * kk, acc[m].x);
            atomicAdd(o + 2 * kk + 1, acc[m].y);
        }
    }
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_helmholtz_e2p_from_items_f64(int order, double k, int32_t nitems, const int32_t *items,
                                       const double *level_rscales,
                                       const int32_t *source_box_lists, const double *centers,
                                       int64_t center_stride, const double *src_expansions,
                                       const double *targets, int64_t target_stride,
                                       double scale, double *result, void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz m2p items: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("helmholtz m2p items: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !level_rscales || !source_box_lists || !centers || !src_expansions ||
        !targets || !result)
        return bad_arg("helmholtz m2p items: null pointer argument");
    if ((reinterpret_cast<uintptr_t>(items) | reinterpret_cast<uintptr_t>(src_expansions)) & 15)
        return bad_arg("helmholtz m2p items: items and expansions must be 16-byte aligned");
    const int blocks = (nitems + HITEM_WARPS - 1) / HITEM_WARPS;
#define CALL_HM2PI(P)                                                                            \
    (hm2p_items_kernel<P><<<blocks, 32 * HITEM_WARPS, 0, as_stream(stream)>>>(                  \
         nitems, reinterpret_cast<const int4 *>(items), level_rscales, k, source_box_lists,    \
         centers, center_stride, reinterpret_cast<const z2 *>(src_expansions), targets,        \
         target_stride, scale, result),                                                        \
     check_launch("hm2p_items_kernel"))
    SUMPY_ORDER_SWITCH(order, CALL_HM2PI)
#undef CALL_HM2PI
}

int sumpy_helmholtz_p2e_from_items_f64(int order, double k, int32_t nitems, const int32_t *items,
                                       const double *level_rscales, const int32_t *source_index,
                                       const double *centers, int64_t center_stride,
                                       const double *sources, int64_t source_stride,
                                       const double *strength, double *tgt_expansions,
                                       void *stream)
{
    if (!order_ok(order)) { set_last_error("helmholtz p2l items: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("helmholtz p2l items: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !level_rscales || !source_index || !centers || !sources || !strength ||
        !tgt_expansions)
        return bad_arg("helmholtz p2l items: null pointer argument");
    if ((reinterpret_cast<uintptr_t>(items) | reinterpret_cast<uintptr_t>(strength)) & 15)
        return bad_arg("helmholtz p2l items: items and strengths must be 16-byte aligned");
    const int blocks = (nitems + HP2LI_WARPS - 1) / HP2LI_WARPS;
#define CALL_HP2LI(P)                                                                            \
    (hp2l_items_kernel<P><<<blocks, 32 * HP2LI_WARPS, 0, as_stream(stream)>>>(                  \
         nitems, reinterpret_cast<const int4 *>(items), level_rscales, k, source_index,        \
         centers, center_stride, sources, source_stride,                                        \
         reinterpret_cast<const z2 *>(strength), tgt_expansions),                               \
     check_launch("hp2l_items_kernel"))
    SUMPY_ORDER_SWITCH(order, CALL_HP2LI)
#undef CALL_HP2LI
}

}  // extern "C"
