// Laplace M2P (List 3, E2PFromCSR: sumpy/e2p.py:231-334 driven by
// sumpy/fmm.py:645-676) and P2L (List 4, P2EFromCSR: sumpy/p2e.py:186-264
// driven by sumpy/fmm.py:678-711) of all levels in one launch each, FP64
// throughout: the FP64 forms of the mixed item kernels in expansions.cu.
//
// The host cuts the work into items of a few rounds each over every level,
// longest first (the per-level launches leave the GPU idle behind a box
// with a long list and run the levels one after another); the items of one
// target box add their partial sums with FP64 atomics. Multipoles and
// locals are the flat [nboxes][(P+1)^2] arrays of a uniform-order FMM.
#include "common.cuh"
#include "derivs.cuh"
#include "taylor.cuh"

namespace sumpy {
namespace {

constexpr int LI_WARPS = 4;     // M2P warps per CTA
constexpr int LP2L_WARPS = 2;   // P2L warps per CTA (N x 33 doubles of shared memory each)
constexpr int LDSTRIDE = 33;    // lanes per coefficient row + 1 (bank spread)

// item = {first target, first List-3 entry, number of List-3 boxes,
//         targets (1..32) | source level << 8}; the chunk's targets take
// g = next_pow2(ntc) lanes, the 32 / g lane groups stride over the boxes.
// GRAD: the target gradient d/dt D[mi] = D[mi + e_d] / rscale from layers one
// degree higher, with D on (2, j, k) = -D(0, j+2, k) - D(0, j, k+2).
template <int P, bool GRAD>
__global__ void __launch_bounds__(32 * LI_WARPS)
m2p_items_f64_kernel(int32_t nitems, const int4 *__restrict__ items,
                     const double *__restrict__ level_rscale, const int32_t *__restrict__ src_lists,
                     const double *__restrict__ centers, int64_t cstride,
                     const double *__restrict__ mpoles, const double *__restrict__ targets,
                     int64_t tstride, double scale, double *__restrict__ result,
                     double *__restrict__ grad)
{
    constexpr int N = (P + 1) * (P + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * LI_WARPS + warp;
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
    const double rs = level_rscale[lev], Rinv = 1.0 / rs;
    double acc = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    if (active) {
        const double tx = targets[t], ty = targets[tstride + t], tz = targets[2 * tstride + t];
        for (int k = ph; k < nb; k += nph) {
            const int32_t sb = src_lists[l0 + k];
            const double *M = mpoles + (int64_t)sb * N;
            laplace_layers<GRAD ? P + 1 : P>(
                tx - centers[sb], ty - centers[cstride + sb], tz - centers[2 * cstride + sb], rs,
                Rinv, [&](int s, int i, int j, int kk, double v) {
                    const int deg = i + j + kk;
                    if (deg <= P) acc = fma(__ldg(M + s), v, acc);
                    if (GRAD && deg >= 1) {
                        if (j >= 1) gy = fma(__ldg(M + stored_index(i, j - 1, kk)), v, gy);
                        if (kk >= 1) gz = fma(__ldg(M + stored_index(i, j, kk - 1)), v, gz);
                        if (i == 1) {
                            gx = fma(__ldg(M + stored_index(0, j, kk)), v, gx);
                        } else {
                            if (j >= 2) gx = fma(-__ldg(M + stored_index(1, j - 2, kk)), v, gx);
                            if (kk >= 2) gx = fma(-__ldg(M + stored_index(1, j, kk - 2)), v, gx);
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
        if (result) atomicAdd(result + t, scale * acc);
        if (GRAD) {
            const double gs = scale * Rinv;
            atomicAdd(grad + t, gs * gx);
            atomicAdd(grad + tstride + t, gs * gy);
            atomicAdd(grad + 2 * tstride + t, gs * gz);
        }
    }
}

// P2L item = {target box, first entry of the flat List-4 source index
// array, number of sources, target level}: 32 sources per round, one per
// lane; each lane writes q D of its source into the warp's shared transpose
// and every lane then sums its coefficients over the round's sources.
template <int P>
__global__ void __launch_bounds__(32 * LP2L_WARPS)
p2l_items_f64_kernel(int32_t nitems, const int4 *__restrict__ items,
                     const double *__restrict__ level_rscale, const int32_t *__restrict__ src_index,
                     const double *__restrict__ centers, int64_t cstride,
                     const double *__restrict__ sources, int64_t sstride,
                     const double *__restrict__ q, double *__restrict__ out)
{
    constexpr int N = (P + 1) * (P + 1);
    constexpr int NPL = (N + 31) / 32;
    extern __shared__ double smd[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * LP2L_WARPS + warp;
    if (it >= nitems) return;
    double *D = smd + warp * (N * LDSTRIDE);
    const int4 item = items[it];
    const int32_t tb = item.x, f0 = item.y, cnt = item.z, lev = item.w;
    const double c0 = centers[tb], c1 = centers[cstride + tb], c2 = centers[2 * cstride + tb];
    const double rs = level_rscale[lev], Rinv = 1.0 / rs;
    double acc[NPL];
#pragma unroll
    for (int m = 0; m < NPL; ++m) acc[m] = 0.0;
    for (int32_t base = 0; base < cnt; base += 32) {
        const int nsc = min(32, cnt - base);
        if (lane < nsc) {
            const int32_t s = src_index[f0 + base + lane];
            const double qq = q[s];
            laplace_layers<P>(c0 - sources[s], c1 - sources[sstride + s],
                              c2 - sources[2 * sstride + s], rs, Rinv,
                              [&](int k, int, int, int, double v) { D[k * LDSTRIDE + lane] = qq * v; });
        }
        __syncwarp();
#pragma unroll
        for (int m = 0; m < NPL; ++m) {
            const int k = lane + 32 * m;
            if (k < N) {
                double sum = 0.0;
                for (int l2 = 0; l2 < nsc; ++l2) sum += D[k * LDSTRIDE + l2];
                acc[m] += sum;
            }
        }
        __syncwarp();
    }
    double *o = out + (int64_t)tb * N;
#pragma unroll
    for (int m = 0; m < NPL; ++m) {
        const int k = lane + 32 * m;
        if (k < N) atomicAdd(o + k, acc[m]);
    }
}

template <bool GRAD>
int launch_m2p_items_f64(int order, int32_t nitems, const int32_t *items,
                         const double *level_rscales, const int32_t *source_box_lists,
                         const double *centers, int64_t center_stride,
                         const double *src_expansions, const double *targets,
                         int64_t target_stride, double scale, double *result, double *grad,
                         void *stream)
{
    if (!order_ok(order)) { set_last_error("m2p items f64: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("m2p items f64: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !level_rscales || !source_box_lists || !centers || !src_expansions ||
        !targets || (GRAD ? !grad : !result))
        return bad_arg("m2p items f64: null pointer argument");
    if (reinterpret_cast<uintptr_t>(items) & 15)
        return bad_arg("m2p items f64: items must be 16-byte aligned");
    const int blocks = (nitems + LI_WARPS - 1) / LI_WARPS;
#define CALL_M2PIF(P)                                                                            \
    (m2p_items_f64_kernel<P, GRAD><<<blocks, 32 * LI_WARPS, 0, as_stream(stream)>>>(              \
         nitems, reinterpret_cast<const int4 *>(items), level_rscales, source_box_lists, centers, \
         center_stride, src_expansions, targets, target_stride, scale, result, grad),            \
     check_launch("m2p_items_f64_kernel"))
    SUMPY_ORDER_SWITCH(order, CALL_M2PIF)
#undef CALL_M2PIF
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_e2p_from_items_f64(int order, int32_t nitems, const int32_t *items,
                             const double *level_rscales, const int32_t *source_box_lists,
                             const double *centers, int64_t center_stride,
                             const double *src_expansions, const double *targets,
                             int64_t target_stride, double scale, double *result, void *stream)
{
    return launch_m2p_items_f64<false>(order, nitems, items, level_rscales, source_box_lists,
                                       centers, center_stride, src_expansions, targets,
                                       target_stride, scale, result, nullptr, stream);
}

int sumpy_e2p_from_items_grad_f64(int order, int32_t nitems, const int32_t *items,
                                  const double *level_rscales, const int32_t *source_box_lists,
                                  const double *centers, int64_t center_stride,
                                  const double *src_expansions, const double *targets,
                                  int64_t target_stride, double scale, double *result,
                                  double *grad, void *stream)
{
    return launch_m2p_items_f64<true>(order, nitems, items, level_rscales, source_box_lists,
                                      centers, center_stride, src_expansions, targets,
                                      target_stride, scale, result, grad, stream);
}

int sumpy_p2e_from_items_f64(int order, int32_t nitems, const int32_t *items,
                             const double *level_rscales, const int32_t *source_index,
                             const double *centers, int64_t center_stride,
                             const double *sources, int64_t source_stride,
                             const double *strength, double *tgt_expansions, void *stream)
{
    if (!order_ok(order)) { set_last_error("p2l items f64: unsupported order"); return SUMPY_EUNSUPPORTED; }
    if (nitems < 0) return bad_arg("p2l items f64: nitems < 0");
    if (nitems == 0) return SUMPY_OK;
    if (!items || !level_rscales || !source_index || !centers || !sources || !strength ||
        !tgt_expansions)
        return bad_arg("p2l items f64: null pointer argument");
    if (reinterpret_cast<uintptr_t>(items) & 15)
        return bad_arg("p2l items f64: items must be 16-byte aligned");
    const int blocks = (nitems + LP2L_WARPS - 1) / LP2L_WARPS;
#define CALL_P2LIF(P)                                                                            \
    (prepare_smem(p2l_items_f64_kernel<P>,                                                       \
                  sizeof(double) * (P + 1) * (P + 1) * LDSTRIDE * LP2L_WARPS)                    \
         ? SUMPY_ELAUNCH                                                                         \
         : (p2l_items_f64_kernel<P><<<blocks, 32 * LP2L_WARPS,                                   \
                                      sizeof(double) * (P + 1) * (P + 1) * LDSTRIDE * LP2L_WARPS, \
                                      as_stream(stream)>>>(                                      \
                nitems, reinterpret_cast<const int4 *>(items), level_rscales, source_index,     \
                centers, center_stride, sources, source_stride, strength, tgt_expansions),      \
            check_launch("p2l_items_f64_kernel")))
    SUMPY_ORDER_SWITCH(order, CALL_P2LIF)
#undef CALL_P2LIF
}

}  // extern "C"
