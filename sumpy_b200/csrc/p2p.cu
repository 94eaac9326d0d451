// Near-field (List 1) and all-pairs P2P for the 3D Laplace kernel.
//
// P2PFromCSR (sumpy/p2p.py:484-799): for each target box, the sources of
// the boxes in its CSR list. Layout on the GPU: one warp per target box.
// A box holds at most a few dozen targets, so the warp is split into
// `phases`: the targets of a chunk occupy g = next_pow2(ntargets) lanes and
// the 32/g phases stride over the sources; a shuffle-xor tree sums the
// phases at the end. Sources are staged per warp in shared memory, 32 at a
// time, with coalesced loads. Results are assigned (p2p.py:617).
#include "common.cuh"

namespace sumpy {
namespace {

constexpr int P2P_WARPS = 8;

struct SrcPt {
    double x, y, z, q;
};

template <bool MIXED, bool GRAD = false>
__global__ void __launch_bounds__(32 * P2P_WARPS)
p2p_csr_kernel(int32_t ntgt_boxes, const int32_t *__restrict__ target_boxes,
               const int32_t *__restrict__ src_box_starts, const int32_t *__restrict__ src_box_lists,
               const int32_t *__restrict__ box_src_starts, const int32_t *__restrict__ box_src_counts,
               const int32_t *__restrict__ box_tgt_starts, const int32_t *__restrict__ box_tgt_counts,
               const double *__restrict__ sources, int64_t sstride, const double *__restrict__ strength,
               const double *__restrict__ targets, int64_t tstride,
               const int32_t *__restrict__ target_to_source, double scale, double *__restrict__ result,
               double *__restrict__ grad = nullptr)
{
    __shared__ SrcPt buf[P2P_WARPS][32];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int ib = blockIdx.x * P2P_WARPS + warp;
    if (ib >= ntgt_boxes) return;  // whole warp leaves together
    SrcPt *wb = buf[warp];

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
        double acc = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        for (int32_t l = ls; l < le; ++l) {
            const int32_t sb = src_box_lists[l];
            const int32_t s0 = box_src_starts[sb];
            const int32_t ns = box_src_counts[sb];
            float accf = 0.f, gxf = 0.f, gyf = 0.f, gzf = 0.f;
            for (int32_t sc = 0; sc < ns; sc += 32) {
                const int nsc = min(32, ns - sc);
                if (lane < nsc) {
                    const int32_t s = s0 + sc + lane;
                    wb[lane].x = sources[s];
                    wb[lane].y = sources[sstride + s];
                    wb[lane].z = sources[2 * sstride + s];
                    wb[lane].q = strength[s];
                }
                __syncwarp();
                if (active) {
                    for (int j = ph; j < nsc; j += nph) {
                        const int32_t s = s0 + sc + j;
                        if (s == self) continue;
                        const SrcPt sp = wb[j];
                        if (MIXED) {
                            const float dx = (float)(tx - sp.x);
                            const float dy = (float)(ty - sp.y);
                            const float dz = (float)(tz - sp.z);
                            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            const float ri = rsqrtf(r2);
                            const float qr = (float)sp.q * ri;
                            accf += qr;
                            if (GRAD) {
                                // d/dt (q/|t-s|) = -q (t-s)/|t-s|^3
                                const float w = qr * ri * ri;
                                gxf = fmaf(-w, dx, gxf);
                                gyf = fmaf(-w, dy, gyf);
                                gzf = fmaf(-w, dz, gzf);
                            }
                        } else {
                            const double dx = tx - sp.x, dy = ty - sp.y, dz = tz - sp.z;
                            const double r2 = dx * dx + dy * dy + dz * dz;
                            const double ri = rsqrt(r2);
                            const double qr = sp.q * ri;
                            acc += qr;
                            if (GRAD) {
                                const double w = qr * ri * ri;
                                gx -= w * dx;
                                gy -= w * dy;
                                gz -= w * dz;
                            }
                        }
                    }
                }
                __syncwarp();
            }
            if (MIXED) {
                acc += (double)accf;
                if (GRAD) { gx += (double)gxf; gy += (double)gyf; gz += (double)gzf; }
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
            if (result) result[t] = scale * acc;
            if (GRAD) {
                grad[t] = scale * gx;
                grad[tstride + t] = scale * gy;
                grad[2 * tstride + t] = scale * gz;
            }
        }
    }
}

constexpr int DIRECT_THREADS = 256;

template <bool GRAD>
__global__ void __launch_bounds__(DIRECT_THREADS)
p2p_direct_kernel(int64_t ntgt, const double *__restrict__ targets, int64_t tstride,
                  int64_t nsrc, const double *__restrict__ sources, int64_t sstride,
                  const double *__restrict__ strength, const int32_t *__restrict__ target_to_source,
                  double scale, double *__restrict__ result, double *__restrict__ grad)
{
    __shared__ SrcPt tile[DIRECT_THREADS];
    const int64_t t = (int64_t)blockIdx.x * DIRECT_THREADS + threadIdx.x;
    const bool active = t < ntgt;
    double tx = 0, ty = 0, tz = 0;
    int64_t self = -1;
    if (active) {
        tx = targets[t];
        ty = targets[tstride + t];
        tz = targets[2 * tstride + t];
        if (target_to_source) self = target_to_source[t];
    }
    double acc = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    for (int64_t s0 = 0; s0 < nsrc; s0 += DIRECT_THREADS) {
        const int64_t s = s0 + threadIdx.x;
        if (s < nsrc) {
            tile[threadIdx.x].x = sources[s];
            tile[threadIdx.x].y = sources[sstride + s];
            tile[threadIdx.x].z = sources[2 * sstride + s];
            tile[threadIdx.x].q = strength[s];
        }
        __syncthreads();
        const int n = (int)min((int64_t)DIRECT_THREADS, nsrc - s0);
        if (active) {
            for (int j = 0; j < n; ++j) {
                if (s0 + j == self) continue;
                const double dx = tx - tile[j].x, dy = ty - tile[j].y, dz = tz - tile[j].z;
                const double ri = rsqrt(dx * dx + dy * dy + dz * dz);
                const double qr = tile[j].q * ri;
                acc += qr;
                if (GRAD) {
                    const double w = qr * ri * ri;
                    gx -= w * dx;
                    gy -= w * dy;
                    gz -= w * dz;
                }
            }
        }
        __syncthreads();
    }
    if (active) {
        if (result) result[t] = scale * acc;
        if (GRAD) {
            grad[t] = scale * gx;
            grad[tstride + t] = scale * gy;
            grad[2 * tstride + t] = scale * gz;
        }
    }
}

template <bool MIXED, bool GRAD = false>
int launch_p2p_csr(int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *ss,
                   const int32_t *sl, const int32_t *bss, const int32_t *bsc, const int32_t *bts,
                   const int32_t *btc, const double *sources, int64_t sstride,
                   const double *strength, const double *targets, int64_t tstride,
                   const int32_t *tts, double scale, double *result, void *stream,
                   double *grad = nullptr)
{
    if (ntgt_boxes < 0) return bad_arg("p2p: ntgt_boxes < 0");
    if (ntgt_boxes == 0) return SUMPY_OK;
    if (!target_boxes || !ss || !sl || !bss || !bsc || !bts || !btc || !sources || !strength ||
        !targets || (!result && !GRAD) || (GRAD && !grad))
        return bad_arg("p2p: null pointer argument");
    const int blocks = (ntgt_boxes + P2P_WARPS - 1) / P2P_WARPS;
    p2p_csr_kernel<MIXED, GRAD><<<blocks, 32 * P2P_WARPS, 0, as_stream(stream)>>>(
        ntgt_boxes, target_boxes, ss, sl, bss, bsc, bts, btc, sources, sstride, strength,
        targets, tstride, tts, scale, result, grad);
    return check_launch("p2p_csr_kernel");
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_p2p_from_csr_f64(int32_t ntgt_boxes, const int32_t *target_boxes,
                           const int32_t *source_box_starts, const int32_t *source_box_lists,
                           const int32_t *box_source_starts,
                           const int32_t *box_source_counts_nonchild,
                           const int32_t *box_target_starts,
                           const int32_t *box_target_counts_nonchild, const double *sources,
                           int64_t source_stride, const double *strength, const double *targets,
                           int64_t target_stride, const int32_t *target_to_source, double scale,
                           double *result, void *stream)
{
    return launch_p2p_csr<false>(ntgt_boxes, target_boxes, source_box_starts, source_box_lists,
                                 box_source_starts, box_source_counts_nonchild, box_target_starts,
                                 box_target_counts_nonchild, sources, source_stride, strength,
                                 targets, target_stride, target_to_source, scale, result, stream);
}

int sumpy_p2p_from_csr_mixed(int32_t ntgt_boxes, const int32_t *target_boxes,
                             const int32_t *source_box_starts, const int32_t *source_box_lists,
                             const int32_t *box_source_starts,
                             const int32_t *box_source_counts_nonchild,
                             const int32_t *box_target_starts,
                             const int32_t *box_target_counts_nonchild, const double *sources,
                             int64_t source_stride, const double *strength, const double *targets,
                             int64_t target_stride, const int32_t *target_to_source, double scale,
                             double *result, void *stream)
{
    return launch_p2p_csr<true>(ntgt_boxes, target_boxes, source_box_starts, source_box_lists,
                                box_source_starts, box_source_counts_nonchild, box_target_starts,
                                box_target_counts_nonchild, sources, source_stride, strength,
                                targets, target_stride, target_to_source, scale, result, stream);
}

int sumpy_p2p_from_csr_grad_f64(int32_t ntgt_boxes, const int32_t *target_boxes,
                                const int32_t *source_box_starts, const int32_t *source_box_lists,
                                const int32_t *box_source_starts,
                                const int32_t *box_source_counts_nonchild,
                                const int32_t *box_target_starts,
                                const int32_t *box_target_counts_nonchild,
                                const double *sources, int64_t source_stride,
                                const double *strength, const double *targets,
                                int64_t target_stride, const int32_t *target_to_source,
                                double scale, double *result, double *grad, void *stream)
{
    return launch_p2p_csr<false, true>(ntgt_boxes, target_boxes, source_box_starts,
                                       source_box_lists, box_source_starts,
                                       box_source_counts_nonchild, box_target_starts,
                                       box_target_counts_nonchild, sources, source_stride,
                                       strength, targets, target_stride, target_to_source, scale,
                                       result, stream, grad);
}

int sumpy_p2p_from_csr_grad_mixed(int32_t ntgt_boxes, const int32_t *target_boxes,
                                  const int32_t *source_box_starts, const int32_t *source_box_lists,
                                  const int32_t *box_source_starts,
                                  const int32_t *box_source_counts_nonchild,
                                  const int32_t *box_target_starts,
                                  const int32_t *box_target_counts_nonchild,
                                  const double *sources, int64_t source_stride,
                                  const double *strength, const double *targets,
                                  int64_t target_stride, const int32_t *target_to_source,
                                  double scale, double *result, double *grad, void *stream)
{
    return launch_p2p_csr<true, true>(ntgt_boxes, target_boxes, source_box_starts,
                                      source_box_lists, box_source_starts,
                                      box_source_counts_nonchild, box_target_starts,
                                      box_target_counts_nonchild, sources, source_stride, strength,
                                      targets, target_stride, target_to_source, scale, result,
                                      stream, grad);
}

int sumpy_p2p_direct_f64(int64_t ntargets, const double *targets, int64_t target_stride,
                         int64_t nsources, const double *sources, int64_t source_stride,
                         const double *strength, const int32_t *target_to_source, double scale,
                         double *result, void *stream)
{
    if (ntargets < 0 || nsources < 0) return bad_arg("p2p_direct: negative size");
    if (ntargets == 0) return SUMPY_OK;
    if (!targets || !result || (nsources > 0 && (!sources || !strength)))
        return bad_arg("p2p_direct: null pointer argument");
    const int64_t blocks = (ntargets + DIRECT_THREADS - 1) / DIRECT_THREADS;
    if (blocks > INT32_MAX) return bad_arg("p2p_direct: too many targets");
    p2p_direct_kernel<false><<<(unsigned)blocks, DIRECT_THREADS, 0, as_stream(stream)>>>(
        ntargets, targets, target_stride, nsources, sources, source_stride, strength,
        target_to_source, scale, result, nullptr);
    return check_launch("p2p_direct_kernel");
}

int sumpy_p2p_direct_grad_f64(int64_t ntargets, const double *targets, int64_t target_stride,
                              int64_t nsources, const double *sources, int64_t source_stride,
                              const double *strength, const int32_t *target_to_source,
                              double scale, double *result, double *grad, void *stream)
{
    if (ntargets < 0 || nsources < 0) return bad_arg("p2p_direct_grad: negative size");
    if (ntargets == 0) return SUMPY_OK;
    if (!targets || !grad || (nsources > 0 && (!sources || !strength)))
        return bad_arg("p2p_direct_grad: null pointer argument");
    const int64_t blocks = (ntargets + DIRECT_THREADS - 1) / DIRECT_THREADS;
    if (blocks > INT32_MAX) return bad_arg("p2p_direct_grad: too many targets");
    p2p_direct_kernel<true><<<(unsigned)blocks, DIRECT_THREADS, 0, as_stream(stream)>>>(
        ntargets, targets, target_stride, nsources, sources, source_stride, strength,
        target_to_source, scale, result, grad);
    return check_launch("p2p_direct_kernel");
}

}  // extern "C"
