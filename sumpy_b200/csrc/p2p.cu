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

template <bool GRAD = false>
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
                        const double dx = tx - sp.x, dy = ty - sp.y, dz = tz - sp.z;
                        const double r2 = dx * dx + dy * dy + dz * dz;
                        const double ri = rsqrt(r2);
                        const double qr = sp.q * ri;
                        acc += qr;
                        if (GRAD) {
                            // d/dt (q/|t-s|) = -q (t-s)/|t-s|^3
                            const double w = qr * ri * ri;
                            gx -= w * dx;
                            gy -= w * dy;
                            gz -= w * dz;
                        }
                    }
                }
                __syncwarp();
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

// {{{ mixed-precision List 1 over a flat source sequence

// The mixed form above costs three FP64 subtractions and four FP64->FP32
// conversions per pair, and stages each source box separately (a 33-source
// box is a batch of 32 and a batch of 1). Here each coordinate is split once
// per staged source into hi + lo FP32 parts (x = hi + lo to ~2^-48
// relative), so a pair's offset (t_hi - s_hi) + (t_lo - s_lo) is FP32
// arithmetic accurate to a few FP32 ulps of the offset itself; the sources of
// all boxes in a target box's list form one flat sequence (a warp prefix sum
// over up to 32 list entries per window), staged 32 at a time into a
// double-buffered shared slot while the next batch's loads are in flight; a
// short last batch is padded with zero-strength sources far away (1e18), so
// every batch is 32 sources. Targets: a chunk of ntc <= 32 targets takes
// ntc lanes per phase and 32 / ntc phases, phase ph taking the batch's
// sources j = ph (mod phases). Self-interaction is tested only in batches
// that hold some lane's own source. Per batch the FP32 partial sums are
// added into FP64.
constexpr int P2PF_WARPS = 8;
constexpr float P2PF_FAR = 1e18f;
#ifndef SUMPY_P2PF_MINB
#define SUMPY_P2PF_MINB 3   // CTAs per SM the value kernel is built for (register cap 85)
#endif

__device__ __forceinline__ void split_hl(double v, float &hi, float &lo)
{
    hi = __double2float_rn(v);
    lo = __double2float_rn(v - (double)hi);
}

struct P2PTarget {
    float xh, xl, yh, yl, zh, zl;
};

// 1/sqrt(x) by the MUFU approximation, denormal inputs flushed (PTX
// rsqrt.approx.ftz.f32, relative error below 2^-22): r^2 of a List-1 pair
// is zero (excluded self pair) or far above the FP32 denormal range
__device__ __forceinline__ float rsqrt_ftz(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// sources j = j0, j0 + step, ... < 32 of one staged batch against one target
template <bool CHECK, bool GRAD, int STEP>
__device__ __forceinline__ void p2p_batch(const float4 *__restrict__ hi, const float4 *__restrict__ lo,
                                          const P2PTarget &t, int j0, int step, int jself,
                                          float &acc, float &gx, float &gy, float &gz)
{
    const int st = STEP ? STEP : step;
#pragma unroll(STEP ? 32 : 4)
    for (int j = j0; j < 32; j += st) {
        const float4 h = hi[j];
        const float4 l = lo[j];
        const float dx = (t.xh - h.x) + (t.xl - l.x);
        const float dy = (t.yh - h.y) + (t.yl - l.y);
        const float dz = (t.zh - h.z) + (t.zl - l.z);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float ri = rsqrt_ftz(r2);
        if (CHECK && j == jself) continue;
        if (GRAD) {
            // d/dt (q/|t-s|) = -q (t-s)/|t-s|^3
            const float qr = h.w * ri;
            const float w = qr * ri * ri;
            acc += qr;
            gx = fmaf(-w, dx, gx);
            gy = fmaf(-w, dy, gy);
            gz = fmaf(-w, dz, gz);
        } else {
            acc = fmaf(h.w, ri, acc);
        }
    }
}

// The same for all 32 sources against one target, two sources per
// instruction with the packed FP32 pairs of sm_100 (FADD2 / FMUL2 / FFMA2):
// source pair m holds sources 2m and 2m + 1 as {-x_hi, -y_hi} {-z_hi, q}
// {-x_lo, -y_lo} {-z_lo, -} (float2 halves); per pair the same roundings as
// p2p_batch, the sum kept as two partial sums.
__device__ __forceinline__ void p2p_batch_packed(const float4 *__restrict__ P0,
                                                 const float4 *__restrict__ P1,
                                                 const float4 *__restrict__ P2,
                                                 const float4 *__restrict__ P3,
                                                 const P2PTarget &t, float &acc)
{
    const float2 txh = make_float2(t.xh, t.xh), txl = make_float2(t.xl, t.xl);
    const float2 tyh = make_float2(t.yh, t.yh), tyl = make_float2(t.yl, t.yl);
    const float2 tzh = make_float2(t.zh, t.zh), tzl = make_float2(t.zl, t.zl);
    float2 a2 = make_float2(0.f, 0.f);
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const float4 p0 = P0[m], p1 = P1[m], p2 = P2[m], p3 = P3[m];
        const float2 dx = __fadd2_rn(__fadd2_rn(txh, make_float2(p0.x, p0.y)),
                                     __fadd2_rn(txl, make_float2(p2.x, p2.y)));
        const float2 dy = __fadd2_rn(__fadd2_rn(tyh, make_float2(p0.z, p0.w)),
                                     __fadd2_rn(tyl, make_float2(p2.z, p2.w)));
        const float2 dz = __fadd2_rn(__fadd2_rn(tzh, make_float2(p1.x, p1.y)),
                                     __fadd2_rn(tzl, make_float2(p3.x, p3.y)));
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
        a2 = __ffma2_rn(make_float2(p1.z, p1.w), ri, a2);
    }
    acc += a2.x + a2.y;
}

// The same for a target shared by nph lanes (nph = 32 / targets in the pass,
// boxes of at most 16 targets): the lane of phase ph takes the staged source
// pairs ph, ph + nph, ... (every pair in exactly one phase), two sources per
// instruction like p2p_batch_packed; padding sources are far away with
// q = 0.
__device__ __forceinline__ void p2p_batch_packed_phased(const float4 *__restrict__ P0,
                                                        const float4 *__restrict__ P1,
                                                        const float4 *__restrict__ P2,
                                                        const float4 *__restrict__ P3,
                                                        const P2PTarget &t, int ph, int nph,
                                                        float &acc)
{
    const float2 txh = make_float2(t.xh, t.xh), txl = make_float2(t.xl, t.xl);
    const float2 tyh = make_float2(t.yh, t.yh), tyl = make_float2(t.yl, t.yl);
    const float2 tzh = make_float2(t.zh, t.zh), tzl = make_float2(t.zl, t.zl);
    float2 a2 = make_float2(0.f, 0.f);
#pragma unroll 4
    for (int m = ph; m < 16; m += nph) {
        const float4 p0 = P0[m], p1 = P1[m], p2 = P2[m], p3 = P3[m];
        const float2 dx = __fadd2_rn(__fadd2_rn(txh, make_float2(p0.x, p0.y)),
                                     __fadd2_rn(txl, make_float2(p2.x, p2.y)));
        const float2 dy = __fadd2_rn(__fadd2_rn(tyh, make_float2(p0.z, p0.w)),
                                     __fadd2_rn(tyl, make_float2(p2.z, p2.w)));
        const float2 dz = __fadd2_rn(__fadd2_rn(tzh, make_float2(p1.x, p1.y)),
                                     __fadd2_rn(tzl, make_float2(p3.x, p3.y)));
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
        a2 = __ffma2_rn(make_float2(p1.z, p1.w), ri, a2);
    }
    acc += a2.x + a2.y;
}

// The same for two targets per lane: each source pair is read from shared
// memory once and used for both targets (half the shared loads per pair).
__device__ __forceinline__ void p2p_batch_packed2(const float4 *__restrict__ P0,
                                                  const float4 *__restrict__ P1,
                                                  const float4 *__restrict__ P2,
                                                  const float4 *__restrict__ P3,
                                                  const P2PTarget &t, const P2PTarget &u,
                                                  float &acc, float &acc2)
{
    const float2 txh = make_float2(t.xh, t.xh), txl = make_float2(t.xl, t.xl);
    const float2 tyh = make_float2(t.yh, t.yh), tyl = make_float2(t.yl, t.yl);
    const float2 tzh = make_float2(t.zh, t.zh), tzl = make_float2(t.zl, t.zl);
    const float2 uxh = make_float2(u.xh, u.xh), uxl = make_float2(u.xl, u.xl);
    const float2 uyh = make_float2(u.yh, u.yh), uyl = make_float2(u.yl, u.yl);
    const float2 uzh = make_float2(u.zh, u.zh), uzl = make_float2(u.zl, u.zl);
    float2 a2 = make_float2(0.f, 0.f), b2 = make_float2(0.f, 0.f);
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const float4 p0 = P0[m], p1 = P1[m], p2 = P2[m], p3 = P3[m];
        const float2 sxh = make_float2(p0.x, p0.y), syh = make_float2(p0.z, p0.w);
        const float2 szh = make_float2(p1.x, p1.y), q = make_float2(p1.z, p1.w);
        const float2 sxl = make_float2(p2.x, p2.y), syl = make_float2(p2.z, p2.w);
        const float2 szl = make_float2(p3.x, p3.y);
        {
            const float2 dx = __fadd2_rn(__fadd2_rn(txh, sxh), __fadd2_rn(txl, sxl));
            const float2 dy = __fadd2_rn(__fadd2_rn(tyh, syh), __fadd2_rn(tyl, syl));
            const float2 dz = __fadd2_rn(__fadd2_rn(tzh, szh), __fadd2_rn(tzl, szl));
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            a2 = __ffma2_rn(q, make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y)), a2);
        }
        {
            const float2 dx = __fadd2_rn(__fadd2_rn(uxh, sxh), __fadd2_rn(uxl, sxl));
            const float2 dy = __fadd2_rn(__fadd2_rn(uyh, syh), __fadd2_rn(uyl, syl));
            const float2 dz = __fadd2_rn(__fadd2_rn(uzh, szh), __fadd2_rn(uzl, szl));
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            b2 = __ffma2_rn(q, make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y)), b2);
        }
    }
    acc += a2.x + a2.y;
    acc2 += b2.x + b2.y;
}

template <bool GRAD>
__global__ void __launch_bounds__(32 * P2PF_WARPS, GRAD ? 4 : SUMPY_P2PF_MINB)
p2p_flat_mixed_kernel(int32_t ntgt_boxes, const int32_t *__restrict__ target_boxes,
                      const int32_t *__restrict__ src_box_starts,
                      const int32_t *__restrict__ src_box_lists,
                      const int32_t *__restrict__ box_src_starts,
                      const int32_t *__restrict__ box_src_counts,
                      const int32_t *__restrict__ box_tgt_starts,
                      const int32_t *__restrict__ box_tgt_counts,
                      const double *__restrict__ sources, int64_t sstride,
                      const double *__restrict__ strength, const double *__restrict__ targets,
                      int64_t tstride, const int32_t *__restrict__ target_to_source, double scale,
                      double *__restrict__ result, double *__restrict__ grad)
{
    __shared__ float4 shi[P2PF_WARPS][2][32];   // x, y, z hi parts, q
    __shared__ float4 slo[P2PF_WARPS][2][32];   // x, y, z lo parts
    __shared__ float4 spk[P2PF_WARPS][2][4][16];   // the same as source pairs (packed path)
    __shared__ double red[P2PF_WARPS][GRAD ? 4 : 1][32];
    const unsigned FULL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ib = blockIdx.x * P2PF_WARPS + warp;
    if (ib >= ntgt_boxes) return;  // whole warp leaves together
    const int32_t tb = target_boxes[ib];
    const int32_t t0 = box_tgt_starts[tb], nt = box_tgt_counts[tb];
    const int32_t ls = src_box_starts[ib], le = src_box_starts[ib + 1];

    // more than 32 targets left: a pass of up to 64, two targets per lane
    // (lane l: targets tc + l and tc + 32 + l) sharing each staged source
    for (int32_t tc = 0; tc < nt;) {
        const bool two = !GRAD && nt - tc > 32;
        const int ntc = min(32, nt - tc);
        const int nph = 32 / ntc;
        const int tl = lane % ntc, ph = lane / ntc;
        const bool active = ph < nph;
        const int32_t t = t0 + tc + tl;
        P2PTarget tg = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int32_t self = -1;
        if (active) {
            split_hl(targets[t], tg.xh, tg.xl);
            split_hl(targets[tstride + t], tg.yh, tg.yl);
            split_hl(targets[2 * tstride + t], tg.zh, tg.zl);
            if (target_to_source) self = target_to_source[t];
        }
        // the second target of this lane (far away when the pass has none)
        const bool active2 = two && tc + 32 + lane < nt;
        const int32_t t2 = t0 + tc + 32 + lane;
        P2PTarget tg2 = {P2PF_FAR, 0.f, P2PF_FAR, 0.f, P2PF_FAR, 0.f};
        int32_t self2 = -1;
        if (active2) {
            split_hl(targets[t2], tg2.xh, tg2.xl);
            split_hl(targets[tstride + t2], tg2.yh, tg2.yl);
            split_hl(targets[2 * tstride + t2], tg2.zh, tg2.zl);
            if (target_to_source) self2 = target_to_source[t2];
        }
        double acc = 0.0, acc2 = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        for (int32_t w0 = ls; w0 < le; w0 += 32) {
            // one window of up to 32 list entries: lane k holds entry k's
            // source range; inclusive prefix sum of the counts
            const int nw = min(32, le - w0);
            int32_t bs0 = 0, bn = 0;
            if (lane < nw) {
                const int32_t sb = src_box_lists[w0 + lane];
                bs0 = box_src_starts[sb];
                bn = box_src_counts[sb];
            }
            int32_t cum = bn;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t v = __shfl_up_sync(FULL, cum, o);
                if (lane >= o) cum += v;
            }
            const int32_t S = __shfl_sync(FULL, cum, 31);
            // flat position of this lane's own source in the window, if any
            int32_t fself = -1, fself2 = -1;
            if (target_to_source) {
                for (int k = 0; k < nw; ++k) {
                    const int32_t b0 = __shfl_sync(FULL, bs0, k);
                    const int32_t n = __shfl_sync(FULL, bn, k);
                    const int32_t c = __shfl_sync(FULL, cum, k);
                    if (self >= b0 && self < b0 + n) fself = c - n + (self - b0);
                    if (self2 >= b0 && self2 < b0 + n) fself2 = c - n + (self2 - b0);
                }
            }
            // source of flat index f (f < S): entry k = #lanes with cum <= f
            auto locate = [&](int32_t f) {
                int k = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const int32_t v = __shfl_sync(FULL, cum, k + step - 1);
                    if (v <= f) k += step;
                }
                const int32_t b0 = __shfl_sync(FULL, bs0, k);
                const int32_t c = __shfl_sync(FULL, cum, k);
                const int32_t n = __shfl_sync(FULL, bn, k);
                return b0 + f - (c - n);
            };
            const int nbat = (S + 31) / 32;
            double px = P2PF_FAR, py = P2PF_FAR, pz = P2PF_FAR, pq = 0.0;
            {
                const int32_t s = locate(min(lane, max(S - 1, 0)));
                if (lane < S) {
                    px = sources[s]; py = sources[sstride + s]; pz = sources[2 * sstride + s];
                    pq = strength[s];
                }
            }
            for (int bt = 0; bt < nbat; ++bt) {
                const int slot = bt & 1;
                {
                    float4 h, l;
                    split_hl(px, h.x, l.x);
                    split_hl(py, h.y, l.y);
                    split_hl(pz, h.z, l.z);
                    h.w = (float)pq;
                    l.w = 0.f;
                    shi[warp][slot][lane] = h;
                    slo[warp][slot][lane] = l;
                    if (!GRAD) {
                        float *pk = reinterpret_cast<float *>(spk[warp][slot][0]);
                        const int m = lane >> 1, hh = lane & 1;
                        pk[0 * 64 + 4 * m + hh] = -h.x;
                        pk[0 * 64 + 4 * m + 2 + hh] = -h.y;
                        pk[1 * 64 + 4 * m + hh] = -h.z;
                        pk[1 * 64 + 4 * m + 2 + hh] = h.w;
                        pk[2 * 64 + 4 * m + hh] = -l.x;
                        pk[2 * 64 + 4 * m + 2 + hh] = -l.y;
                        pk[3 * 64 + 4 * m + hh] = -l.z;
                    }
                }
                if (bt + 1 < nbat) {
                    const int32_t f = 32 * (bt + 1) + lane;
                    const int32_t s = locate(min(f, S - 1));
                    px = py = pz = P2PF_FAR;
                    pq = 0.0;
                    if (f < S) {
                        px = sources[s]; py = sources[sstride + s];
                        pz = sources[2 * sstride + s]; pq = strength[s];
                    }
                }
                __syncwarp();
                const int jself = fself - 32 * bt;   // outside [0, 32) if not in this batch
                const int jself2 = fself2 - 32 * bt;
                const bool check = __any_sync(FULL, active && jself >= 0 && jself < 32);
                const bool check2 = two &&
                                    __any_sync(FULL, active2 && jself2 >= 0 && jself2 < 32);
                if (two) {
                    // every lane holds a first target (ntc = 32, one phase)
                    float a = 0.f, a2 = 0.f, dx_ = 0.f, dy_ = 0.f, dz_ = 0.f;
                    const float4 *H = shi[warp][slot], *L = slo[warp][slot];
                    if (check || check2) {
                        // (rare) batches holding a lane's own source: one target at a
                        // time, the compact loop
                        p2p_batch<true, false, 0>(H, L, tg, 0, 1, jself, a, dx_, dy_, dz_);
                        p2p_batch<true, false, 0>(H, L, tg2, 0, 1, jself2, a2, dx_, dy_, dz_);
                    } else {
                        p2p_batch_packed2(spk[warp][slot][0], spk[warp][slot][1],
                                          spk[warp][slot][2], spk[warp][slot][3], tg, tg2, a,
                                          a2);
                    }
                    acc += (double)a;
                    acc2 += (double)a2;
                } else if (active) {
                    float a = 0.f, ax = 0.f, ay = 0.f, az = 0.f;
                    const float4 *H = shi[warp][slot], *L = slo[warp][slot];
                    if (nph == 1) {
                        if (check) {
                            p2p_batch<true, GRAD, 1>(H, L, tg, 0, 1, jself, a, ax, ay, az);
                        } else if constexpr (GRAD) {
                            p2p_batch<false, GRAD, 1>(H, L, tg, 0, 1, jself, a, ax, ay, az);
                        } else {
                            p2p_batch_packed(spk[warp][slot][0], spk[warp][slot][1],
                                             spk[warp][slot][2], spk[warp][slot][3], tg, a);
                        }
                    } else {
                        if (check) {
                            p2p_batch<true, GRAD, 0>(H, L, tg, ph, nph, jself, a, ax, ay, az);
                        } else if constexpr (GRAD) {
                            p2p_batch<false, GRAD, 0>(H, L, tg, ph, nph, jself, a, ax, ay, az);
                        } else {
                            p2p_batch_packed_phased(spk[warp][slot][0], spk[warp][slot][1],
                                                    spk[warp][slot][2], spk[warp][slot][3], tg,
                                                    ph, nph, a);
                        }
                    }
                    acc += (double)a;
                    if (GRAD) { gx += (double)ax; gy += (double)ay; gz += (double)az; }
                }
                // slot is rewritten by batch bt + 2, after the next __syncwarp
            }
            __syncwarp();   // the next window restages slot 0
        }
        if (active2) result[t2] = scale * acc2;
        // sum the phases (lanes tl, tl + ntc, ...) through shared memory
        red[warp][0][lane] = acc;
        if (GRAD) { red[warp][1][lane] = gx; red[warp][2][lane] = gy; red[warp][3][lane] = gz; }
        __syncwarp();
        if (lane < ntc) {
            double v = 0.0, vx = 0.0, vy = 0.0, vz = 0.0;
            for (int q = 0; q < nph; ++q) {
                v += red[warp][0][lane + q * ntc];
                if (GRAD) {
                    vx += red[warp][1][lane + q * ntc];
                    vy += red[warp][2][lane + q * ntc];
                    vz += red[warp][3][lane + q * ntc];
                }
            }
            if (result) result[t] = scale * v;
            if (GRAD) {
                grad[t] = scale * vx;
                grad[tstride + t] = scale * vy;
                grad[2 * tstride + t] = scale * vz;
            }
        }
        __syncwarp();
        tc += two ? 64 : 32;
    }
}

// }}}

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
    if (MIXED) {
        const int blocks = (ntgt_boxes + P2PF_WARPS - 1) / P2PF_WARPS;
        p2p_flat_mixed_kernel<GRAD><<<blocks, 32 * P2PF_WARPS, 0, as_stream(stream)>>>(
            ntgt_boxes, target_boxes, ss, sl, bss, bsc, bts, btc, sources, sstride, strength,
            targets, tstride, tts, scale, result, grad);
        return check_launch("p2p_flat_mixed_kernel");
    }
    const int blocks = (ntgt_boxes + P2P_WARPS - 1) / P2P_WARPS;
    p2p_csr_kernel<GRAD><<<blocks, 32 * P2P_WARPS, 0, as_stream(stream)>>>(
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
