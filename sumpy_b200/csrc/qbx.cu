// QBX layer potentials: sumpy's LayerPotential / LayerPotentialMatrixGenerator /
// LayerPotentialMatrixSubsetGenerator (sumpy/qbx.py:250-340, 345-420) for the
// 3D Laplace and Helmholtz kernels, FP64 (complex128 for Helmholtz).
//
// For target t with expansion center c and source s, with a = c - s and
// b = t - c, sumpy forms the source's local expansion about c and evaluates
// it at t (the pair expressions at sumpy/qbx.py:118-157). For the line
// Taylor expansion (sumpy/expansion/local.py:116-185) the value is
//     sum_{i <= p} (1/i!) d^i/dtau^i G(a + tau b) |_{tau = 0},
// and for the volume Taylor expansions (plain or PDE-compressed, local.py
// :225-309) it is sum_{|mi| <= p} D^mi G(a) b^mi / mi!, the same number: the
// degree-i terms of the volume sum are (b . grad)^i G(a) / i!. So both are
// computed from the Taylor series of G along the line:
//   Laplace (G = 1/r): with A = |a|^2, w = a.b / A, v = |b|^2 / A,
//     1/|a + tau b| = A^{-1/2} sum_i T_i tau^i, T_0 = 1, T_1 = -w,
//     (n + 1) T_{n+1} = -(2n + 1) w T_n - n v T_{n-1}
//     (the Legendre generating function; P_i(x) rho^i with x the cosine
//     between -a and b and rho = |b| / |a|): O(p) per pair.
//   Helmholtz (G = e^{ikr}/r): the addition theorem regrouped by powers of
//     tau (helmholtz_line below): the Laplace terms T_n times a spherical
//     Hankel recurrence in n times truncated spherical Bessel series, O(p)
//     complex and O(p^2 / 4) real operations per pair.
// Derivatives are carried through the recurrences (with respect to their
// variables: w, v, and for Helmholtz |a| and k^2 |b|^2) and combined by the
// chain rule:
//   target derivative, line Taylor: d/da_axis of each coefficient (sumpy
//     applies the target kernel's derivative to the coefficients with
//     respect to avec, qbx.py:128-132);
//   target derivative, volume Taylor: d/db_axis of the truncated sum (the
//     expansion's evaluate differentiates with respect to bvec);
//   source derivative (axis, or directional along a per-source vector):
//     -d/da (AxisSourceDerivative / DirectionalSourceDerivative
//     postprocess_at_source).
// The kernel's 1/(4 pi) and the strengths (quadrature weights already
// folded in, qbx.py:305-310) are applied as sumpy does. expansion_radii only
// set rscale in sumpy, which cancels; they are not needed here.
#include <cstdint>

#include "common.cuh"

namespace sumpy {
namespace {

constexpr int QBX_MAX_ORDER = 32;
constexpr int QBX_THREADS = 128;
constexpr int QBX_TILE = 128;

enum QbxMode {
    QBX_VALUE = 0,
    QBX_TGT_DERIV_LINE = 1,    // d/da_axis
    QBX_TGT_DERIV_VOLUME = 2,  // d/db_axis
    QBX_SRC_DERIV_AXIS = 3,    // -d/da_axis
    QBX_SRC_DERIV_DIR = 4,     // -dir . grad_a
};

struct C2 {
    double re, im;
};
__device__ __forceinline__ C2 cadd(C2 a, C2 b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ C2 csub(C2 a, C2 b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ C2 cmul(C2 a, C2 b)
{
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ C2 cscale(C2 a, double s) { return {a.re * s, a.im * s}; }

// Laplace line sum and its derivatives with respect to a and b
struct LapOut {
    double val;
    double ga[3], gb[3];
};

// 1 / (n + 1), n <= QBX_MAX_ORDER: the recurrence's divisions, read as
// broadcasts from the constant cache (every thread is at the same n)
#define QBX_INV4(n) 1.0 / ((n) + 1.0), 1.0 / ((n) + 2.0), 1.0 / ((n) + 3.0), 1.0 / ((n) + 4.0)
__constant__ double c_qbx_inv[QBX_MAX_ORDER + 4] = {
    QBX_INV4(0), QBX_INV4(4), QBX_INV4(8), QBX_INV4(12), QBX_INV4(16), QBX_INV4(20),
    QBX_INV4(24), QBX_INV4(28), QBX_INV4(32)};
#undef QBX_INV4

template <bool GRAD>
__device__ __forceinline__ LapOut laplace_line(int p, const double a[3], const double b[3])
{
    const double A = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
    const double D = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    const double B2 = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
    const double rinv = rsqrt(A);
    const double Ainv = rinv * rinv;
    const double w = D * Ainv, v = B2 * Ainv;
    // T_n and, with GRAD, dT_n/dw and dT_n/dv
    double Tm1 = 0.0, T = 1.0, S = 1.0;
    double Wm1 = 0.0, W = 0.0, SW = 0.0;
    double Vm1 = 0.0, V = 0.0, SV = 0.0;
    double c1 = 1.0, c2 = 0.0;   // 2n + 1, n
    double cw = w, cv = 0.0;     // (2n + 1) w, n v
    const double w2 = 2.0 * w;
    for (int n = 0; n < p; ++n) {
        const double inv = c_qbx_inv[n];
        const double Tn = -fma(cw, T, cv * Tm1) * inv;
        if (GRAD) {
            const double Wn = (-c1 * (T + w * W) - c2 * v * Wm1) * inv;
            const double Vn = (-c1 * w * V - c2 * (Tm1 + v * Vm1)) * inv;
            Wm1 = W; W = Wn; SW += Wn;
            Vm1 = V; V = Vn; SV += Vn;
            c1 += 2.0;
            c2 += 1.0;
        }
        Tm1 = T; T = Tn; S += Tn;
        cw += w2;
        cv += v;
    }
    LapOut o;
    o.val = S * rinv;
    if (GRAD) {
        for (int d = 0; d < 3; ++d) {
            const double dw_da = b[d] * Ainv - 2.0 * D * a[d] * Ainv * Ainv;
            const double dv_da = -2.0 * B2 * a[d] * Ainv * Ainv;
            o.ga[d] = rinv * (SW * dw_da + SV * dv_da) - S * a[d] * Ainv * rinv;
            o.gb[d] = rinv * (SW * a[d] * Ainv + SV * 2.0 * b[d] * Ainv);
        }
    }
    return o;
}

// Helmholtz line sum and derivatives (complex)
struct HelmOut {
    C2 val;
    C2 ga[3], gb[3];
};

// Recurrence constants of the Helmholtz line sum, folded at compile time:
// hv[n] = 1 / ((2n + 1)(2n - 1)) (n >= 1) and g[n][m] = 1 / ((m + 1)(2n + 2m + 3))
struct HelmTables {
    double hv[QBX_MAX_ORDER + 1];
    double g[QBX_MAX_ORDER + 1][QBX_MAX_ORDER / 2 + 1];
};
constexpr HelmTables make_helm_tables()
{
    HelmTables t{};
    for (int n = 0; n <= QBX_MAX_ORDER; ++n) {
        t.hv[n] = n == 0 ? 0.0 : 1.0 / ((2.0 * n + 1.0) * (2.0 * n - 1.0));
        for (int m = 0; m <= QBX_MAX_ORDER / 2; ++m)
            t.g[n][m] = 1.0 / ((m + 1.0) * (2.0 * n + 2.0 * m + 3.0));
    }
    return t;
}
__constant__ HelmTables c_helm = make_helm_tables();

// The degree-N Taylor coefficient of G(a + tau b) = e^{ik|a + tau b|} / |a + tau b|
// follows from the addition theorem e^{ik|x - y|}/|x - y| = ik sum_n (2n + 1)
// j_n(k|x|) h_n(k|y|) P_n(cos) (x = tau b, y = -a) by collecting powers of tau
// in j_n(k tau |b|) = sum_m (-1)^m (k tau |b|)^{n + 2m} / (2^m m! (2n + 2m + 1)!!).
// Truncated at total degree p the line sum is
//   S = sum_{n <= p} T_n(w, v) V_n(r) G_n(Z),
// with T_n = P_n(x) rho^n the Laplace recurrence's terms (x the cosine between
// -a and b, rho = |b| / |a|), r = |a|, Z = k^2 |b|^2,
//   V_n = ik (k r)^n h_n(k r) / (2n - 1)!!:  V_0 = e^{ikr} / r,
//     V_1 = e^{ikr} (1/r - ik),  V_{n+1} = V_n - (k r)^2 V_{n-1} / ((2n + 1)(2n - 1)),
//   G_n = sum_{m <= (p - n) / 2} (-Z / 2)^m / (m! prod_{j=1..m} (2n + 2j + 1)).
// (k -> 0 gives V_n = 1/r, G_n = 1: the Laplace sum.) O(p^2 / 4) real
// multiply-adds for the G_n and O(p) complex ones: no series convolutions.
// Derivatives by the chain rule through w, v, r and Z.
template <bool GRAD>
__device__ __forceinline__ HelmOut helmholtz_line(int p, double k, const double a[3],
                                                  const double b[3])
{
    const double A = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
    const double D = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    const double B2 = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
    const double rinv = rsqrt(A);
    const double Ainv = rinv * rinv;
    const double r = A * rinv;
    const double w = D * Ainv, v = B2 * Ainv;
    const double k2 = k * k;
    const double K2 = k2 * A;          // (k r)^2
    const double hz = -0.5 * k2 * B2;  // -Z / 2
    double sn, cs;
    sincos(k * r, &sn, &cs);
    const C2 e = {cs, sn};
    // V_n, V_{n-1}, V_1 and their r derivatives
    C2 Vc = cscale(e, rinv), Vp = {0.0, 0.0};
    const C2 V1 = cmul(e, C2{rinv, -k});
    C2 dVc = {0.0, 0.0}, dVp = {0.0, 0.0}, dV1 = {0.0, 0.0};
    if (GRAD) {
        dVc = cmul(e, C2{-Ainv, k * rinv});       // e (ik / r - 1 / r^2)
        dV1 = cmul(e, C2{k2 - Ainv, k * rinv});   // e (ik / r + k^2 - 1 / r^2)
    }
    double Tm1 = 0.0, T = 1.0, Wm1 = 0.0, W = 0.0, Um1 = 0.0, U = 0.0;
    double c1 = 1.0, c2 = 0.0;   // 2n + 1, n
    double cw = w, cv = 0.0;     // (2n + 1) w, n v
    const double w2 = 2.0 * w;
    C2 S = {0.0, 0.0}, Sw = {0.0, 0.0}, Sv = {0.0, 0.0}, Sr = {0.0, 0.0}, Sz = {0.0, 0.0};
    for (int n = 0; n <= p; ++n) {
        // G_n and, with GRAD, dG_n / dZ = sum_m m c_m Z^{m-1}
        double G = 1.0, t = 1.0, Gd = 0.0, q = 0.0, mm = 1.0;
        const int M = (p - n) >> 1;
        for (int m = 0; m < M; ++m) {
            const double f = c_helm.g[n][m];
            t *= hz * f;
            G += t;
            if (GRAD) {
                q = m == 0 ? -0.5 * f : q * hz * f;
                Gd += mm * q;
                mm += 1.0;
            }
        }
        const double TG = T * G;
        S = cadd(S, cscale(Vc, TG));
        if (GRAD) {
            Sw = cadd(Sw, cscale(Vc, W * G));
            Sv = cadd(Sv, cscale(Vc, U * G));
            Sr = cadd(Sr, cscale(dVc, TG));
            Sz = cadd(Sz, cscale(Vc, T * Gd));
        }
        if (n == p) break;
        // T_{n+1} (and dT/dw, dT/dv)
        const double inv = c_qbx_inv[n];
        const double Tn = -fma(cw, T, cv * Tm1) * inv;
        if (GRAD) {
            const double Wn = (-c1 * (T + w * W) - c2 * v * Wm1) * inv;
            const double Un = (-c1 * w * U - c2 * (Tm1 + v * Um1)) * inv;
            Wm1 = W; W = Wn;
            Um1 = U; U = Un;
            c1 += 2.0;
            c2 += 1.0;
        }
        Tm1 = T; T = Tn;
        cw += w2;
        cv += v;
        // V_{n+1}
        C2 Vn = V1, dVn = dV1;
        if (n > 0) {
            const double h = c_helm.hv[n];
            Vn = csub(Vc, cscale(Vp, K2 * h));
            if (GRAD)
                dVn = csub(dVc, cadd(cscale(Vp, 2.0 * k2 * r * h), cscale(dVp, K2 * h)));
        }
        Vp = Vc; Vc = Vn;
        if (GRAD) { dVp = dVc; dVc = dVn; }
    }
    HelmOut o;
    o.val = S;
    if (GRAD) {
        for (int d = 0; d < 3; ++d) {
            const double dw_da = b[d] * Ainv - 2.0 * D * a[d] * Ainv * Ainv;
            const double dv_da = -2.0 * B2 * a[d] * Ainv * Ainv;
            o.ga[d] = cadd(cadd(cscale(Sw, dw_da), cscale(Sv, dv_da)), cscale(Sr, a[d] * rinv));
            o.gb[d] = cadd(cadd(cscale(Sw, a[d] * Ainv), cscale(Sv, 2.0 * b[d] * Ainv)),
                           cscale(Sz, 2.0 * k2 * b[d]));
        }
    }
    return o;
}

template <int MODE>
__device__ __forceinline__ double laplace_pair(int p, int axis, const double a[3],
                                               const double b[3], const double *dir)
{
    if (MODE == QBX_VALUE) return laplace_line<false>(p, a, b).val;
    const LapOut o = laplace_line<true>(p, a, b);
    if (MODE == QBX_TGT_DERIV_LINE) return o.ga[axis];
    if (MODE == QBX_TGT_DERIV_VOLUME) return o.gb[axis];
    if (MODE == QBX_SRC_DERIV_AXIS) return -o.ga[axis];
    return -(dir[0] * o.ga[0] + dir[1] * o.ga[1] + dir[2] * o.ga[2]);
}

template <int MODE>
__device__ __forceinline__ C2 helmholtz_pair(int p, double k, int axis, const double a[3],
                                             const double b[3], const double *dir)
{
    if (MODE == QBX_VALUE) return helmholtz_line<false>(p, k, a, b).val;
    const HelmOut o = helmholtz_line<true>(p, k, a, b);
    if (MODE == QBX_TGT_DERIV_LINE) return o.ga[axis];
    if (MODE == QBX_TGT_DERIV_VOLUME) return o.gb[axis];
    if (MODE == QBX_SRC_DERIV_AXIS) return cscale(o.ga[axis], -1.0);
    return cscale(cadd(cadd(cscale(o.ga[0], dir[0]), cscale(o.ga[1], dir[1])),
                       cscale(o.ga[2], dir[2])), -1.0);
}

// G threads per target (G a power of two <= 32, so a group never straddles
// a warp): the block's 128 / G targets share tiles of sources staged in shared
// memory, lane g of a group takes the tile's sources j = g mod G, and the
// group sums its partials with a fixed shuffle tree (deterministic). G grows
// when there are few targets, so that small target sets still fill the SMs.
template <int MODE, bool HELM>
__global__ void __launch_bounds__(QBX_THREADS)
qbx_lpot_kernel(int p, double k, int axis, int group, int64_t ntgt,
                const double *__restrict__ targets, int64_t tstride,
                const double *__restrict__ centers, int64_t cstride, int64_t nsrc,
                const double *__restrict__ sources, int64_t sstride,
                const double *__restrict__ dirs, int64_t dstride,
                const double *__restrict__ strength, double scale, double *__restrict__ result)
{
    __shared__ double s_x[QBX_TILE], s_y[QBX_TILE], s_z[QBX_TILE];
    __shared__ double s_q[QBX_TILE], s_qi[HELM ? QBX_TILE : 1];
    __shared__ double s_d[MODE == QBX_SRC_DERIV_DIR ? 3 : 1][QBX_TILE];
    const int g = threadIdx.x & (group - 1);
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x / group) + threadIdx.x / group;
    const bool active = t < ntgt;
    double c[3] = {0, 0, 0}, b[3] = {0, 0, 0};
    if (active) {
        for (int d = 0; d < 3; ++d) {
            c[d] = centers[d * cstride + t];
            b[d] = targets[d * tstride + t] - c[d];
        }
    }
    double acc = 0.0, acci = 0.0;
    for (int64_t s0 = 0; s0 < nsrc; s0 += QBX_TILE) {
        const int m = (int)(nsrc - s0 < QBX_TILE ? nsrc - s0 : QBX_TILE);
        __syncthreads();
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            const int64_t s = s0 + j;
            s_x[j] = sources[s];
            s_y[j] = sources[sstride + s];
            s_z[j] = sources[2 * sstride + s];
            if (HELM) {
                s_q[j] = strength[2 * s];
                s_qi[j] = strength[2 * s + 1];
            } else {
                s_q[j] = strength[s];
            }
            if (MODE == QBX_SRC_DERIV_DIR)
                for (int d = 0; d < 3; ++d) s_d[d][j] = dirs[d * dstride + s];
        }
        __syncthreads();
        if (!active) continue;
        for (int j = g; j < m; j += group) {
            const double a[3] = {c[0] - s_x[j], c[1] - s_y[j], c[2] - s_z[j]};
            double dir[3] = {0, 0, 0};
            if (MODE == QBX_SRC_DERIV_DIR)
                for (int d = 0; d < 3; ++d) dir[d] = s_d[d][j];
            if (HELM) {
                const C2 v = helmholtz_pair<MODE>(p, k, axis, a, b, dir);
                acc += v.re * s_q[j] - v.im * s_qi[j];
                acci += v.re * s_qi[j] + v.im * s_q[j];
            } else {
                acc += laplace_pair<MODE>(p, axis, a, b, dir) * s_q[j];
            }
        }
    }
    // every lane of the warp takes part (inactive ones hold zeros)
    for (int off = group >> 1; off > 0; off >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, off, group);
        if (HELM) acci += __shfl_down_sync(0xffffffffu, acci, off, group);
    }
    if (active && g == 0) {
        if (HELM) {
            result[2 * t] = scale * acc;
            result[2 * t + 1] = scale * acci;
        } else {
            result[t] = scale * acc;
        }
    }
}

// matrix entries: entry e = (tgt[e] or e / nsrc, src[e] or e % nsrc)
template <int MODE, bool HELM, bool SUBSET>
__global__ void qbx_matrix_kernel(int p, double k, int axis, int64_t nentries, int64_t nsrc,
                                  const int32_t *__restrict__ tgtidx,
                                  const int32_t *__restrict__ srcidx,
                                  const double *__restrict__ targets, int64_t tstride,
                                  const double *__restrict__ centers, int64_t cstride,
                                  const double *__restrict__ sources, int64_t sstride,
                                  const double *__restrict__ dirs, int64_t dstride, double scale,
                                  double *__restrict__ out)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nentries;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = SUBSET ? tgtidx[e] : e / nsrc;
        const int64_t s = SUBSET ? srcidx[e] : e - (e / nsrc) * nsrc;
        double a[3], b[3], dir[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d) {
            const double cd = centers[d * cstride + t];
            a[d] = cd - sources[d * sstride + s];
            b[d] = targets[d * tstride + t] - cd;
            if (MODE == QBX_SRC_DERIV_DIR) dir[d] = dirs[d * dstride + s];
        }
        if (HELM) {
            const C2 g = helmholtz_pair<MODE>(p, k, axis, a, b, dir);
            out[2 * e] = scale * g.re;
            out[2 * e + 1] = scale * g.im;
        } else {
            out[e] = scale * laplace_pair<MODE>(p, axis, a, b, dir);
        }
    }
}

int check_common(int order, int mode, int axis)
{
    if (order < 0 || order > QBX_MAX_ORDER) return bad_arg("qbx: order must be in [0, 32]");
    if (mode < QBX_VALUE || mode > QBX_SRC_DERIV_DIR) return bad_arg("qbx: unknown mode");
    if (mode != QBX_VALUE && mode != QBX_SRC_DERIV_DIR && (axis < 0 || axis > 2))
        return bad_arg("qbx: axis must be 0, 1 or 2");
    return SUMPY_OK;
}

// threads per target: the smallest power of two <= 32 that gives two blocks
// per SM (148 SMs), so that a few targets against many sources fill the GPU
int lpot_group(int64_t ntgt, int64_t nsrc)
{
    int group = 1;
    while (group < 32 && group < nsrc &&
           (ntgt + QBX_THREADS / group - 1) / (QBX_THREADS / group) < 2 * 148)
        group *= 2;
    return group;
}

template <bool HELM>
int qbx_lpot_launch(int order, int mode, int axis, double k, int64_t ntgt,
                    const double *targets, int64_t tstride, const double *centers,
                    int64_t cstride, int64_t nsrc, const double *sources, int64_t sstride,
                    const double *dirs, int64_t dstride, const double *strength, double scale,
                    double *result, void *stream)
{
    int rc = check_common(order, mode, axis);
    if (rc) return rc;
    if (ntgt < 0 || nsrc < 0) return bad_arg("qbx: negative size");
    if (ntgt == 0) return SUMPY_OK;
    if (!targets || !centers || !result) return bad_arg("qbx: null target-side pointer");
    if (nsrc > 0 && (!sources || !strength || (mode == QBX_SRC_DERIV_DIR && !dirs)))
        return bad_arg("qbx: null source-side pointer");
    const int group = lpot_group(ntgt, nsrc);
    const int per_block = QBX_THREADS / group;
    const unsigned blocks = (unsigned)((ntgt + per_block - 1) / per_block);
    cudaStream_t st = as_stream(stream);
#define QBX_LAUNCH(M)                                                                        \
    qbx_lpot_kernel<M, HELM><<<blocks, QBX_THREADS, 0, st>>>(                                  \
        order, k, axis, group, ntgt, targets, tstride, centers, cstride, nsrc, sources,        \
        sstride, dirs, dstride, strength, scale, result)
    switch (mode) {
    case QBX_VALUE: QBX_LAUNCH(QBX_VALUE); break;
    case QBX_TGT_DERIV_LINE: QBX_LAUNCH(QBX_TGT_DERIV_LINE); break;
    case QBX_TGT_DERIV_VOLUME: QBX_LAUNCH(QBX_TGT_DERIV_VOLUME); break;
    case QBX_SRC_DERIV_AXIS: QBX_LAUNCH(QBX_SRC_DERIV_AXIS); break;
    default: QBX_LAUNCH(QBX_SRC_DERIV_DIR); break;
    }
#undef QBX_LAUNCH
    return check_launch("qbx_lpot_kernel");
}

template <bool HELM, bool SUBSET>
int qbx_matrix_launch(int order, int mode, int axis, double k, int64_t nentries, int64_t nsrc,
                      const int32_t *tgtidx, const int32_t *srcidx, const double *targets,
                      int64_t tstride, const double *centers, int64_t cstride,
                      const double *sources, int64_t sstride, const double *dirs,
                      int64_t dstride, double scale, double *out, void *stream)
{
    int rc = check_common(order, mode, axis);
    if (rc) return rc;
    if (nentries < 0 || nsrc < 0) return bad_arg("qbx: negative size");
    if (nentries == 0) return SUMPY_OK;
    if (!out || !targets || !centers || !sources || (mode == QBX_SRC_DERIV_DIR && !dirs) ||
        (SUBSET && (!tgtidx || !srcidx)) || (!SUBSET && nsrc == 0))
        return bad_arg("qbx: null pointer argument or empty source set");
    const int64_t b = (nentries + 255) / 256;
    const unsigned blocks = (unsigned)(b < 148 * 64 ? b : 148 * 64);
    cudaStream_t st = as_stream(stream);
#define QBX_MLAUNCH(M)                                                                       \
    qbx_matrix_kernel<M, HELM, SUBSET><<<blocks, 256, 0, st>>>(                                \
        order, k, axis, nentries, nsrc, tgtidx, srcidx, targets, tstride, centers, cstride,    \
        sources, sstride, dirs, dstride, scale, out)
    switch (mode) {
    case QBX_VALUE: QBX_MLAUNCH(QBX_VALUE); break;
    case QBX_TGT_DERIV_LINE: QBX_MLAUNCH(QBX_TGT_DERIV_LINE); break;
    case QBX_TGT_DERIV_VOLUME: QBX_MLAUNCH(QBX_TGT_DERIV_VOLUME); break;
    case QBX_SRC_DERIV_AXIS: QBX_MLAUNCH(QBX_SRC_DERIV_AXIS); break;
    default: QBX_MLAUNCH(QBX_SRC_DERIV_DIR); break;
    }
#undef QBX_MLAUNCH
    return check_launch("qbx_matrix_kernel");
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_qbx_lpot_laplace_f64(int order, int mode, int axis, int64_t ntargets,
                               const double *targets, int64_t target_stride,
                               const double *centers, int64_t center_stride, int64_t nsources,
                               const double *sources, int64_t source_stride,
                               const double *source_dirs, int64_t dir_stride,
                               const double *strength, double scale, double *result,
                               void *stream)
{
    return qbx_lpot_launch<false>(order, mode, axis, 0.0, ntargets, targets, target_stride,
                                  centers, center_stride, nsources, sources, source_stride,
                                  source_dirs, dir_stride, strength, scale, result, stream);
}

int sumpy_qbx_lpot_helmholtz_f64(int order, int mode, int axis, double k, int64_t ntargets,
                                 const double *targets, int64_t target_stride,
                                 const double *centers, int64_t center_stride, int64_t nsources,
                                 const double *sources, int64_t source_stride,
                                 const double *source_dirs, int64_t dir_stride,
                                 const double *strength, double scale, double *result,
                                 void *stream)
{
    return qbx_lpot_launch<true>(order, mode, axis, k, ntargets, targets, target_stride,
                                 centers, center_stride, nsources, sources, source_stride,
                                 source_dirs, dir_stride, strength, scale, result, stream);
}

int sumpy_qbx_matrix_laplace_f64(int order, int mode, int axis, int64_t ntargets,
                                 const double *targets, int64_t target_stride,
                                 const double *centers, int64_t center_stride,
                                 int64_t nsources, const double *sources,
                                 int64_t source_stride, const double *source_dirs,
                                 int64_t dir_stride, double scale, double *result, void *stream)
{
    if (ntargets < 0 || nsources < 0) return bad_arg("qbx: negative size");
    return qbx_matrix_launch<false, false>(order, mode, axis, 0.0, ntargets * nsources, nsources,
                                           nullptr, nullptr, targets, target_stride, centers,
                                           center_stride, sources, source_stride, source_dirs,
                                           dir_stride, scale, result, stream);
}

int sumpy_qbx_matrix_helmholtz_f64(int order, int mode, int axis, double k, int64_t ntargets,
                                   const double *targets, int64_t target_stride,
                                   const double *centers, int64_t center_stride,
                                   int64_t nsources, const double *sources,
                                   int64_t source_stride, const double *source_dirs,
                                   int64_t dir_stride, double scale, double *result,
                                   void *stream)
{
    if (ntargets < 0 || nsources < 0) return bad_arg("qbx: negative size");
    return qbx_matrix_launch<true, false>(order, mode, axis, k, ntargets * nsources, nsources,
                                          nullptr, nullptr, targets, target_stride, centers,
                                          center_stride, sources, source_stride, source_dirs,
                                          dir_stride, scale, result, stream);
}

int sumpy_qbx_matrix_subset_laplace_f64(int order, int mode, int axis, int64_t nentries,
                                        const int32_t *tgtindices, const int32_t *srcindices,
                                        const double *targets, int64_t target_stride,
                                        const double *centers, int64_t center_stride,
                                        const double *sources, int64_t source_stride,
                                        const double *source_dirs, int64_t dir_stride,
                                        double scale, double *result, void *stream)
{
    return qbx_matrix_launch<false, true>(order, mode, axis, 0.0, nentries, 0, tgtindices,
                                          srcindices, targets, target_stride, centers,
                                          center_stride, sources, source_stride, source_dirs,
                                          dir_stride, scale, result, stream);
}

int sumpy_qbx_matrix_subset_helmholtz_f64(int order, int mode, int axis, double k,
                                          int64_t nentries, const int32_t *tgtindices,
                                          const int32_t *srcindices, const double *targets,
                                          int64_t target_stride, const double *centers,
                                          int64_t center_stride, const double *sources,
                                          int64_t source_stride, const double *source_dirs,
                                          int64_t dir_stride, double scale, double *result,
                                          void *stream)
{
    return qbx_matrix_launch<true, true>(order, mode, axis, k, nentries, 0, tgtindices,
                                         srcindices, targets, target_stride, centers,
                                         center_stride, sources, source_stride, source_dirs,
                                         dir_stride, scale, result, stream);
}

}  // extern "C"
