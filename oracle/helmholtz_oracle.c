/*
 * helmholtz_oracle.c -- FP64 CPU restatement of sumpy's 3D Helmholtz FMM
 * operators (HelmholtzKernel(3), G = exp(i k r) / r, compressed Taylor
 * expansions).
 *
 * TEST INFRASTRUCTURE ONLY. Like fmm_oracle.c this is the oracle: only
 * tests/, the smoke check in __graft_entry__.py and the cpu_baseline /
 * reference arm of bench.py may load it. The product never calls it.
 *
 * Complex arrays are interleaved (re, im) float64, i.e. C99 double complex.
 * Conventions as in fmm_oracle.c (a = center - source, b = target - center,
 * d = target center - source center; 1/(4 pi) only on point outputs).
 *
 * Kernel-specific pieces (everything else is the Laplace file's algorithm
 * with complex values):
 *   - derivatives: HelmholtzDerivativeTaker / RadialDerivativeTaker.diff
 *     (sumpy/derivative_taker.py:269-389): for a radial G, with
 *     g_q = ((1/r) d/dr)^q G,
 *       D(mi, q) = x_i rs D(mi - e_i, q + 1)                 (first i, mi_i == 1)
 *       D(mi, q) = (mi_i - 1) rs^2 D(mi - 2e_i, q + 1)
 *                  + x_i rs D(mi - e_i, q + 1)               (else first mi_i >= 2)
 *       D(0, q)  = g_q,  g_0 = e^{ikr}/r,  g_1 = (ikr - 1) e^{ikr}/r^3,
 *       g_q = (-(2q - 1) g_{q-1} - k^2 g_{q-2}) / r^2      (q >= 2);
 *   - PDE projection (sumpy/expansion/__init__.py:754-886 with the PDE
 *     Laplacian + k^2, sumpy/kernel.py:838-844): for mi0 >= 2
 *       u_mi = -u_{mi-2e0+2e1} - u_{mi-2e0+2e2} - k^2 rs^2 u_{mi-2e0}.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;
#define I_ _Complex_I

typedef struct {
    int p;
    int nfull, nstored;
    int (*full)[3];
    int (*stored)[3];
    int *lut;
    int *stored_of_full;
} hmi;

static int hlut(const hmi *t, int i, int j, int k)
{
    if (i < 0 || j < 0 || k < 0 || i + j + k > t->p) return -1;
    return t->lut[(i * (t->p + 1) + j) * (t->p + 1) + k];
}

/* full ids sorted by (|mi|, mi0, mi1, mi2); stored = mi0 < 2 */
static void hmi_init(hmi *t, int p)
{
    t->p = p;
    int cap = (p + 1) * (p + 2) * (p + 3) / 6;
    t->full = malloc(sizeof(int[3]) * cap);
    t->stored = malloc(sizeof(int[3]) * cap);
    t->lut = malloc(sizeof(int) * (p + 1) * (p + 1) * (p + 1));
    t->stored_of_full = malloc(sizeof(int) * cap);
    for (int i = 0; i < (p + 1) * (p + 1) * (p + 1); ++i) t->lut[i] = -1;
    int nf = 0, ns = 0;
    for (int deg = 0; deg <= p; ++deg)
        for (int i = 0; i <= deg; ++i)
            for (int j = 0; j <= deg - i; ++j) {
                int k = deg - i - j;
                t->full[nf][0] = i; t->full[nf][1] = j; t->full[nf][2] = k;
                t->lut[(i * (p + 1) + j) * (p + 1) + k] = nf;
                if (i < 2) {
                    t->stored[ns][0] = i; t->stored[ns][1] = j; t->stored[ns][2] = k;
                    t->stored_of_full[nf] = ns++;
                } else {
                    t->stored_of_full[nf] = -1;
                }
                ++nf;
            }
    t->nfull = nf;
    t->nstored = ns;
}

static void hmi_free(hmi *t)
{
    free(t->full); free(t->stored); free(t->lut); free(t->stored_of_full);
}

static double hfact(int n)
{
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}

/* stored -> full (CSEMatVecOperator.matvec, rows in order) */
static void h_project(const hmi *t, double kappa, const cplx *stored, cplx *full)
{
    for (int f = 0; f < t->nfull; ++f) {
        int s = t->stored_of_full[f];
        if (s >= 0) { full[f] = stored[s]; continue; }
        const int *m = t->full[f];
        full[f] = -full[hlut(t, m[0] - 2, m[1] + 2, m[2])]
                  - full[hlut(t, m[0] - 2, m[1], m[2] + 2)]
                  - kappa * full[hlut(t, m[0] - 2, m[1], m[2])];
    }
}

/* full -> stored (transpose_matvec, rows in reverse order); full_in is copied */
static void h_compress(const hmi *t, double kappa, const cplx *full_in, cplx *stored)
{
    cplx *w = malloc(sizeof(cplx) * t->nfull);
    memcpy(w, full_in, sizeof(cplx) * t->nfull);
    for (int f = t->nfull - 1; f >= 0; --f) {
        if (t->stored_of_full[f] >= 0) continue;
        const int *m = t->full[f];
        w[hlut(t, m[0] - 2, m[1] + 2, m[2])] -= w[f];
        w[hlut(t, m[0] - 2, m[1], m[2] + 2)] -= w[f];
        w[hlut(t, m[0] - 2, m[1], m[2])] -= kappa * w[f];
    }
    for (int f = 0; f < t->nfull; ++f)
        if (t->stored_of_full[f] >= 0) stored[t->stored_of_full[f]] = w[f];
    free(w);
}

/* D(mi) = rs^|mi| d^mi G(x) for mi0 <= maxi0 (<= 1), |mi| <= maxdeg, by the
 * recursion above. out is [(maxi0+1)][(maxdeg+1)][(maxdeg+1)]. */
static void h_derivs(const double x[3], double rs, double k, int maxi0, int maxdeg, cplx *out)
{
    const int M = maxdeg + 1, NI = maxi0 + 1;
    /* E[q][i][j][l], q + |mi| <= maxdeg */
    cplx *E = malloc(sizeof(cplx) * (size_t)M * NI * M * M);
#define EI(q, i, j, l) E[(((size_t)(q) * NI + (i)) * M + (j)) * M + (l)]
    const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    const double r = sqrt(r2);
    const cplx eikr = cexp(_Complex_I * k * r);
    for (int q = 0; q <= maxdeg; ++q) {
        cplx g;
        if (q == 0) g = eikr / r;
        else if (q == 1) g = (_Complex_I * k * r - 1.0) * eikr / (r2 * r);
        else g = (-(2.0 * q - 1.0) * EI(q - 1, 0, 0, 0) - k * k * EI(q - 2, 0, 0, 0)) / r2;
        EI(q, 0, 0, 0) = g;
    }
    for (int deg = 1; deg <= maxdeg; ++deg)
        for (int i = 0; i <= (deg < maxi0 ? deg : maxi0); ++i)
            for (int j = 0; j <= deg - i; ++j) {
                int l = deg - i - j;
                int mi[3] = {i, j, l};
                int ax = -1;
                for (int a = 0; a < 3; ++a) if (mi[a] == 1) { ax = a; break; }
                int two = 0;
                if (ax < 0) {
                    for (int a = 0; a < 3; ++a) if (mi[a] >= 2) { ax = a; break; }
                    two = 1;
                }
                int m1[3] = {i, j, l}, m2[3] = {i, j, l};
                m1[ax] -= 1; m2[ax] -= 2;
                for (int q = 0; q + deg <= maxdeg; ++q) {
                    cplx v = x[ax] * rs * EI(q + 1, m1[0], m1[1], m1[2]);
                    if (two) v += (mi[ax] - 1) * rs * rs * EI(q + 1, m2[0], m2[1], m2[2]);
                    EI(q, i, j, l) = v;
                }
            }
    for (int i = 0; i <= maxi0; ++i)
        for (int j = 0; j <= maxdeg; ++j)
            for (int l = 0; l <= maxdeg; ++l)
                out[((size_t)i * M + j) * M + l] = (i + j + l <= maxdeg) ? EI(0, i, j, l) : 0.0;
#undef EI
    free(E);
}

/* ---------------------------- point operators ---------------------------- */

int oracle_helm_ncoeff(int p) { return (p + 1) * (p + 1); }

/* P2M for one box (multipole.py:77-114 with the Helmholtz compression) */
static void h_p2m_box(const hmi *t, double rs, double k, const double c[3], int n,
                      const double *sx, const double *sy, const double *sz,
                      const cplx *q, cplx *out)
{
    cplx *full = calloc(t->nfull, sizeof(cplx));
    for (int s = 0; s < n; ++s) {
        double a[3] = {(c[0] - sx[s]) / rs, (c[1] - sy[s]) / rs, (c[2] - sz[s]) / rs};
        for (int f = 0; f < t->nfull; ++f) {
            const int *mi = t->full[f];
            double v = 1.0;
            for (int ax = 0; ax < 3; ++ax) v *= pow(a[ax], mi[ax]) / hfact(mi[ax]);
            full[f] += q[s] * v;
        }
    }
    h_compress(t, k * k * rs * rs, full, out);
    free(full);
}

void oracle_helm_p2m_point(int p, double rs, double k, const double *center, int n,
                           const double *sx, const double *sy, const double *sz,
                           const double *q, double *out)
{
    hmi t; hmi_init(&t, p);
    h_p2m_box(&t, rs, k, center, n, sx, sy, sz, (const cplx *)q, (cplx *)out);
    hmi_free(&t);
}

/* P2L (local.py:225-271): L[s] += q D(s)(center - source) */
static void h_p2l_add(const hmi *t, double rs, double k, const double c[3], int n,
                      const double *sx, const double *sy, const double *sz,
                      const cplx *q, cplx *out, cplx *tab)
{
    int p = t->p, M = p + 1;
    for (int s = 0; s < n; ++s) {
        double a[3] = {c[0] - sx[s], c[1] - sy[s], c[2] - sz[s]};
        h_derivs(a, rs, k, 1, p, tab);
        for (int st = 0; st < t->nstored; ++st) {
            const int *mi = t->stored[st];
            out[st] += q[s] * tab[((size_t)mi[0] * M + mi[1]) * M + mi[2]];
        }
    }
}

void oracle_helm_p2l_point(int p, double rs, double k, const double *center, int n,
                           const double *sx, const double *sy, const double *sz,
                           const double *q, double *out)
{
    hmi t; hmi_init(&t, p);
    cplx *tab = malloc(sizeof(cplx) * 2 * (p + 1) * (p + 1));
    cplx *o = (cplx *)out;
    for (int i = 0; i < t.nstored; ++i) o[i] = 0.0;
    h_p2l_add(&t, rs, k, center, n, sx, sy, sz, (const cplx *)q, o, tab);
    free(tab);
    hmi_free(&t);
}

/* L2P (local.py:284-309) */
static cplx h_l2p_eval(const hmi *t, double rs, double k, const cplx *coeffs,
                       const double b[3], cplx *full)
{
    h_project(t, k * k * rs * rs, coeffs, full);
    double bs[3] = {b[0] / rs, b[1] / rs, b[2] / rs};
    cplx acc = 0.0;
    for (int f = 0; f < t->nfull; ++f) {
        const int *mi = t->full[f];
        double v = 1.0;
        for (int ax = 0; ax < 3; ++ax) v *= pow(bs[ax], mi[ax]) / hfact(mi[ax]);
        acc += full[f] * v;
    }
    return acc;
}

void oracle_helm_l2p_point(int p, double rs, double k, const double *coeffs,
                           const double *b, double *out)
{
    hmi t; hmi_init(&t, p);
    cplx *full = malloc(sizeof(cplx) * t.nfull);
    *(cplx *)out = h_l2p_eval(&t, rs, k, (const cplx *)coeffs, b, full);
    free(full);
    hmi_free(&t);
}

/* M2P (multipole.py:131-157) */
static cplx h_m2p_eval(const hmi *t, double rs, double k, const cplx *coeffs,
                       const double b[3], cplx *tab)
{
    int p = t->p, M = p + 1;
    h_derivs(b, rs, k, 1, p, tab);
    cplx acc = 0.0;
    for (int st = 0; st < t->nstored; ++st) {
        const int *mi = t->stored[st];
        acc += coeffs[st] * tab[((size_t)mi[0] * M + mi[1]) * M + mi[2]];
    }
    return acc;
}

void oracle_helm_m2p_point(int p, double rs, double k, const double *coeffs,
                           const double *b, double *out)
{
    hmi t; hmi_init(&t, p);
    cplx *tab = malloc(sizeof(cplx) * 2 * (p + 1) * (p + 1));
    *(cplx *)out = h_m2p_eval(&t, rs, k, (const cplx *)coeffs, b, tab);
    free(tab);
    hmi_free(&t);
}

/* M2M (multipole.py:159-407): stored source coefficients in the target's
 * full slots (others zero) times (r_src/r_tgt)^|mi|, shifts along axes
 * (1, 2, 0), compression with the target rscale. Accumulates. */
static void h_m2m_add(const hmi *ts, const hmi *tt, double rsrc, double rtgt, double k,
                      const double dvec[3], const cplx *in, cplx *out)
{
    int nf = tt->nfull;
    cplx *cur = calloc(nf, sizeof(cplx));
    cplx *nxt = calloc(nf, sizeof(cplx));
    cplx *res = malloc(sizeof(cplx) * tt->nstored);
    double ratio = rsrc / rtgt;
    for (int st = 0; st < tt->nstored; ++st) {
        const int *mi = tt->stored[st];
        int si = hlut(ts, mi[0], mi[1], mi[2]);
        if (si < 0 || ts->stored_of_full[si] < 0) continue;
        cur[hlut(tt, mi[0], mi[1], mi[2])] =
            in[ts->stored_of_full[si]] * pow(ratio, mi[0] + mi[1] + mi[2]);
    }
    const int dims[3] = {1, 2, 0};
    for (int di = 0; di < 3; ++di) {
        int d = dims[di];
        double dd = dvec[d] / rtgt;
        for (int f = 0; f < nf; ++f) {
            const int *tm = tt->full[f];
            cplx acc = 0.0;
            for (int q = 0; q <= tm[d]; ++q) {
                int im[3] = {tm[0], tm[1], tm[2]};
                im[d] = q;
                acc += cur[hlut(tt, im[0], im[1], im[2])] * pow(dd, tm[d] - q) /
                       hfact(tm[d] - q);
            }
            nxt[f] = acc;
        }
        cplx *sw = cur; cur = nxt; nxt = sw;
    }
    h_compress(tt, k * k * rtgt * rtgt, cur, res);
    for (int st = 0; st < tt->nstored; ++st) out[st] += res[st];
    free(cur); free(nxt); free(res);
}

void oracle_helm_m2m_point(int psrc, int ptgt, double rsrc, double rtgt, double k,
                           const double *dvec, const double *in, double *out)
{
    hmi ts, tt; hmi_init(&ts, psrc); hmi_init(&tt, ptgt);
    cplx *o = (cplx *)out;
    for (int i = 0; i < tt.nstored; ++i) o[i] = 0.0;
    h_m2m_add(&ts, &tt, rsrc, rtgt, k, dvec, (const cplx *)in, o);
    hmi_free(&ts); hmi_free(&tt);
}

/* L2L (local.py:346-464): full from stored with the source rscale, Taylor
 * shift axes 0, 1, 2 truncated at p_src, times (r_tgt/r_src)^|mi|. */
static void h_l2l_add(const hmi *ts, const hmi *tt, double rsrc, double rtgt, double k,
                      const double dvec[3], const cplx *in, cplx *out)
{
    int nf = ts->nfull, p = ts->p;
    cplx *cur = malloc(sizeof(cplx) * nf);
    cplx *nxt = malloc(sizeof(cplx) * nf);
    h_project(ts, k * k * rsrc * rsrc, in, cur);
    for (int d = 0; d < 3; ++d) {
        double dd = dvec[d] / rsrc;
        for (int f = 0; f < nf; ++f) {
            const int *om = ts->full[f];
            int deg = om[0] + om[1] + om[2];
            cplx acc = 0.0;
            for (int q = 0; q <= p - deg; ++q) {
                int sm[3] = {om[0], om[1], om[2]};
                sm[d] += q;
                acc += pow(dd, q) * cur[hlut(ts, sm[0], sm[1], sm[2])] / hfact(q);
            }
            nxt[f] = acc;
        }
        cplx *sw = cur; cur = nxt; nxt = sw;
    }
    double ratio = rtgt / rsrc;
    for (int st = 0; st < tt->nstored; ++st) {
        const int *mi = tt->stored[st];
        int f = hlut(ts, mi[0], mi[1], mi[2]);
        if (f < 0) continue;
        out[st] += cur[f] * pow(ratio, mi[0] + mi[1] + mi[2]);
    }
    free(cur); free(nxt);
}

void oracle_helm_l2l_point(int psrc, int ptgt, double rsrc, double rtgt, double k,
                           const double *dvec, const double *in, double *out)
{
    hmi ts, tt; hmi_init(&ts, psrc); hmi_init(&tt, ptgt);
    cplx *o = (cplx *)out;
    for (int i = 0; i < tt.nstored; ++i) o[i] = 0.0;
    h_l2l_add(&ts, &tt, rsrc, rtgt, k, dvec, (const cplx *)in, o);
    hmi_free(&ts); hmi_free(&tt);
}

/* M2L class data (m2l.py:461-537): derivatives with mi0 <= 1 from the
 * recursion, mi0 == 2 from the projection with the source rscale; laid out
 * on the (3, 2p+1, 2p+1) circulant grid at the (src id + tgt id) sums. */
static void h_m2l_class_data(const hmi *t, double rsrc, double k, const double dvec[3],
                             cplx *dcirc, cplx *tab)
{
    int p = t->p, M = 2 * p + 1, E1 = 2 * p + 1, E2 = 2 * p + 1;
    h_derivs(dvec, rsrc, k, 1, 2 * p, tab);
    const double kappa = k * k * rsrc * rsrc;
    for (int i = 0; i < 3 * E1 * E2; ++i) dcirc[i] = 0.0;
    for (int a = 0; a < t->nstored; ++a)
        for (int b = 0; b < t->nstored; ++b) {
            int m[3] = {t->stored[a][0] + t->stored[b][0], t->stored[a][1] + t->stored[b][1],
                        t->stored[a][2] + t->stored[b][2]};
            cplx v;
            if (m[0] < 2) {
                v = tab[((size_t)m[0] * M + m[1]) * M + m[2]];
            } else {
                v = -tab[((size_t)0 * M + m[1] + 2) * M + m[2]]
                    - tab[((size_t)0 * M + m[1]) * M + m[2] + 2]
                    - kappa * tab[((size_t)0 * M + m[1]) * M + m[2]];
            }
            dcirc[(m[0] * E1 + m[1]) * E2 + m[2]] = v;
        }
}

/* Toeplitz apply (tools.py:689-701) and postprocess (m2l.py:679-698) */
static void h_m2l_apply_add(const hmi *t, double rsrc, double rtgt, const cplx *dcirc,
                            const cplx *in, cplx *out, cplx *mcirc)
{
    int p = t->p, E1 = 2 * p + 1, E2 = 2 * p + 1, nc = 3 * E1 * E2;
    for (int i = 0; i < nc; ++i) mcirc[i] = 0.0;
    for (int s = 0; s < t->nstored; ++s)
        mcirc[(t->stored[s][0] * E1 + t->stored[s][1]) * E2 + t->stored[s][2]] = in[s];
    double ratio = rtgt / rsrc;
    for (int tt = 0; tt < t->nstored; ++tt) {
        const int *mi = t->stored[tt];
        int row = (mi[0] * E1 + mi[1]) * E2 + mi[2];
        cplx acc = 0.0;
        for (int col = row; col < nc; ++col) acc += mcirc[col - row] * dcirc[col];
        out[tt] += acc * pow(ratio, mi[0] + mi[1] + mi[2]);
    }
}

void oracle_helm_m2l_point(int p, double rsrc, double rtgt, double k, const double *dvec,
                           const double *in, double *out)
{
    hmi t; hmi_init(&t, p);
    int nc = 3 * (2 * p + 1) * (2 * p + 1);
    cplx *tab = malloc(sizeof(cplx) * 2 * (2 * p + 1) * (2 * p + 1));
    cplx *dc = malloc(sizeof(cplx) * nc), *mc = malloc(sizeof(cplx) * nc);
    cplx *o = (cplx *)out;
    h_m2l_class_data(&t, rsrc, k, dvec, dc, tab);
    for (int i = 0; i < t.nstored; ++i) o[i] = 0.0;
    h_m2l_apply_add(&t, rsrc, rtgt, dc, (const cplx *)in, o, mc);
    free(tab); free(dc); free(mc);
    hmi_free(&t);
}

/* Derivative table D(mi) for mi0 <= 1, |mi| <= maxdeg at one point (tests). */
void oracle_helm_derivs(const double *x, double rs, double k, int maxdeg, double *out)
{
    h_derivs(x, rs, k, 1, maxdeg, (cplx *)out);
}

/* ----------------------------- FMM stages ------------------------------ */

/* Direct sum: pot[t] = 1/(4 pi) sum_s q_s e^{ik|t-s|}/|t-s| (self skipped) */
void oracle_helm_p2p_direct(int64_t ntgt, const double *tx, const double *ty, const double *tz,
                            int64_t nsrc, const double *sx, const double *sy, const double *sz,
                            double k, const double *qd, const int32_t *target_to_source,
                            double *potd)
{
    const cplx *q = (const cplx *)qd;
    cplx *pot = (cplx *)potd;
    const double scale = 1.0 / (4.0 * M_PI);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t t = 0; t < ntgt; ++t) {
        cplx acc = 0.0;
        int64_t self = target_to_source ? target_to_source[t] : -1;
        for (int64_t s = 0; s < nsrc; ++s) {
            if (s == self) continue;
            double dx = tx[t] - sx[s], dy = ty[t] - sy[s], dz = tz[t] - sz[s];
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            acc += q[s] * cexp(I_ * k * r) / r;
        }
        pot[t] = scale * acc;
    }
}

void oracle_helm_p2p_csr(int32_t ntgt_boxes, const int32_t *target_boxes,
                         const int32_t *src_box_starts, const int32_t *src_box_lists,
                         const int32_t *box_src_starts, const int32_t *box_src_counts,
                         const int32_t *box_tgt_starts, const int32_t *box_tgt_counts,
                         const double *sx, const double *sy, const double *sz, double k,
                         const double *qd, const double *tx, const double *ty,
                         const double *tz, const int32_t *target_to_source, double *potd)
{
    const cplx *q = (const cplx *)qd;
    cplx *pot = (cplx *)potd;
    const double scale = 1.0 / (4.0 * M_PI);
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t ib = 0; ib < ntgt_boxes; ++ib) {
        int32_t tb = target_boxes[ib];
        for (int32_t t = box_tgt_starts[tb]; t < box_tgt_starts[tb] + box_tgt_counts[tb]; ++t) {
            cplx acc = 0.0;
            int32_t self = target_to_source ? target_to_source[t] : -1;
            for (int32_t l = src_box_starts[ib]; l < src_box_starts[ib + 1]; ++l) {
                int32_t sb = src_box_lists[l];
                for (int32_t s = box_src_starts[sb]; s < box_src_starts[sb] + box_src_counts[sb]; ++s) {
                    if (s == self) continue;
                    double dx = tx[t] - sx[s], dy = ty[t] - sy[s], dz = tz[t] - sz[s];
                    double r = sqrt(dx * dx + dy * dy + dz * dz);
                    acc += q[s] * cexp(I_ * k * r) / r;
                }
            }
            pot[t] = scale * acc;
        }
    }
}

void oracle_helm_p2m_level(int p, double rs, double k, int32_t nboxes, const int32_t *boxes,
                           int32_t level_start_ibox, const double *cx, const double *cy,
                           const double *cz, const int32_t *box_src_starts,
                           const int32_t *box_src_counts, const double *sx, const double *sy,
                           const double *sz, const double *qd, double *outd)
{
    hmi t; hmi_init(&t, p);
    const cplx *q = (const cplx *)qd;
    cplx *out = (cplx *)outd;
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < nboxes; ++i) {
        int32_t b = boxes[i];
        double c[3] = {cx[b], cy[b], cz[b]};
        int32_t s0 = box_src_starts[b];
        h_p2m_box(&t, rs, k, c, box_src_counts[b], sx + s0, sy + s0, sz + s0, q + s0,
                  out + (int64_t)(b - level_start_ibox) * t.nstored);
    }
    hmi_free(&t);
}

void oracle_helm_m2m_level(int psrc, int ptgt, double rsrc, double rtgt, double k,
                           int32_t nboxes, const int32_t *boxes, const int32_t *box_child_ids,
                           int64_t child_stride, const double *cx, const double *cy,
                           const double *cz, int32_t src_level_start, const double *srcd,
                           int32_t tgt_level_start, double *tgtd)
{
    hmi ts, tt; hmi_init(&ts, psrc); hmi_init(&tt, ptgt);
    const cplx *src = (const cplx *)srcd;
    cplx *tgt = (cplx *)tgtd;
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < nboxes; ++i) {
        int32_t b = boxes[i];
        for (int c = 0; c < 8; ++c) {
            int32_t ch = box_child_ids[c * child_stride + b];
            if (ch == 0) continue;
            double d[3] = {cx[b] - cx[ch], cy[b] - cy[ch], cz[b] - cz[ch]};
            h_m2m_add(&ts, &tt, rsrc, rtgt, k, d, src + (int64_t)(ch - src_level_start) * ts.nstored,
                      tgt + (int64_t)(b - tgt_level_start) * tt.nstored);
        }
    }
    hmi_free(&ts); hmi_free(&tt);
}

void oracle_helm_m2l_level(int p, double rs, double k, int32_t ntgt_boxes,
                           const int32_t *target_boxes, const int32_t *src_box_starts,
                           const int32_t *src_box_lists, const int32_t *entry_classes,
                           int32_t nclasses_level, int32_t class_level_start,
                           const double *class_vectors, int64_t class_stride,
                           int32_t level_start_ibox, const double *mpd, double *locd)
{
    hmi t; hmi_init(&t, p);
    const cplx *mp = (const cplx *)mpd;
    cplx *loc = (cplx *)locd;
    int nc = 3 * (2 * p + 1) * (2 * p + 1);
    cplx *data = malloc(sizeof(cplx) * (size_t)nc * (nclasses_level > 0 ? nclasses_level : 1));
#pragma omp parallel
    {
        cplx *tab = malloc(sizeof(cplx) * 2 * (2 * p + 1) * (2 * p + 1));
#pragma omp for schedule(dynamic, 4)
        for (int32_t c = 0; c < nclasses_level; ++c) {
            int64_t gc = class_level_start + c;
            double d[3] = {class_vectors[gc], class_vectors[class_stride + gc],
                           class_vectors[2 * class_stride + gc]};
            h_m2l_class_data(&t, rs, k, d, data + (size_t)c * nc, tab);
        }
        free(tab);
        cplx *mc = malloc(sizeof(cplx) * nc);
#pragma omp for schedule(dynamic, 8)
        for (int32_t i = 0; i < ntgt_boxes; ++i) {
            int32_t tb = target_boxes[i];
            cplx *out = loc + (int64_t)(tb - level_start_ibox) * t.nstored;
            for (int32_t l = src_box_starts[i]; l < src_box_starts[i + 1]; ++l) {
                int32_t sb = src_box_lists[l];
                int32_t c = entry_classes[l] - class_level_start;
                h_m2l_apply_add(&t, rs, rs, data + (size_t)c * nc,
                                mp + (int64_t)(sb - level_start_ibox) * t.nstored, out, mc);
            }
        }
        free(mc);
    }
    free(data);
    hmi_free(&t);
}

void oracle_helm_m2p_level(int p, double rs, double k, int32_t ntgt_boxes,
                           const int32_t *target_boxes, const int32_t *src_box_starts,
                           const int32_t *src_box_lists, const double *cx, const double *cy,
                           const double *cz, int32_t src_level_start, const double *mpd,
                           const int32_t *box_tgt_starts, const int32_t *box_tgt_counts,
                           const double *tx, const double *ty, const double *tz, double *potd)
{
    hmi t; hmi_init(&t, p);
    const cplx *mp = (const cplx *)mpd;
    cplx *pot = (cplx *)potd;
    const double scale = 1.0 / (4.0 * M_PI);
#pragma omp parallel
    {
        cplx *tab = malloc(sizeof(cplx) * 2 * (p + 1) * (p + 1));
#pragma omp for schedule(dynamic, 8)
        for (int32_t i = 0; i < ntgt_boxes; ++i) {
            int32_t tb = target_boxes[i];
            for (int32_t tg = box_tgt_starts[tb]; tg < box_tgt_starts[tb] + box_tgt_counts[tb]; ++tg) {
                cplx acc = 0.0;
                for (int32_t l = src_box_starts[i]; l < src_box_starts[i + 1]; ++l) {
                    int32_t sb = src_box_lists[l];
                    double b[3] = {tx[tg] - cx[sb], ty[tg] - cy[sb], tz[tg] - cz[sb]};
                    acc += h_m2p_eval(&t, rs, k, mp + (int64_t)(sb - src_level_start) * t.nstored,
                                      b, tab);
                }
                pot[tg] += scale * acc;
            }
        }
        free(tab);
    }
    hmi_free(&t);
}

void oracle_helm_p2l_level(int p, double rs, double k, int32_t ntgt_boxes,
                           const int32_t *target_boxes, const int32_t *src_box_starts,
                           const int32_t *src_box_lists, const double *cx, const double *cy,
                           const double *cz, const int32_t *box_src_starts,
                           const int32_t *box_src_counts, const double *sx, const double *sy,
                           const double *sz, const double *qd, int32_t level_start_ibox,
                           double *locd)
{
    hmi t; hmi_init(&t, p);
    const cplx *q = (const cplx *)qd;
    cplx *loc = (cplx *)locd;
#pragma omp parallel
    {
        cplx *tab = malloc(sizeof(cplx) * 2 * (p + 1) * (p + 1));
        cplx *acc = malloc(sizeof(cplx) * t.nstored);
#pragma omp for schedule(dynamic, 8)
        for (int32_t i = 0; i < ntgt_boxes; ++i) {
            int32_t tb = target_boxes[i];
            double c[3] = {cx[tb], cy[tb], cz[tb]};
            for (int m = 0; m < t.nstored; ++m) acc[m] = 0.0;
            for (int32_t l = src_box_starts[i]; l < src_box_starts[i + 1]; ++l) {
                int32_t sb = src_box_lists[l];
                int32_t s0 = box_src_starts[sb];
                h_p2l_add(&t, rs, k, c, box_src_counts[sb], sx + s0, sy + s0, sz + s0, q + s0,
                          acc, tab);
            }
            cplx *out = loc + (int64_t)(tb - level_start_ibox) * t.nstored;
            for (int m = 0; m < t.nstored; ++m) out[m] = acc[m];
        }
        free(tab); free(acc);
    }
    hmi_free(&t);
}

void oracle_helm_l2l_level(int psrc, int ptgt, double rsrc, double rtgt, double k,
                           int32_t nboxes, const int32_t *boxes, const int32_t *box_parent_ids,
                           const double *cx, const double *cy, const double *cz,
                           int32_t src_level_start, const double *srcd,
                           int32_t tgt_level_start, double *tgtd)
{
    hmi ts, tt; hmi_init(&ts, psrc); hmi_init(&tt, ptgt);
    const cplx *src = (const cplx *)srcd;
    cplx *tgt = (cplx *)tgtd;
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < nboxes; ++i) {
        int32_t b = boxes[i];
        int32_t par = box_parent_ids[b];
        double d[3] = {cx[b] - cx[par], cy[b] - cy[par], cz[b] - cz[par]};
        h_l2l_add(&ts, &tt, rsrc, rtgt, k, d, src + (int64_t)(par - src_level_start) * ts.nstored,
                  tgt + (int64_t)(b - tgt_level_start) * tt.nstored);
    }
    hmi_free(&ts); hmi_free(&tt);
}

void oracle_helm_l2p_level(int p, double rs, double k, int32_t nboxes, const int32_t *boxes,
                           const double *cx, const double *cy, const double *cz,
                           int32_t level_start_ibox, const double *locd,
                           const int32_t *box_tgt_starts, const int32_t *box_tgt_counts,
                           const double *tx, const double *ty, const double *tz, double *potd)
{
    hmi t; hmi_init(&t, p);
    const cplx *loc = (const cplx *)locd;
    cplx *pot = (cplx *)potd;
    const double scale = 1.0 / (4.0 * M_PI);
#pragma omp parallel
    {
        cplx *full = malloc(sizeof(cplx) * t.nfull);
#pragma omp for schedule(dynamic, 16)
        for (int32_t i = 0; i < nboxes; ++i) {
            int32_t b = boxes[i];
            const cplx *co = loc + (int64_t)(b - level_start_ibox) * t.nstored;
            for (int32_t tg = box_tgt_starts[b]; tg < box_tgt_starts[b] + box_tgt_counts[b]; ++tg) {
                double bv[3] = {tx[tg] - cx[b], ty[tg] - cy[b], tz[tg] - cz[b]};
                pot[tg] = scale * h_l2p_eval(&t, rs, k, co, bv, full);
            }
        }
        free(full);
    }
    hmi_free(&t);
}
