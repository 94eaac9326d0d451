/*
 * fmm_oracle.c -- FP64 CPU restatement of sumpy's 3D Laplace FMM operators.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the oracle: only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline / reference arm of bench.py
 * may load it, and only as the checker or the timed CPU baseline. The product
 * (sumpy_b200) never calls it.
 *
 * Every routine restates the reference algorithm it cites (paths relative to
 * the sumpy source tree). Conventions (sumpy MEMO): a = center - source,
 * b = target - center, d = target center - source center. Kernel G = 1/|x|;
 * the 1/(4 pi) scaling is applied only where sumpy applies it, on point
 * outputs (sumpy/p2p.py:617, sumpy/e2p.py:167,285-287).
 *
 * Coefficient sets (sumpy/expansion/__init__.py:563-886, Laplace 3D):
 *   full ids   = all mi with |mi| <= p, sorted by (|mi|, mi0, mi1, mi2)
 *   stored ids = full ids with mi0 < 2, same order, (p+1)^2 of them
 *   projection = u_mi = -u_{mi-2e0+2e1} - u_{mi-2e0+2e2} for mi0 >= 2
 *                (rscale factors cancel: both terms have the same degree).
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -shared).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXP 32

/* ------------------------------------------------------------------ */
/* multi-index tables                                                  */
/* ------------------------------------------------------------------ */

typedef struct {
    int p;
    int nfull, nstored;
    int (*full)[3];        /* full ids in sumpy order */
    int (*stored)[3];      /* stored ids in sumpy order */
    int *lut;              /* (p+1)^3 -> full index or -1 */
    int *stored_of_full;   /* full index -> stored index or -1 */
} mi_table;

static int lut_at(const mi_table *t, int i, int j, int k)
{
    if (i < 0 || j < 0 || k < 0 || i + j + k > t->p) return -1;
    return t->lut[(i * (t->p + 1) + j) * (t->p + 1) + k];
}

/* sumpy/expansion/__init__.py:299-313 (ids with |mi| <= p) sorted with the
 * degree-lexicographic key of LinearPDEBasedExpansionTermsWrangler
 * (__init__.py:643-652 for Laplace: axis permutation is the identity). */
static void mi_table_init(mi_table *t, int p)
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

static void mi_table_free(mi_table *t)
{
    free(t->full); free(t->stored); free(t->lut); free(t->stored_of_full);
}

static double factorial(int n)
{
    double r = 1.0;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
}

/* Stored local coefficients -> full derivative set.
 * CSEMatVecOperator.matvec of the projection matrix (__init__.py:510-531,
 * rows built at 830-853): rows in full order; non-stored rows combine
 * earlier outputs. */
static void project_to_full(const mi_table *t, const double *stored, double *full)
{
    for (int f = 0; f < t->nfull; ++f) {
        int s = t->stored_of_full[f];
        if (s >= 0) { full[f] = stored[s]; continue; }
        const int *mi = t->full[f];
        int a = lut_at(t, mi[0] - 2, mi[1] + 2, mi[2]);
        int b = lut_at(t, mi[0] - 2, mi[1], mi[2] + 2);
        full[f] = -full[a] - full[b];
    }
}

/* Full multipole coefficients -> stored.
 * CSEMatVecOperator.transpose_matvec (__init__.py:533-548): rows walked in
 * reverse; non-stored rows push their value onto the outputs they refer to. */
static void compress_from_full(const mi_table *t, const double *full_in, double *stored)
{
    double *work = malloc(sizeof(double) * t->nfull);
    memcpy(work, full_in, sizeof(double) * t->nfull);
    for (int s = 0; s < t->nstored; ++s) stored[s] = 0.0;
    for (int f = t->nfull - 1; f >= 0; --f) {
        int s = t->stored_of_full[f];
        if (s >= 0) { stored[s] += work[f]; continue; }
        const int *mi = t->full[f];
        int a = lut_at(t, mi[0] - 2, mi[1] + 2, mi[2]);
        int b = lut_at(t, mi[0] - 2, mi[1], mi[2] + 2);
        work[a] += -work[f];
        work[b] += -work[f];
    }
    free(work);
}

/* ------------------------------------------------------------------ */
/* Laplace derivative recurrence                                        */
/* ------------------------------------------------------------------ */

/* Scaled derivatives D[mi] = rscale^|mi| d^mi (1/|x|) at x, for mi with
 * mi0 <= maxi0 and |mi| <= maxdeg, stored in tab[(i*(M+1)+j)*(M+1)+k],
 * M = maxdeg. LaplaceDerivativeTaker.diff (sumpy/derivative_taker.py:211-262):
 * entries with max(mi) <= 1 come from direct differentiation times rscale
 * per derivative (ExprDerivativeTaker.diff, derivative_taker.py:156-174);
 * the rest from the 3D recurrence in the scaled variables x/rscale. */
static void laplace_derivs(const double x[3], double rscale, int maxi0, int maxdeg,
                           double *tab)
{
    const int M = maxdeg;
#define T(i, j, k) tab[((i) * (M + 1) + (j)) * (M + 1) + (k)]
    double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    double r = sqrt(r2);
    double xs[3] = {x[0] / rscale, x[1] / rscale, x[2] / rscale};
    double rs2 = xs[0] * xs[0] + xs[1] * xs[1] + xs[2] * xs[2];
    for (int deg = 0; deg <= maxdeg; ++deg)
        for (int i = 0; i <= (deg < maxi0 ? deg : maxi0); ++i)
            for (int j = 0; j <= deg - i; ++j) {
                int k = deg - i - j;
                int mi[3] = {i, j, k};
                int mx = i > j ? i : j; if (k > mx) mx = k;
                if (mx <= 1) {
                    /* d^mi (1/r) for mi in {0,1}^3 */
                    double v;
                    int o = i + j + k;
                    if (o == 0) v = 1.0 / r;
                    else if (o == 1) {
                        double c = i ? x[0] : (j ? x[1] : x[2]);
                        v = -c / (r2 * r);
                    } else if (o == 2) {
                        double c1 = i ? x[0] : x[1];
                        double c2 = k ? x[2] : x[1];
                        v = 3.0 * c1 * c2 / (r2 * r2 * r);
                    } else {
                        v = -15.0 * x[0] * x[1] * x[2] / (r2 * r2 * r2 * r);
                    }
                    for (int q = 0; q < o; ++q) v *= rscale;
                    T(i, j, k) = v;
                    continue;
                }
                int d = (i >= 2) ? 0 : ((j >= 2) ? 1 : 2);
                double e = 0.0;
                for (int ax = 0; ax < 3; ++ax) {
                    int n = mi[ax];
                    int m1[3] = {i, j, k}, m2[3] = {i, j, k};
                    m1[ax] -= 1; m2[ax] -= 2;
                    double d1 = (m1[ax] >= 0) ? T(m1[0], m1[1], m1[2]) : 0.0;
                    double d2 = (m2[ax] >= 0) ? T(m2[0], m2[1], m2[2]) : 0.0;
                    if (ax == d) {
                        e -= (2 * n - 1) * xs[ax] * d1;
                        e -= (double)(n - 1) * (n - 1) * d2;
                    } else {
                        e -= 2 * n * xs[ax] * d1;
                        e -= (double)n * (n - 1) * d2;
                    }
                }
                T(i, j, k) = e / rs2;
            }
#undef T
}

/* ------------------------------------------------------------------ */
/* point-level operators                                                */
/* ------------------------------------------------------------------ */

int oracle_ncoeff(int p) { return (p + 1) * (p + 1); }

/* threads a parallel region of this library runs on (the CPU baseline's core count) */
int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
int oracle_nfull(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }

void oracle_stored_ids(int p, int *ids)
{
    mi_table t; mi_table_init(&t, p);
    memcpy(ids, t.stored, sizeof(int[3]) * t.nstored);
    mi_table_free(&t);
}

void oracle_full_ids(int p, int *ids)
{
    mi_table t; mi_table_init(&t, p);
    memcpy(ids, t.full, sizeof(int[3]) * t.nfull);
    mi_table_free(&t);
}

/* P2M for one box: VolumeTaylorMultipoleExpansionBase.coefficients_from_source_vec
 * (sumpy/expansion/multipole.py:77-114): full coefficients
 * sum_s q_s (a_s/r)^mi / mi!, then the transposed projection. */
static void p2m_box(const mi_table *t, double rscale, const double c[3], int n,
                    const double *sx, const double *sy, const double *sz,
                    const double *q, double *out)
{
    double *full = calloc(t->nfull, sizeof(double));
    for (int s = 0; s < n; ++s) {
        double a[3] = {(c[0] - sx[s]) / rscale, (c[1] - sy[s]) / rscale,
                       (c[2] - sz[s]) / rscale};
        for (int f = 0; f < t->nfull; ++f) {
            const int *mi = t->full[f];
            double v = q[s];
            for (int ax = 0; ax < 3; ++ax)
                v *= pow(a[ax], mi[ax]) / factorial(mi[ax]);
            full[f] += v;
        }
    }
    compress_from_full(t, full, out);
    free(full);
}

void oracle_p2m_point(int p, double rscale, const double *center, int n,
                      const double *sx, const double *sy, const double *sz,
                      const double *q, double *out)
{
    mi_table t; mi_table_init(&t, p);
    p2m_box(&t, rscale, center, n, sx, sy, sz, q, out);
    mi_table_free(&t);
}

/* P2L for one (box, sources) pair, accumulating: VolumeTaylorLocalExpansionBase
 * .coefficients_from_source_vec (sumpy/expansion/local.py:225-271). */
static void p2l_add(const mi_table *t, double rscale, const double c[3], int n,
                    const double *sx, const double *sy, const double *sz,
                    const double *q, double *out, double *tab)
{
    int p = t->p;
    for (int s = 0; s < n; ++s) {
        double a[3] = {c[0] - sx[s], c[1] - sy[s], c[2] - sz[s]};
        laplace_derivs(a, rscale, 1, p, tab);
        for (int st = 0; st < t->nstored; ++st) {
            const int *mi = t->stored[st];
            out[st] += q[s] * tab[(mi[0] * (p + 1) + mi[1]) * (p + 1) + mi[2]];
        }
    }
}

void oracle_p2l_point(int p, double rscale, const double *center, int n,
                      const double *sx, const double *sy, const double *sz,
                      const double *q, double *out)
{
    mi_table t; mi_table_init(&t, p);
    double *tab = malloc(sizeof(double) * (p + 1) * (p + 1) * (p + 1));
    for (int i = 0; i < t.nstored; ++i) out[i] = 0.0;
    p2l_add(&t, rscale, center, n, sx, sy, sz, q, out, tab);
    free(tab);
    mi_table_free(&t);
}

/* L2P at one target (no kernel scaling): VolumeTaylorLocalExpansionBase.evaluate
 * (sumpy/expansion/local.py:284-309). */
static double l2p_eval(const mi_table *t, double rscale, const double *coeffs,
                       const double b[3], double *full)
{
    project_to_full(t, coeffs, full);
    double bs[3] = {b[0] / rscale, b[1] / rscale, b[2] / rscale};
    double acc = 0.0;
    for (int f = 0; f < t->nfull; ++f) {
        const int *mi = t->full[f];
        double v = full[f];
        for (int ax = 0; ax < 3; ++ax) v *= pow(bs[ax], mi[ax]) / factorial(mi[ax]);
        acc += v;
    }
    return acc;
}

double oracle_l2p_point(int p, double rscale, const double *coeffs, const double *b)
{
    mi_table t; mi_table_init(&t, p);
    double *full = malloc(sizeof(double) * t.nfull);
    double v = l2p_eval(&t, rscale, coeffs, b, full);
    free(full);
    mi_table_free(&t);
    return v;
}

/* M2P at one target (no kernel scaling): VolumeTaylorMultipoleExpansionBase
 * .evaluate (sumpy/expansion/multipole.py:131-157). */
static double m2p_eval(const mi_table *t, double rscale, const double *coeffs,
                       const double b[3], double *tab)
{
    int p = t->p;
    laplace_derivs(b, rscale, 1, p, tab);
    double acc = 0.0;
    for (int st = 0; st < t->nstored; ++st) {
        const int *mi = t->stored[st];
        acc += coeffs[st] * tab[(mi[0] * (p + 1) + mi[1]) * (p + 1) + mi[2]];
    }
    return acc;
}

double oracle_m2p_point(int p, double rscale, const double *coeffs, const double *b)
{
    mi_table t; mi_table_init(&t, p);
    double *tab = malloc(sizeof(double) * (p + 1) * (p + 1) * (p + 1));
    double v = m2p_eval(&t, rscale, coeffs, b, tab);
    free(tab);
    mi_table_free(&t);
    return v;
}

/* M2M, accumulating into out: the default (_fast_version) path of
 * VolumeTaylorMultipoleExpansionBase.translate_from
 * (sumpy/expansion/multipole.py:159-348, 400-407). For Laplace the stored
 * ids all lie on hyperplanes normal to axis 0, so one pass over the axes
 * (1, 2, 0) performs the shift, followed by the transposed projection. */
static void m2m_add(const mi_table *ts, const mi_table *tt, double rsrc, double rtgt,
                    const double dvec[3], const double *in, double *out)
{
    int nf = tt->nfull;
    double *cur = calloc(nf, sizeof(double));
    double *nxt = calloc(nf, sizeof(double));
    double *res = malloc(sizeof(double) * tt->nstored);
    double ratio = rsrc / rtgt;
    for (int st = 0; st < tt->nstored; ++st) {
        const int *mi = tt->stored[st];
        int si = lut_at(ts, mi[0], mi[1], mi[2]);
        if (si < 0 || ts->stored_of_full[si] < 0) continue;
        int f = lut_at(tt, mi[0], mi[1], mi[2]);
        cur[f] = in[ts->stored_of_full[si]] * pow(ratio, mi[0] + mi[1] + mi[2]);
    }
    const int dims[3] = {1, 2, 0};
    for (int di = 0; di < 3; ++di) {
        int d = dims[di];
        double dd = dvec[d] / rtgt;
        for (int f = 0; f < nf; ++f) {
            const int *tm = tt->full[f];
            double acc = 0.0;
            for (int k = 0; k <= tm[d]; ++k) {
                int im[3] = {tm[0], tm[1], tm[2]};
                im[d] = k;
                double v = cur[lut_at(tt, im[0], im[1], im[2])];
                v /= factorial(tm[d] - k);
                v *= pow(dd, tm[d] - k);
                acc += v;
            }
            nxt[f] = acc;
        }
        double *sw = cur; cur = nxt; nxt = sw;
    }
    compress_from_full(tt, cur, res);
    for (int st = 0; st < tt->nstored; ++st) out[st] += res[st];
    free(cur); free(nxt); free(res);
}

void oracle_m2m_point(int psrc, int ptgt, double rsrc, double rtgt,
                      const double *dvec, const double *in, double *out)
{
    mi_table ts, tt; mi_table_init(&ts, psrc); mi_table_init(&tt, ptgt);
    for (int i = 0; i < tt.nstored; ++i) out[i] = 0.0;
    m2m_add(&ts, &tt, rsrc, rtgt, dvec, in, out);
    mi_table_free(&ts); mi_table_free(&tt);
}

/* L2L, accumulating into out: the default path of
 * VolumeTaylorLocalExpansionBase.translate_from (sumpy/expansion/local.py:346-464):
 * full derivatives from stored, Taylor shift one axis at a time (axes 0,1,2),
 * truncated to total degree <= p_src, times (r_tgt/r_src)^|mi|. */
static void l2l_add(const mi_table *ts, const mi_table *tt, double rsrc, double rtgt,
                    const double dvec[3], const double *in, double *out)
{
    int nf = ts->nfull, p = ts->p;
    double *cur = malloc(sizeof(double) * nf);
    double *nxt = malloc(sizeof(double) * nf);
    project_to_full(ts, in, cur);
    for (int d = 0; d < 3; ++d) {
        double dd = dvec[d] / rsrc;
        for (int f = 0; f < nf; ++f) {
            const int *om = ts->full[f];
            int deg = om[0] + om[1] + om[2];
            double acc = 0.0;
            for (int q = 0; q <= p - deg; ++q) {
                int sm[3] = {om[0], om[1], om[2]};
                sm[d] += q;
                acc += pow(dd, q) * cur[lut_at(ts, sm[0], sm[1], sm[2])] / factorial(q);
            }
            nxt[f] = acc;
        }
        double *sw = cur; cur = nxt; nxt = sw;
    }
    double ratio = rtgt / rsrc;
    for (int st = 0; st < tt->nstored; ++st) {
        const int *mi = tt->stored[st];
        int f = lut_at(ts, mi[0], mi[1], mi[2]);
        if (f < 0) continue;
        out[st] += cur[f] * pow(ratio, mi[0] + mi[1] + mi[2]);
    }
    free(cur); free(nxt);
}

void oracle_l2l_point(int psrc, int ptgt, double rsrc, double rtgt,
                      const double *dvec, const double *in, double *out)
{
    mi_table ts, tt; mi_table_init(&ts, psrc); mi_table_init(&tt, ptgt);
    for (int i = 0; i < tt.nstored; ++i) out[i] = 0.0;
    l2l_add(&ts, &tt, rsrc, rtgt, dvec, in, out);
    mi_table_free(&ts); mi_table_free(&tt);
}

/* ------------------------------------------------------------------ */
/* M2L (translation-class form)                                         */
/* ------------------------------------------------------------------ */

/* Circulant-grid derivative vector for one translation vector:
 * VolumeTaylorM2LTranslation.translation_classes_dependent_data
 * (sumpy/expansion/m2l.py:461-537) with the index set of
 * _translation_classes_dependent_data_mis (m2l.py:403-459). Grid extents are
 * max_mi = (2, 2p, 2p) + 1 per axis, C order. Derivatives with mi0 <= 1 come
 * from the recurrence; mi0 == 2 from the Laplace projection. Entries that are
 * not a sum (src id + tgt id) stay zero. */
typedef struct {
    int p;
    int ext[3];
    int ncirc;
} circ_grid;

static void circ_init(circ_grid *g, int p)
{
    g->p = p;
    g->ext[0] = 3; g->ext[1] = 2 * p + 1; g->ext[2] = 2 * p + 1;
    g->ncirc = g->ext[0] * g->ext[1] * g->ext[2];
}

static int circ_index(const circ_grid *g, int i, int j, int k)
{
    return (i * g->ext[1] + j) * g->ext[2] + k;
}

static void m2l_class_data(const mi_table *t, const circ_grid *g, double rsrc,
                           const double dvec[3], double *dcirc, double *tab)
{
    int p = t->p, M = 2 * p;
    laplace_derivs(dvec, rsrc, 1, M, tab);
    for (int i = 0; i < g->ncirc; ++i) dcirc[i] = 0.0;
    for (int a = 0; a < t->nstored; ++a)
        for (int b = 0; b < t->nstored; ++b) {
            int m[3] = {t->stored[a][0] + t->stored[b][0],
                        t->stored[a][1] + t->stored[b][1],
                        t->stored[a][2] + t->stored[b][2]};
            double v;
            if (m[0] < 2) {
                v = tab[(m[0] * (M + 1) + m[1]) * (M + 1) + m[2]];
            } else {
                v = -tab[(0 * (M + 1) + m[1] + 2) * (M + 1) + m[2]]
                    - tab[(0 * (M + 1) + m[1]) * (M + 1) + m[2] + 2];
            }
            dcirc[circ_index(g, m[0], m[1], m[2])] = v;
        }
}

/* Apply one M2L with precomputed class data, accumulating into out:
 * preprocess (m2l.py:539-558, scatter stored mpole coefficients into the
 * circulant grid), Toeplitz matvec (sumpy/tools.py:689-701:
 * out[row] = sum_{col >= row} first_row[col-row] * vector[col], with the
 * multipole as first row and the derivatives as vector), postprocess
 * (m2l.py:679-698: pick the target ids, times (r_tgt/r_src)^|mi|). Only
 * the rows kept by postprocessing are formed. */
static void m2l_apply_add(const mi_table *t, const circ_grid *g, double rsrc,
                          double rtgt, const double *dcirc, const double *in,
                          double *out, double *mcirc)
{
    for (int i = 0; i < g->ncirc; ++i) mcirc[i] = 0.0;
    for (int s = 0; s < t->nstored; ++s)
        mcirc[circ_index(g, t->stored[s][0], t->stored[s][1], t->stored[s][2])] = in[s];
    double ratio = rtgt / rsrc;
    for (int tt = 0; tt < t->nstored; ++tt) {
        const int *mi = t->stored[tt];
        int row = circ_index(g, mi[0], mi[1], mi[2]);
        double acc = 0.0;
        for (int col = row; col < g->ncirc; ++col)
            acc += mcirc[col - row] * dcirc[col];
        out[tt] += acc * pow(ratio, mi[0] + mi[1] + mi[2]);
    }
}

void oracle_m2l_point(int p, double rsrc, double rtgt, const double *dvec,
                      const double *in, double *out)
{
    mi_table t; mi_table_init(&t, p);
    circ_grid g; circ_init(&g, p);
    double *tab = malloc(sizeof(double) * (2 * p + 1) * (2 * p + 1) * (2 * p + 1));
    double *dc = malloc(sizeof(double) * g.ncirc);
    double *mc = malloc(sizeof(double) * g.ncirc);
    m2l_class_data(&t, &g, rsrc, dvec, dc, tab);
    for (int i = 0; i < t.nstored; ++i) out[i] = 0.0;
    m2l_apply_add(&t, &g, rsrc, rtgt, dc, in, out, mc);
    free(tab); free(dc); free(mc);
    mi_table_free(&t);
}

/* ------------------------------------------------------------------ */
/* FMM stages over a tree (the wrangler methods, sumpy/fmm.py:609-1083) */
/* ------------------------------------------------------------------ */

/* Direct sum (sumpy/p2p.py:215-285; exclude_self as in p2p.py:162-170):
 * pot[t] = 1/(4 pi) sum_s q_s / |t - s|, skipping s == target_to_source[t]
 * when that array is given. */
void oracle_p2p_direct(int64_t ntgt, const double *tx, const double *ty,
                       const double *tz, int64_t nsrc, const double *sx,
                       const double *sy, const double *sz, const double *q,
                       const int32_t *target_to_source, double *pot)
{
    const double scale = 1.0 / (4.0 * M_PI);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t t = 0; t < ntgt; ++t) {
        double acc = 0.0;
        int64_t self = target_to_source ? target_to_source[t] : -1;
        for (int64_t s = 0; s < nsrc; ++s) {
            if (s == self) continue;
            double dx = tx[t] - sx[s], dy = ty[t] - sy[s], dz = tz[t] - sz[s];
            acc += q[s] / sqrt(dx * dx + dy * dy + dz * dz);
        }
        pot[t] = scale * acc;
    }
}

/* P2PFromCSR (sumpy/p2p.py:484-670, CPU variant 626-670): result is
 * assigned (not accumulated) for every target of every listed target box. */
void oracle_p2p_csr(int32_t ntgt_boxes, const int32_t *target_boxes,
                    const int32_t *src_box_starts, const int32_t *src_box_lists,
                    const int32_t *box_src_starts, const int32_t *box_src_counts,
                    const int32_t *box_tgt_starts, const int32_t *box_tgt_counts,
                    const double *sx, const double *sy, const double *sz,
                    const double *q, const double *tx, const double *ty,
                    const double *tz, const int32_t *target_to_source, double *pot)
{
    const double scale = 1.0 / (4.0 * M_PI);
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t ib = 0; ib < ntgt_boxes; ++ib) {
        int32_t tb = target_boxes[ib];
        for (int32_t t = box_tgt_starts[tb]; t < box_tgt_starts[tb] + box_tgt_counts[tb]; ++t) {
            double acc = 0.0;
            int32_t self = target_to_source ? target_to_source[t] : -1;
            for (int32_t l = src_box_starts[ib]; l < src_box_starts[ib + 1]; ++l) {
                int32_t sb = src_box_lists[l];
                for (int32_t s = box_src_starts[sb]; s < box_src_starts[sb] + box_src_counts[sb]; ++s) {
                    if (s == self) continue;
                    double dx = tx[t] - sx[s], dy = ty[t] - sy[s], dz = tz[t] - sz[s];
                    acc += q[s] / sqrt(dx * dx + dy * dy + dz * dz);
                }
            }
            pot[t] = scale * acc;
        }
    }
}

/* form_multipoles for one level (fmm.py:609-641 -> P2EFromSingleBox,
 * sumpy/p2e.py:155-261): expansions of the listed boxes are assigned. */
void oracle_p2m_level(int p, double rscale, int32_t nboxes, const int32_t *boxes,
                      int32_t level_start_ibox, const double *cx, const double *cy,
                      const double *cz, const int32_t *box_src_starts,
                      const int32_t *box_src_counts, const double *sx,
                      const double *sy, const double *sz, const double *q,
                      double *mpoles_level)
{
    mi_table t; mi_table_init(&t, p);
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < nboxes; ++i) {
        int32_t b = boxes[i];
        double c[3] = {cx[b], cy[b], cz[b]};
        int32_t s0 = box_src_starts[b];
        p2m_box(&t, rscale, c, box_src_counts[b], sx + s0, sy + s0, sz + s0, q + s0,
                mpoles_level + (int64_t)(b - level_start_ibox) * t.nstored);
    }
    mi_table_free(&t);
}

/* coarsen_multipoles for one (source level -> target level) step
 * (fmm.py:643-695 -> E2EFromChildren, sumpy/e2e.py:866-978):
 * parent += M2M(child) over nonzero box_child_ids. box_child_ids is
 * [8][nboxes_aligned] with stride child_stride. */
void oracle_m2m_level(int psrc, int ptgt, double rsrc, double rtgt, int32_t nboxes,
                      const int32_t *boxes, const int32_t *box_child_ids,
                      int64_t child_stride, const double *cx, const double *cy,
                      const double *cz, int32_t src_level_start, const double *src_mp,
                      int32_t tgt_level_start, double *tgt_mp)
{
    mi_table ts, tt; mi_table_init(&ts, psrc); mi_table_init(&tt, ptgt);
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < nboxes; ++i) {
        int32_t b = boxes[i];
        for (int c = 0; c < 8; ++c) {
            int32_t ch = box_child_ids[c * child_stride + b];
            if (ch == 0) continue;
            double d[3] = {cx[b] - cx[ch], cy[b] - cy[ch], cz[b] - cz[ch]};
            m2m_add(&ts, &tt, rsrc, rtgt, d,
                    src_mp + (int64_t)(ch - src_level_start) * ts.nstored,
                    tgt_mp + (int64_t)(b - tgt_level_start) * tt.nstored);
        }
    }
    mi_table_free(&ts); mi_table_free(&tt);
}

/* multipole_to_local for one level with translation classes
 * (fmm.py:723-920; M2LUsingTranslationClassesDependentData, e2e.py:310-558):
 * class data computed once per class for this level from the class distance
 * vectors (fmm.py:752-754), then per List-2 entry the Toeplitz apply.
 * class_vectors is [3][nclasses_total] (stride class_stride); classes of
 * this level are class_level_start + class index. */
void oracle_m2l_level(int p, double rscale, int32_t ntgt_boxes,
                      const int32_t *target_boxes, const int32_t *src_box_starts,
                      const int32_t *src_box_lists, const int32_t *entry_classes,
                      int32_t nclasses_level, int32_t class_level_start,
                      const double *class_vectors, int64_t class_stride,
                      int32_t level_start_ibox, const double *mp_level,
                      double *loc_level)
{
    mi_table t; mi_table_init(&t, p);
    circ_grid g; circ_init(&g, p);
    double *data = malloc(sizeof(double) * (size_t)g.ncirc * (nclasses_level > 0 ? nclasses_level : 1));
#pragma omp parallel
    {
        double *tab = malloc(sizeof(double) * (2 * p + 1) * (2 * p + 1) * (2 * p + 1));
#pragma omp for schedule(dynamic, 4)
        for (int32_t c = 0; c < nclasses_level; ++c) {
            int64_t gc = class_level_start + c;
            double d[3] = {class_vectors[gc], class_vectors[class_stride + gc],
                           class_vectors[2 * class_stride + gc]};
            m2l_class_data(&t, &g, rscale, d, data + (size_t)c * g.ncirc, tab);
        }
        free(tab);
        double *mc = malloc(sizeof(double) * g.ncirc);
#pragma omp for schedule(dynamic, 8)
        for (int32_t i = 0; i < ntgt_boxes; ++i) {
            int32_t tb = target_boxes[i];
            double *out = loc_level + (int64_t)(tb - level_start_ibox) * t.nstored;
            for (int32_t l = src_box_starts[i]; l < src_box_starts[i + 1]; ++l) {
                int32_t sb = src_box_lists[l];
                int32_t c = entry_classes[l] - class_level_start;
                m2l_apply_add(&t, &g, rscale, rscale, data + (size_t)c * g.ncirc,
                              mp_level + (int64_t)(sb - level_start_ibox) * t.nstored,
                              out, mc);
            }
        }
        free(mc);
    }
    free(data);
    mi_table_free(&t);
}

/* eval_multipoles for one source level (fmm.py:922-961 -> E2PFromCSR,
 * sumpy/e2p.py:233-343): pot[t] += 1/(4 pi) sum over listed source boxes. */
void oracle_m2p_level(int p, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
                      const int32_t *src_box_starts, const int32_t *src_box_lists,
                      const double *cx, const double *cy, const double *cz,
                      int32_t src_level_start, const double *mp_level,
                      const int32_t *box_tgt_starts, const int32_t *box_tgt_counts,
                      const double *tx, const double *ty, const double *tz, double *pot)
{
    mi_table t; mi_table_init(&t, p);
    const double scale = 1.0 / (4.0 * M_PI);
#pragma omp parallel
    {
        double *tab = malloc(sizeof(double) * (p + 1) * (p + 1) * (p + 1));
#pragma omp for schedule(dynamic, 8)
        for (int32_t i = 0; i < ntgt_boxes; ++i) {
            int32_t tb = target_boxes[i];
            for (int32_t tg = box_tgt_starts[tb]; tg < box_tgt_starts[tb] + box_tgt_counts[tb]; ++tg) {
                double acc = 0.0;
                for (int32_t l = src_box_starts[i]; l < src_box_starts[i + 1]; ++l) {
                    int32_t sb = src_box_lists[l];
                    double b[3] = {tx[tg] - cx[sb], ty[tg] - cy[sb], tz[tg] - cz[sb]};
                    acc += m2p_eval(&t, rscale,
                                    mp_level + (int64_t)(sb - src_level_start) * t.nstored,
                                    b, tab);
                }
                pot[tg] += scale * acc;
            }
        }
        free(tab);
    }
    mi_table_free(&t);
}

/* form_locals for one level (fmm.py:963-1002 -> P2EFromCSR, sumpy/p2e.py:268-388):
 * expansions of the listed boxes are assigned from their List-4 sources. */
void oracle_p2l_level(int p, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
                      const int32_t *src_box_starts, const int32_t *src_box_lists,
                      const double *cx, const double *cy, const double *cz,
                      const int32_t *box_src_starts, const int32_t *box_src_counts,
                      const double *sx, const double *sy, const double *sz,
                      const double *q, int32_t level_start_ibox, double *loc_level)
{
    mi_table t; mi_table_init(&t, p);
#pragma omp parallel
    {
        double *tab = malloc(sizeof(double) * (p + 1) * (p + 1) * (p + 1));
        double *acc = malloc(sizeof(double) * t.nstored);
#pragma omp for schedule(dynamic, 8)
        for (int32_t i = 0; i < ntgt_boxes; ++i) {
            int32_t tb = target_boxes[i];
            double c[3] = {cx[tb], cy[tb], cz[tb]};
            for (int k = 0; k < t.nstored; ++k) acc[k] = 0.0;
            for (int32_t l = src_box_starts[i]; l < src_box_starts[i + 1]; ++l) {
                int32_t sb = src_box_lists[l];
                int32_t s0 = box_src_starts[sb];
                p2l_add(&t, rscale, c, box_src_counts[sb], sx + s0, sy + s0, sz + s0,
                        q + s0, acc, tab);
            }
            double *out = loc_level + (int64_t)(tb - level_start_ibox) * t.nstored;
            for (int k = 0; k < t.nstored; ++k) out[k] = acc[k];
        }
        free(tab); free(acc);
    }
    mi_table_free(&t);
}

/* refine_locals for one (parent level -> child level) step
 * (fmm.py:1004-1045 -> E2EFromParent, sumpy/e2e.py:985-1083): child += L2L(parent). */
void oracle_l2l_level(int psrc, int ptgt, double rsrc, double rtgt, int32_t nboxes,
                      const int32_t *boxes, const int32_t *box_parent_ids,
                      const double *cx, const double *cy, const double *cz,
                      int32_t src_level_start, const double *src_loc,
                      int32_t tgt_level_start, double *tgt_loc)
{
    mi_table ts, tt; mi_table_init(&ts, psrc); mi_table_init(&tt, ptgt);
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < nboxes; ++i) {
        int32_t b = boxes[i];
        int32_t par = box_parent_ids[b];
        double d[3] = {cx[b] - cx[par], cy[b] - cy[par], cz[b] - cz[par]};
        l2l_add(&ts, &tt, rsrc, rtgt, d,
                src_loc + (int64_t)(par - src_level_start) * ts.nstored,
                tgt_loc + (int64_t)(b - tgt_level_start) * tt.nstored);
    }
    mi_table_free(&ts); mi_table_free(&tt);
}

/* eval_locals for one level (fmm.py:1047-1083 -> E2PFromSingleBox,
 * sumpy/e2p.py:123-226): pot[t] = 1/(4 pi) * L2P, assigned. */
void oracle_l2p_level(int p, double rscale, int32_t nboxes, const int32_t *boxes,
                      const double *cx, const double *cy, const double *cz,
                      int32_t level_start_ibox, const double *loc_level,
                      const int32_t *box_tgt_starts, const int32_t *box_tgt_counts,
                      const double *tx, const double *ty, const double *tz, double *pot)
{
    mi_table t; mi_table_init(&t, p);
    const double scale = 1.0 / (4.0 * M_PI);
#pragma omp parallel
    {
        double *full = malloc(sizeof(double) * t.nfull);
#pragma omp for schedule(dynamic, 16)
        for (int32_t i = 0; i < nboxes; ++i) {
            int32_t b = boxes[i];
            const double *co = loc_level + (int64_t)(b - level_start_ibox) * t.nstored;
            for (int32_t tg = box_tgt_starts[b]; tg < box_tgt_starts[b] + box_tgt_counts[b]; ++tg) {
                double bv[3] = {tx[tg] - cx[b], ty[tg] - cy[b], tz[tg] - cz[b]};
                pot[tg] = scale * l2p_eval(&t, rscale, co, bv, full);
            }
        }
        free(full);
    }
    mi_table_free(&t);
}
