/*
 * sumpy_b200.h -- C-ABI of the B200 (sm_100a) FMM evaluation kernels.
 *
 * Each entry point replaces one loopy kernel that sumpy's expansion wrangler
 * (sumpy/fmm.py:264-1086) launches per tree level, with the same argument
 * meaning: box-number arrays and CSR lists from the tree/traversal, level
 * views of the expansion arrays ("base_ibox" = first box number of the
 * level; expansion of box b at row b - base_ibox, coefficients contiguous),
 * SoA coordinates ([3][n] with the given stride), and in-place outputs.
 *
 * Conventions (sumpy MEMO): a = center - source, b = target - center,
 * d = target center - source center. Kernel 1/|x| for 3D Laplace; `scale`
 * (1/(4 pi)) multiplies point outputs only. Coefficients are sumpy's stored
 * set of the LinearPDEConformingVolumeTaylor expansions: the (p+1)^2
 * multi-indices with mi0 < 2 ordered by (|mi|, mi0, mi1, mi2)
 * (sumpy/expansion/__init__.py:643-752).
 *
 * All pointers are device pointers unless stated otherwise; nothing is
 * allocated by any entry point. `stream` is a cudaStream_t (NULL = legacy
 * default stream). Launches are asynchronous; the return value reports
 * argument errors and launch errors only. Errors from a kernel's own checks
 * are written to the optional `status` word (device int32, 0 = ok) where an
 * entry takes one.
 *
 * Return codes: 0 ok, 1 bad argument, 2 CUDA launch error, 3 unsupported
 * order/size. sumpy_last_error() gives a message for the calling thread.
 */
#ifndef SUMPY_B200_H
#define SUMPY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SUMPY_OK = 0,
    SUMPY_EINVAL = 1,
    SUMPY_ELAUNCH = 2,
    SUMPY_EUNSUPPORTED = 3
};

/* Largest expansion order the kernels accept. */
#define SUMPY_MAX_ORDER 16

int sumpy_version(void);
const char *sumpy_last_error(void);

/* ------------------------------------------------------------------ */
/* P2P                                                                  */
/* ------------------------------------------------------------------ */

/* List-1 near field. Replaces P2PFromCSR.__call__ (sumpy/p2p.py:801-833;
 * kernel p2p.py:484-799) as called by SumpyExpansionWrangler.eval_direct
 * (sumpy/fmm.py:697-721):
 *   result[t] = scale * sum_{src boxes in CSR} sum_s strength[s] / |t - s|
 * for every target t of every target box (assigned, not accumulated).
 * target_to_source (may be NULL) excludes the pair s == target_to_source[t]
 * (exclude_self, p2p.py:162-170). FP64 throughout. */
int sumpy_p2p_from_csr_f64(
    int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength,
    const double *targets, int64_t target_stride,
    const int32_t *target_to_source, double scale, double *result, void *stream);

/* Same contract, mixed precision: each coordinate split into FP32 hi + lo
 * parts, the pair offset (t_hi - s_hi) + (t_lo - s_lo), 1/r and the products
 * in FP32, partial sums over each 32 sources in FP32, the target's total in
 * FP64. */
int sumpy_p2p_from_csr_mixed(
    int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength,
    const double *targets, int64_t target_stride,
    const int32_t *target_to_source, double scale, double *result, void *stream);

/* Gradient form: also writes grad[d*target_stride + t] = scale * sum_s
 * strength[s] * d/dt_d (1/|t - s|) (sumpy's AxisTargetDerivative applied to
 * the Laplace kernel, sumpy/kernel.py:2331-2386); result may be NULL. Used
 * for position gradients of the adjoint. FP64, and mixed precision as
 * sumpy_p2p_from_csr_mixed. */
int sumpy_p2p_from_csr_grad_f64(
    int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength,
    const double *targets, int64_t target_stride,
    const int32_t *target_to_source, double scale, double *result, double *grad, void *stream);

int sumpy_p2p_from_csr_grad_mixed(
    int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength,
    const double *targets, int64_t target_stride,
    const int32_t *target_to_source, double scale, double *result, double *grad, void *stream);

/* All-pairs sum. Replaces P2P.__call__ (sumpy/p2p.py:267-285), the direct
 * evaluation sumpy's FMM tests compare against (sumpy/test/test_fmm.py:284-286).
 * result[t] = scale * sum_s strength[s]/|t - s|, skipping s ==
 * target_to_source[t] when that array is given. FP64. */
int sumpy_p2p_direct_f64(
    int64_t ntargets, const double *targets, int64_t target_stride,
    int64_t nsources, const double *sources, int64_t source_stride,
    const double *strength, const int32_t *target_to_source, double scale,
    double *result, void *stream);

/* Gradient of the direct sum: grad[d*target_stride + t] as in
 * sumpy_p2p_from_csr_grad_f64 over all sources; result may be NULL. */
int sumpy_p2p_direct_grad_f64(
    int64_t ntargets, const double *targets, int64_t target_stride,
    int64_t nsources, const double *sources, int64_t source_stride,
    const double *strength, const int32_t *target_to_source, double scale,
    double *result, double *grad, void *stream);

/* Interaction matrix entries. Replace P2PMatrixGenerator.__call__
 * (sumpy/p2p.py:290-349): result[t * nsources + s] = scale * G(t - s), and
 * P2PMatrixSubsetGenerator.__call__ (sumpy/p2p.py:354-477): result[m] =
 * scale * G(targets[tgtindices[m]] - sources[srcindices[m]]); G = 1/r
 * (Laplace) or e^{ikr}/r (Helmholtz, complex result as interleaved (re, im)
 * pairs); result 16-byte aligned. With target_to_source (may be NULL) the entries
 * with source == target_to_source[target] are 0 (exclude_self). FP64. */
int sumpy_p2p_matrix_f64(
    int64_t ntargets, const double *targets, int64_t target_stride,
    int64_t nsources, const double *sources, int64_t source_stride,
    const int32_t *target_to_source, double scale, double *result, void *stream);

int sumpy_helmholtz_p2p_matrix_f64(
    int64_t ntargets, const double *targets, int64_t target_stride,
    int64_t nsources, const double *sources, int64_t source_stride,
    const int32_t *target_to_source, double k, double scale, double *result, void *stream);

int sumpy_p2p_matrix_subset_f64(
    int64_t nresult, const int32_t *tgtindices, const int32_t *srcindices,
    const double *targets, int64_t target_stride, const double *sources,
    int64_t source_stride, const int32_t *target_to_source, double scale, double *result,
    void *stream);

int sumpy_helmholtz_p2p_matrix_subset_f64(
    int64_t nresult, const int32_t *tgtindices, const int32_t *srcindices,
    const double *targets, int64_t target_stride, const double *sources,
    int64_t source_stride, const int32_t *target_to_source, double k, double scale,
    double *result, void *stream);

/* ------------------------------------------------------------------ */
/* P2E                                                                  */
/* ------------------------------------------------------------------ */

/* P2M for the leaf boxes of one level. Replaces P2EFromSingleBox
 * (sumpy/p2e.py:155-261) as called by form_multipoles (sumpy/fmm.py:609-641);
 * math of VolumeTaylorMultipoleExpansionBase.coefficients_from_source_vec
 * (sumpy/expansion/multipole.py:77-114). Expansions of the listed boxes are
 * assigned. */
int sumpy_p2e_from_single_box_f64(
    int order, double rscale, int32_t nsrc_boxes, const int32_t *source_boxes,
    const double *centers, int64_t center_stride,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength,
    int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* P2L from List-4 sources for the boxes of one level. Replaces P2EFromCSR
 * (sumpy/p2e.py:268-388) as called by form_locals (sumpy/fmm.py:963-1002);
 * math of VolumeTaylorLocalExpansionBase.coefficients_from_source_vec
 * (sumpy/expansion/local.py:225-271) with LaplaceDerivativeTaker
 * (sumpy/derivative_taker.py:195-262). Expansions are assigned. */
int sumpy_p2e_from_csr_f64(
    int order, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const double *centers, int64_t center_stride,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength,
    int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* ------------------------------------------------------------------ */
/* E2E                                                                  */
/* ------------------------------------------------------------------ */

/* M2M for the parent boxes of one level. Replaces E2EFromChildren
 * (sumpy/e2e.py:866-978) as called by coarsen_multipoles (sumpy/fmm.py:643-695);
 * math of VolumeTaylorMultipoleExpansionBase.translate_from
 * (sumpy/expansion/multipole.py:159-407): the stored child coefficients,
 * scaled by (r_src/r_tgt)^|mi|, are shifted one axis at a time by
 * d = parent center - child center and compressed back to the stored set.
 * tgt += sum over nonzero box_child_ids[c*child_stride + parent]. */
int sumpy_e2e_from_children_f64(
    int src_order, int tgt_order, double src_rscale, double tgt_rscale,
    int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *box_child_ids, int64_t child_stride,
    const double *centers, int64_t center_stride,
    int32_t src_base_ibox, const double *src_expansions,
    int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* L2L into the boxes of one level. Replaces E2EFromParent
 * (sumpy/e2e.py:985-1083) as called by refine_locals (sumpy/fmm.py:1004-1045);
 * math of VolumeTaylorLocalExpansionBase.translate_from
 * (sumpy/expansion/local.py:311-493): full derivatives from the stored
 * parent coefficients, truncated Taylor shift by d = child center - parent
 * center one axis at a time, times (r_tgt/r_src)^|mi|. tgt += result. */
int sumpy_e2e_from_parent_f64(
    int src_order, int tgt_order, double src_rscale, double tgt_rscale,
    int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *box_parent_ids,
    const double *centers, int64_t center_stride,
    int32_t src_base_ibox, const double *src_expansions,
    int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* M2L applied per translation class as dense FP64 GEMMs, any number of
 * levels in one launch. Replaces M2LUsingTranslationClassesDependentData
 * (sumpy/e2e.py:310-558) with its pre/post-processing and FFTs
 * (sumpy/fmm.py:798-920): in exact arithmetic L[t] = (r_tgt/r_src)^|t|
 * sum_s M[s] D_c[s+t] (sumpy/expansion/m2l.py:363-389, 461-537, 679-698),
 * here with class_matrices[c][t][s] = that operator (row = target
 * coefficient), nclasses of them.
 *
 * The List-2 CSR (from_sep_siblings_starts/lists with the per-entry
 * translation class) is supplied regrouped into a schedule: tiles of
 * tile_width (= 64) target slots, tile_targets[tile*64 + slot] (box
 * numbers, -1 = empty), one scale per tile (tile_scale, the level's
 * operator factor); class groups g with class group_class[g] and one source
 * box per slot group_sources[g*64 + slot] (-1 = none); work items i = groups
 * [item_group_begin[i], item_group_end[i]) of tile item_tile[i]. Source box
 * b's expansion is row b - src_base_ibox of src_expansions, target box t's
 * row t - tgt_base_ibox of tgt_expansions.
 * tgt[t] += tile_scale * sum_groups T_c * src[s], with FP64 atomics. */
int sumpy_m2l_translation_classes_f64(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const double *class_matrices, int32_t src_base_ibox,
    const double *src_expansions, int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* M2L pre-processing for the tensor-core form: split FP64 values into two
 * TF32-representable FP32 planes, x ~ hi + lo (hi = tf32(x), lo =
 * tf32(x - hi), round to nearest), zero-padded from [nmat][rows][cols] to
 * [nmat][rows_pad][cols_pad]. Plays the role of sumpy's
 * M2LPreprocessMultipole (sumpy/e2e.py:676-760), which recasts multipoles
 * into the form the translation consumes; also used once per order on the
 * class operators. */
int sumpy_split_tf32x2(
    int64_t nmat, int32_t rows, int32_t cols, const double *in,
    int32_t rows_pad, int32_t cols_pad, float *hi, float *lo, void *stream);

/* M2L on the tcgen05 tensor cores, split-FP32 (3xTF32), for any number of
 * levels in one launch. Replaces M2LUsingTranslationClassesDependentData
 * (sumpy/e2e.py:310-558) with its pre/post-processing and FFTs
 * (sumpy/fmm.py:798-920); same operator as sumpy_m2l_translation_classes_f64.
 *
 * Schedule: tiles of 128 target slots (tile_targets[tile*128 + slot], box
 * numbers, -1 = empty) with a per-tile scale tile_scale[tile] (the level's
 * operator factor); class groups g with class group_class[g] and one
 * source box per slot group_sources[g*128 + slot] (-1 = none); work items
 * i = groups [item_group_begin[i], item_group_end[i]) of tile item_tile[i].
 * Operators: TF32 planes mats_hi/mats_lo [nclasses][rows_pad][k_pad];
 * multipoles: TF32 planes src_hi/src_lo [src_nrows][k_pad] (both from
 * sumpy_split_tf32x2), row of box b = b - src_base_ibox, and the last row
 * (src_nrows - 1) must be all zeros (it stands in for empty slots).
 * rows_pad is a multiple of 128, k_pad a multiple of 32.
 * Each group's products hi*hi + hi*lo + lo*hi accumulate in FP32 tensor
 * memory and are summed over groups in FP64; tgt[t] += tile_scale * result
 * with FP64 atomics, so items of one tile may run concurrently. status
 * (device int32, may be NULL) receives a nonzero code if a bounded internal
 * wait expired. */
int sumpy_m2l_translation_classes_tf32x3(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const float *mats_hi, const float *mats_lo, int32_t rows_pad,
    int32_t k_pad, int32_t src_nrows, int32_t src_base_ibox, const float *src_hi,
    const float *src_lo, int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status,
    void *stream);

/* The grouped class GEMMs above for any row count n (real values per
 * expansion: ncoeff, or 2 ncoeff for the real embedding of complex data)
 * with K split over k_split CTAs per work item (partial products meet in
 * the FP64 atomic epilogue). Used for the per-level M2M / L2L octant maps
 * (E2EFromChildren / E2EFromParent, sumpy/fmm.py:576-598, 692-712), whose
 * small coarse levels would otherwise leave most SMs idle on the
 * level-serial chain. k_split in [1, ceil(n / 8)] (FP64) or
 * [1, k_pad / 32] (tf32x3); other arguments as for the entries above. */
int sumpy_class_gemm_f64(
    int32_t n, int32_t k_split, int32_t nitems, const int32_t *item_tile,
    const int32_t *item_group_begin, const int32_t *item_group_end, int32_t tile_width,
    const int32_t *tile_targets, const double *tile_scale, const int32_t *group_class,
    const int32_t *group_sources, int32_t nclasses, const double *class_matrices,
    int32_t src_base_ibox, const double *src_expansions, int32_t tgt_base_ibox,
    double *tgt_expansions, void *stream);

int sumpy_class_gemm_tf32x3(
    int32_t n, int32_t k_split, int32_t nitems, const int32_t *item_tile,
    const int32_t *item_group_begin, const int32_t *item_group_end, int32_t tile_width,
    const int32_t *tile_targets, const double *tile_scale, const int32_t *group_class,
    const int32_t *group_sources, int32_t nclasses, const float *mats_hi, const float *mats_lo,
    int32_t rows_pad, int32_t k_pad, int32_t src_nrows, int32_t src_base_ibox,
    const float *src_hi, const float *src_lo, int32_t tgt_base_ibox, double *tgt_expansions,
    int32_t *status, void *stream);

/* The tensor-core M2L and class GEMMs with f16 operands (default of the
 * mixed form): each FP64 operand row -- a class-operator row, or one source
 * box's expansion -- is scaled by a power of two 2^e that brings its largest
 * magnitude into [2^13, 2^14) and split as hi = f16(x 2^e), lo = f16(x 2^e -
 * hi) (sumpy_split_f16x2_rowscale, which also writes row_inv = 2^-e; zero
 * and padding rows: hi = lo = 0, row_inv = 1). The MMAs (kind::f16, FP32
 * accumulation) form hi*hi + hi*lo + lo*hi per class group, as the tf32x3
 * form does with TF32 halves: the same ~22 bits per operand, at twice the
 * tensor rate and with half the operand bytes. The epilogue multiplies each
 * group's FP32 result by src_rinv[source row], then by mats_rinv[class][row]
 * (two FP32 products by powers of two, exact while the contribution lies in
 * the FP32 normal range, as the mixed form's FP32 near field requires) and
 * adds it to the FP64 sums; no operand row leaves the f16 range whatever its
 * magnitude. Planes are f16 [..][k_pad] with k_pad a
 * multiple of 64 (one 128-byte row per pipeline stage); k_split in
 * [1, k_pad / 64]; mats_rinv [nclasses][rows_pad], src_rinv [src_nrows]
 * (float). The last source row (src_nrows - 1) is all zeros. Other
 * arguments as for the tf32x3 entries. */
int sumpy_split_f16x2_rowscale(
    int64_t nmat, int32_t rows, int32_t cols, const double *in,
    int32_t rows_pad, int32_t cols_pad, void *hi, void *lo, float *row_inv, void *stream);

int sumpy_m2l_translation_classes_f16x3(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const void *mats_hi, const void *mats_lo, const float *mats_rinv,
    int32_t rows_pad, int32_t k_pad, int32_t src_nrows, int32_t src_base_ibox,
    const void *src_hi, const void *src_lo, const float *src_rinv, int32_t tgt_base_ibox,
    double *tgt_expansions, int32_t *status, void *stream);

int sumpy_class_gemm_f16x3(
    int32_t n, int32_t k_split, int32_t nitems, const int32_t *item_tile,
    const int32_t *item_group_begin, const int32_t *item_group_end, int32_t tile_width,
    const int32_t *tile_targets, const double *tile_scale, const int32_t *group_class,
    const int32_t *group_sources, int32_t nclasses, const void *mats_hi, const void *mats_lo,
    const float *mats_rinv, int32_t rows_pad, int32_t k_pad, int32_t src_nrows,
    int32_t src_base_ibox, const void *src_hi, const void *src_lo, const float *src_rinv,
    int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status, void *stream);

/* Budget, in SM clock cycles (clock64), of every barrier wait in the
 * tensor-core kernels (the M2L above, the class GEMMs and the Helmholtz
 * M2L), read at each launch. A wait that runs out sets the abort flag of its
 * CTA; the CTA lets the work it has in flight finish, frees its tensor
 * memory, writes 1 (timeout) to the launch's status word and returns, so
 * the context stays usable. cycles <= 0 restores the default (4e9, about
 * two seconds). Budgets below 1e6 cycles poll the barriers without letting
 * the hardware suspend the waiting thread. No counterpart in sumpy (its
 * kernels have no waits); it exists so that tests and callers with a
 * deadline can bound a launch. Also bounds the level waits of
 * sumpy_class_gemm_chain_f64. Process-wide; returns SUMPY_OK. */
int sumpy_set_tc_wait_cycles(int64_t cycles);
int64_t sumpy_get_tc_wait_cycles(void);

/* The FP64 class GEMMs of several tree levels chained in one persistent
 * launch: M2M (E2EFromChildren, sumpy/e2e.py:866-978, driven level by level
 * by coarsen_multipoles, sumpy/fmm.py:643-695) or L2L (E2EFromParent,
 * sumpy/e2e.py:985-1083, driven by refine_locals, sumpy/fmm.py:1004-1045) as
 * octant class GEMMs, where each level's sources are the previous level's
 * targets. Step L of the chain owns work units [step_unit_start[L],
 * step_unit_start[L + 1]) -- unit u = (item, row block, k part) with items
 * from step_item_start[L] and step_ksplit[L] K parts (DEVICE int32 arrays) --
 * and the item arrays are those of sumpy_class_gemm_f64 with tile_width 64,
 * concatenated over the steps; expansions of all levels are rows (box ids)
 * of one flat [nboxes][n] array, accumulated in place. A device counter
 * hands out units in order; a unit of step L starts when all of step L - 1
 * have finished (queue: DEVICE int32 [1 + nsteps], cleared by this call).
 * Each wait is bounded by the budget of sumpy_set_tc_wait_cycles; one that
 * runs out writes 2 to *status and stops its CTA. total_units (host) sizes
 * the grid; nsteps <= 64. */
int sumpy_class_gemm_chain_f64(
    int32_t n, int32_t nsteps, const int32_t *step_unit_start, const int32_t *step_item_start,
    const int32_t *step_ksplit, int32_t total_units, const int32_t *item_tile,
    const int32_t *item_group_begin, const int32_t *item_group_end, int32_t tile_width,
    const int32_t *tile_targets, const double *tile_scale, const int32_t *group_class,
    const int32_t *group_sources, const double *class_matrices, double *expansions,
    int32_t *queue, int32_t *status, void *stream);

/* Same M2L as sumpy_m2l_translation_classes_tf32x3, for callers that cannot
 * allocate device memory while they run (a host application with a fixed
 * device-memory budget, an allocation-free real-time loop, code where an
 * allocation would synchronise the device). No counterpart in sumpy: it
 * exists only for this interface. Takes the level's FP64 multipoles
 * (src_expansions, nsrc_boxes rows of ncoeff, box b at row b - src_base_ibox)
 * and keeps their TF32 planes in a device array built into the library
 * (8 MiB per GPU, held until exit) instead of caller memory; allocates
 * nothing. Limit: (nsrc_boxes + 1) * k_pad <= 1,048,576 and k_pad <= 128
 * (8,191 boxes at order <= 10); larger requests return SUMPY_EINVAL. Each
 * call looks up the array's device address in the current context. With
 * CUDA's default lazy module loading, the first call into the tensor-core
 * M2L on a device (this entry point or the regular one) loads the module
 * and with it reserves the 8 MiB: make one such call while initialising (or
 * set CUDA_MODULE_LOADING=EAGER), and before any stream capture. All calls
 * share the array and it keeps the last call's contents (the zero row the
 * kernel reads is cleared on every call): calls that overlap on the GPU
 * race and must be serialised by the caller. */
int sumpy_m2l_translation_classes_tf32x3_noalloc(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const float *mats_hi, const float *mats_lo, int32_t rows_pad,
    int32_t k_pad, int32_t nsrc_boxes, int32_t src_base_ibox, const double *src_expansions,
    int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status, void *stream);

/* ------------------------------------------------------------------ */
/* E2P                                                                  */
/* ------------------------------------------------------------------ */

/* L2P for the leaf target boxes of one level. Replaces E2PFromSingleBox
 * (sumpy/e2p.py:123-226) as called by eval_locals (sumpy/fmm.py:1047-1083);
 * math of VolumeTaylorLocalExpansionBase.evaluate (sumpy/expansion/local.py:
 * 284-309). result[t] = scale * value (assigned). */
int sumpy_e2p_from_single_box_f64(
    int order, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
    const double *centers, int64_t center_stride,
    int32_t src_base_ibox, const double *src_expansions,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *targets, int64_t target_stride, double scale, double *result,
    void *stream);

/* M2P from List-3 boxes of one source level. Replaces E2PFromCSR
 * (sumpy/e2p.py:233-343) as called by eval_multipoles (sumpy/fmm.py:922-961);
 * math of VolumeTaylorMultipoleExpansionBase.evaluate
 * (sumpy/expansion/multipole.py:131-157). result[t] += scale * value. */
int sumpy_e2p_from_csr_f64(
    int order, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const double *centers, int64_t center_stride,
    int32_t src_base_ibox, const double *src_expansions,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *targets, int64_t target_stride, double scale, double *result,
    void *stream);

/* Gradient forms of L2P and M2P: grad[d*target_stride + t] receives the
 * derivative of the expansion's value with respect to target coordinate d
 * (assigned for L2P, accumulated for M2P, like the values); result may be
 * NULL. L2P: (1/rscale) times the local polynomial with coefficients
 * shifted by e_d; M2P: kernel derivatives of one order more. */
int sumpy_e2p_from_single_box_grad_f64(
    int order, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
    const double *centers, int64_t center_stride,
    int32_t src_base_ibox, const double *src_expansions,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *targets, int64_t target_stride, double scale, double *result,
    double *grad, void *stream);

int sumpy_e2p_from_csr_grad_f64(
    int order, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const double *centers, int64_t center_stride,
    int32_t src_base_ibox, const double *src_expansions,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *targets, int64_t target_stride, double scale, double *result,
    double *grad, void *stream);

/* Mixed-precision E2PFromCSR (List 3) and P2EFromCSR (List 4) for the mixed
 * form: FP64 offsets rounded to FP32, derivative recurrence and products in
 * FP32 per source box / source, FP64 sums. Arguments as the _f64 entries. */
int sumpy_e2p_from_csr_mixed(
    int order, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const double *centers, int64_t center_stride,
    int32_t src_base_ibox, const double *src_expansions,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *targets, int64_t target_stride, double scale, double *result,
    void *stream);

int sumpy_p2e_from_csr_mixed(
    int order, double rscale, int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists,
    const double *centers, int64_t center_stride,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength,
    int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* The mixed List-3 and List-4 stages of all levels in one launch each, over
 * work items cut by the host (the per-level E2PFromCSR / P2EFromCSR calls of
 * sumpy/fmm.py:600-690 merged; same arithmetic as the _mixed entries above).
 * All levels share one order; expansions are the flat [nboxes][(order+1)^2]
 * arrays (box-major over all levels, as with a level-independent order).
 *
 * sumpy_mpoles_to_f32: dst[b][s] = (float) src[b][s] for s < (order+1)^2,
 *   0 up to the row stride npad = ((order+1)^2 + 3) & ~3.
 * sumpy_e2p_from_items_mixed: items int32 [nitems][4] (16-byte aligned) =
 *   {first target, first index into source_box_lists, number of List-3
 *   boxes, ntargets (1..32) | source level << 8}; the item's targets are
 *   consecutive; level_rscales[level] is that level's rscale;
 *   src_expansions_f32 from sumpy_mpoles_to_f32 (16-byte aligned). Adds
 *   scale * potential into result with atomics.
 * sumpy_p2e_from_items_mixed: items {target box, first index into
 *   source_index, number of sources, target level}; source_index lists the
 *   sources of each target box's List-4 boxes. Adds into tgt_expansions
 *   ([nboxes][(order+1)^2]) with atomics. */
/* P2EFromSingleBox (P2M) and E2PFromSingleBox (L2P) of all levels in one
 * launch each (sumpy/fmm.py:540-563 and 729-760 loop over levels), FP64,
 * flat [nboxes][(order+1)^2] expansions as above.
 * sumpy_p2e_from_single_box_levels_f64: box_levels[i] is the level of
 *   source_boxes[i] (its rscale = level_rscales[level]); any box order (the
 *   host lists the largest first). Assigns the boxes' multipoles.
 * sumpy_e2p_from_single_box_packed_f64: items int32 [nitems][2] (8-byte
 *   aligned) = {first slot, number of slots (1..4)}; slots int32 [][4]
 *   (16-byte aligned) = {box, first target, number of targets, level}, at
 *   most 32 targets per item, a box's targets in one or more slots. An item
 *   of more than 4 slots (more than the warp's shared memory holds) is
 *   skipped. Assigns scale * potential to each listed target. */
int sumpy_p2e_from_single_box_levels_f64(
    int order, int32_t nsrc_boxes, const int32_t *source_boxes, const int32_t *box_levels,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength,
    double *expansions, void *stream);

int sumpy_e2p_from_single_box_packed_f64(
    int order, int32_t nitems, const int32_t *items, const int32_t *slots,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const double *src_expansions, const double *targets, int64_t target_stride,
    double scale, double *result, void *stream);

/* The same with the potential's target gradient (E2PFromSingleBox with
 * gradient outputs): grad is [3][target_stride], assigned like result;
 * result may be NULL. */
int sumpy_e2p_from_single_box_packed_grad_f64(
    int order, int32_t nitems, const int32_t *items, const int32_t *slots,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const double *src_expansions, const double *targets, int64_t target_stride,
    double scale, double *result, double *grad, void *stream);

int sumpy_mpoles_to_f32(int order, int64_t nboxes, const double *src_expansions, float *dst,
                        void *stream);

int sumpy_e2p_from_items_mixed(
    int order, int32_t nitems, const int32_t *items, const double *level_rscales,
    const int32_t *source_box_lists, const double *centers, int64_t center_stride,
    const float *src_expansions_f32, const double *targets, int64_t target_stride,
    double scale, double *result, void *stream);

/* The same with the potential's target gradient added into grad
 * ([3][target_stride]); result may be NULL. */
int sumpy_e2p_from_items_grad_mixed(
    int order, int32_t nitems, const int32_t *items, const double *level_rscales,
    const int32_t *source_box_lists, const double *centers, int64_t center_stride,
    const float *src_expansions_f32, const double *targets, int64_t target_stride,
    double scale, double *result, double *grad, void *stream);

int sumpy_p2e_from_items_mixed(
    int order, int32_t nitems, const int32_t *items, const double *level_rscales,
    const int32_t *source_index, const double *centers, int64_t center_stride,
    const double *sources, int64_t source_stride, const double *strength,
    double *tgt_expansions, void *stream);

/* The same item schedules in FP64 throughout (replacing the per-level
 * sumpy_e2p_from_csr_f64 / sumpy_p2e_from_csr_f64 loops of
 * sumpy/fmm.py:645-711 for a uniform-order FMM): src_expansions are the
 * FP64 multipoles [nboxes][(order+1)^2] (no FP32 copy, no alignment rule);
 * items as above (16-byte aligned), M2P items built with one-lane groups
 * (a chunk of ntc targets takes next_pow2(ntc) lanes). The grad form adds
 * the target gradient into grad ([3][target_stride]); result may be NULL. */
int sumpy_e2p_from_items_f64(
    int order, int32_t nitems, const int32_t *items, const double *level_rscales,
    const int32_t *source_box_lists, const double *centers, int64_t center_stride,
    const double *src_expansions, const double *targets, int64_t target_stride,
    double scale, double *result, void *stream);

int sumpy_e2p_from_items_grad_f64(
    int order, int32_t nitems, const int32_t *items, const double *level_rscales,
    const int32_t *source_box_lists, const double *centers, int64_t center_stride,
    const double *src_expansions, const double *targets, int64_t target_stride,
    double scale, double *result, double *grad, void *stream);

int sumpy_p2e_from_items_f64(
    int order, int32_t nitems, const int32_t *items, const double *level_rscales,
    const int32_t *source_index, const double *centers, int64_t center_stride,
    const double *sources, int64_t source_stride, const double *strength,
    double *tgt_expansions, void *stream);

/* ------------------------------------------------------------------------
 * 3D Helmholtz kernel G = exp(i k r) / r (sumpy/kernel.py:755-844), the same
 * loopy kernels as above instantiated for HelmholtzKernel(3): complex data
 * (strengths, expansions, results) as interleaved (re, im) float64 pairs,
 * i.e. complex128 arrays; coordinates real. k is the (real) wave number
 * sumpy passes as the kernel argument "k". Expansions use the Helmholtz PDE
 * projection u_mi = -u_{mi-2e0+2e1} - u_{mi-2e0+2e2} - k^2 rscale^2 u_{mi-2e0}.
 * Arguments otherwise as for the Laplace entry points above.
 * ------------------------------------------------------------------------ */

/* P2PFromCSR (sumpy/p2p.py:484-833) */
int sumpy_helmholtz_p2p_from_csr_f64(
    int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *source_box_starts,
    const int32_t *source_box_lists, const int32_t *box_source_starts,
    const int32_t *box_source_counts_nonchild, const int32_t *box_target_starts,
    const int32_t *box_target_counts_nonchild, const double *sources, int64_t source_stride,
    double k, const double *strength, const double *targets, int64_t target_stride,
    const int32_t *target_to_source, double scale, double *result, void *stream);

/* Same with complex64 arithmetic on FP64 coordinate differences, FP64 sums
 * per source box. */
int sumpy_helmholtz_p2p_from_csr_mixed(
    int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *source_box_starts,
    const int32_t *source_box_lists, const int32_t *box_source_starts,
    const int32_t *box_source_counts_nonchild, const int32_t *box_target_starts,
    const int32_t *box_target_counts_nonchild, const double *sources, int64_t source_stride,
    double k, const double *strength, const double *targets, int64_t target_stride,
    const int32_t *target_to_source, double scale, double *result, void *stream);

/* P2P (sumpy/p2p.py:215-285), all pairs */
int sumpy_helmholtz_p2p_direct_f64(
    int64_t ntargets, const double *targets, int64_t target_stride, int64_t nsources,
    const double *sources, int64_t source_stride, double k, const double *strength,
    const int32_t *target_to_source, double scale, double *result, void *stream);

/* P2EFromSingleBox (sumpy/p2e.py:155-261) */
int sumpy_helmholtz_p2e_from_single_box_f64(
    int order, double rscale, double k, int32_t nsrc_boxes, const int32_t *source_boxes,
    const double *centers, int64_t center_stride, const int32_t *box_source_starts,
    const int32_t *box_source_counts_nonchild, const double *sources, int64_t source_stride,
    const double *strength, int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* E2EFromChildren (sumpy/e2e.py:866-978) */
int sumpy_helmholtz_e2e_from_children_f64(
    int src_order, int tgt_order, double src_rscale, double tgt_rscale, double k,
    int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *box_child_ids,
    int64_t child_stride, const double *centers, int64_t center_stride, int32_t src_base_ibox,
    const double *src_expansions, int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* E2EFromParent (sumpy/e2e.py:985-1083) */
int sumpy_helmholtz_e2e_from_parent_f64(
    int src_order, int tgt_order, double src_rscale, double tgt_rscale, double k,
    int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *box_parent_ids,
    const double *centers, int64_t center_stride, int32_t src_base_ibox,
    const double *src_expansions, int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* M2L per translation class (sumpy/e2e.py:310-859) on complex expansions:
 * class_matrices are the real embeddings [nclasses][2n][2n] (n = (order+1)^2)
 * of the complex operators, blocks [[Re, -Im], [Im, Re]]; otherwise as
 * sumpy_m2l_translation_classes_f64 with 2n real values per box. */
int sumpy_helmholtz_m2l_translation_classes_f64(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const double *class_matrices, int32_t src_base_ibox,
    const double *src_expansions, int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* Same on the tensor cores (split TF32 planes of the real embeddings, rows
 * and k padded for 2n; see sumpy_m2l_translation_classes_tf32x3). */
int sumpy_helmholtz_m2l_translation_classes_tf32x3(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const float *mats_hi, const float *mats_lo, int32_t rows_pad, int32_t k_pad,
    int32_t src_nrows, int32_t src_base_ibox, const float *src_hi, const float *src_lo,
    int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status, void *stream);

/* Same with f16 operand planes (see sumpy_m2l_translation_classes_f16x3). */
int sumpy_helmholtz_m2l_translation_classes_f16x3(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const void *mats_hi, const void *mats_lo, const float *mats_rinv,
    int32_t rows_pad, int32_t k_pad, int32_t src_nrows, int32_t src_base_ibox,
    const void *src_hi, const void *src_lo, const float *src_rinv, int32_t tgt_base_ibox,
    double *tgt_expansions, int32_t *status, void *stream);

/* E2PFromSingleBox (sumpy/e2p.py:123-226): result assigned */
int sumpy_helmholtz_e2p_from_single_box_f64(
    int order, double rscale, double k, int32_t ntgt_boxes, const int32_t *target_boxes,
    const double *centers, int64_t center_stride, int32_t src_base_ibox,
    const double *src_expansions, const int32_t *box_target_starts,
    const int32_t *box_target_counts_nonchild, const double *targets, int64_t target_stride,
    double scale, double *result, void *stream);

/* E2PFromCSR (sumpy/e2p.py:233-343): result accumulated */
int sumpy_helmholtz_e2p_from_csr_f64(
    int order, double rscale, double k, int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists, const double *centers,
    int64_t center_stride, int32_t src_base_ibox, const double *src_expansions,
    const int32_t *box_target_starts, const int32_t *box_target_counts_nonchild,
    const double *targets, int64_t target_stride, double scale, double *result, void *stream);

/* P2EFromCSR (sumpy/p2e.py:268-388): expansions accumulated */
int sumpy_helmholtz_p2e_from_csr_f64(
    int order, double rscale, double k, int32_t ntgt_boxes, const int32_t *target_boxes,
    const int32_t *source_box_starts, const int32_t *source_box_lists, const double *centers,
    int64_t center_stride, const int32_t *box_source_starts,
    const int32_t *box_source_counts_nonchild, const double *sources, int64_t source_stride,
    const double *strength, int32_t tgt_base_ibox, double *tgt_expansions, void *stream);

/* All levels in one launch (one order on every level, flat complex
 * [nboxes][(order+1)^2] expansions; levels and items as for the Laplace
 * _levels / _items entries above, FP64 arithmetic):
 * P2EFromSingleBox and E2PFromSingleBox with per-box levels, E2PFromCSR
 * (List 3) and P2EFromCSR (List 4) over host-cut work items. The List-3
 * items' targets take next_pow2(ntargets) lanes (lane groups of one lane
 * and more); results and locals are added with atomics. */
int sumpy_helmholtz_p2e_from_single_box_levels_f64(
    int order, double k, int32_t nsrc_boxes, const int32_t *source_boxes, const int32_t *box_levels,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const int32_t *box_source_starts, const int32_t *box_source_counts_nonchild,
    const double *sources, int64_t source_stride, const double *strength, double *expansions,
    void *stream);

int sumpy_helmholtz_e2p_from_single_box_levels_f64(
    int order, double k, int32_t ntgt_boxes, const int32_t *target_boxes, const int32_t *box_levels,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const double *src_expansions, const int32_t *box_target_starts,
    const int32_t *box_target_counts_nonchild, const double *targets, int64_t target_stride,
    double scale, double *result, void *stream);

/* Helmholtz E2PFromSingleBox of all levels over packed items as
 * sumpy_e2p_from_single_box_packed_f64 (items of at most 4 slots); the
 * locals are decompressed with kappa = k^2 rscale^2 of each box's level. */
int sumpy_helmholtz_e2p_from_single_box_packed_f64(
    int order, double k, int32_t nitems, const int32_t *items, const int32_t *slots,
    const double *level_rscales, const double *centers, int64_t center_stride,
    const double *src_expansions, const double *targets, int64_t target_stride, double scale,
    double *result, void *stream);

int sumpy_helmholtz_e2p_from_items_f64(
    int order, double k, int32_t nitems, const int32_t *items, const double *level_rscales,
    const int32_t *source_box_lists, const double *centers, int64_t center_stride,
    const double *src_expansions, const double *targets, int64_t target_stride, double scale,
    double *result, void *stream);

int sumpy_helmholtz_p2e_from_items_f64(
    int order, double k, int32_t nitems, const int32_t *items, const double *level_rscales,
    const int32_t *source_index, const double *centers, int64_t center_stride,
    const double *sources, int64_t source_stride, const double *strength,
    double *tgt_expansions, void *stream);

/* ------------------------------------------------------------------ */
/* Tree, interaction lists and translation classes on the GPU           */
/* ------------------------------------------------------------------ */

/* Build the octree, Lists 1-4 and the translation classes of one problem or
 * of a forest of independent problems on the GPU. Replaces boxtree's
 * TreeBuilder / FMMTraversalBuilder / TranslationClassesBuilder as sumpy
 * calls them (sumpy/fmm.py:356-363; the fields consumed are listed at
 * sumpy/fmm.py:372-397, 543-592). Same definitions and the same arrays, bit
 * for bit, as the host builder sumpy_tree_build_in_box (sumpy_b200_tree.h),
 * for a forest as sumpy_b200.forest.merge_trees of per-problem trees built in
 * one root box.
 *
 * Coordinates are DEVICE arrays in user order (problems concatenated);
 * ntargets < 0 or tx == NULL: sources are the targets. nproblems > 1:
 * problem p owns sources [problem_source_starts[p], [p+1]) and targets
 * [problem_target_starts[p], [p+1]) (HOST int64 arrays of nproblems + 1
 * entries, from 0 to the counts); nproblems == 1 ignores them. bbox_min
 * (HOST, 3 doubles) and root_extent fix the root box (every particle must lie
 * in it); bbox_min == NULL: the particles' bounding cube. Work runs on
 * `stream`; the call returns when the build is complete. Allocates device
 * memory (stream-ordered) for its scratch and results: a set-up step, not the
 * evaluation path. The handle owns the result arrays (boxtree's names; plus
 * "box_problem", the problem of each box, and "build_phase_ms", the wall time
 * of the build's phases: bounding box, keys and sort, levels, boxes and
 * colleagues, Lists 1-4, List 3 by level, particles and classes) until
 * sumpy_tree_gpu_free. */
int sumpy_tree_gpu_build(int64_t nsources, const double *sx, const double *sy, const double *sz,
                         int64_t ntargets, const double *tx, const double *ty, const double *tz,
                         int32_t nproblems, const int64_t *problem_source_starts,
                         const int64_t *problem_target_starts, int max_particles_in_box,
                         int max_levels, const double *bbox_min, double root_extent,
                         void *stream, void **handle_out);

/* kind: 0 = int32, 1 = float64; length in elements. */
int sumpy_tree_gpu_array_info(void *handle, const char *name, int *kind, int64_t *length);

/* Copy a result array to dst (device memory when dst_on_device, else host
 * memory; a host copy is complete when the call returns). */
int sumpy_tree_gpu_array_copy(void *handle, const char *name, void *dst, int64_t capacity_bytes,
                              int dst_on_device, void *stream);

void sumpy_tree_gpu_free(void *handle);

/* ---- QBX layer potentials (3D Laplace / Helmholtz, FP64) ----
 *
 * Replace the loopy kernels of sumpy.qbx.LayerPotential (sumpy/qbx.py:250-340),
 * LayerPotentialMatrixGenerator (qbx.py:345-420) and
 * LayerPotentialMatrixSubsetGenerator (qbx.py:425-520) for one (target kernel,
 * source kernel) pair. With a = center - source and b = target - center
 * (qbx.py:283-284), each pair contributes the order-`order` local Taylor
 * expansion about the target's center of the source's kernel, evaluated at the
 * target, times `scale` (the kernel's global scaling constant, 1/(4 pi)).
 * Line Taylor and volume Taylor expansions (plain or PDE-compressed) give the
 * same values; they differ only for target derivatives (modes 1 and 2).
 *
 * mode 0: value; 1: target derivative d/da_axis of each line-Taylor
 * coefficient (qbx.py:121-132); 2: target derivative d/db_axis of a volume
 * Taylor sum (sumpy/expansion/local.py evaluate with AxisTargetDerivative);
 * 3: source derivative -d/da_axis (AxisSourceDerivative); 4: directional
 * source derivative -dir(s) . grad_a (DirectionalSourceDerivative, the
 * double layer), with source_dirs[d * dir_stride + s]. order in [0, 32].
 *
 * Points are DEVICE arrays laid out as x[d * stride + i] (sumpy's (3, n)
 * C-order arrays, stride = n). Helmholtz strengths and results are complex
 * (interleaved re, im); k is the real wave number. expansion_radii are not
 * needed: they only set the expansion's rscale, which cancels. No allocation;
 * the call launches one kernel on `stream` and returns. */
int sumpy_qbx_lpot_laplace_f64(int order, int mode, int axis, int64_t ntargets,
                               const double *targets, int64_t target_stride,
                               const double *centers, int64_t center_stride, int64_t nsources,
                               const double *sources, int64_t source_stride,
                               const double *source_dirs, int64_t dir_stride,
                               const double *strength, double scale, double *result,
                               void *stream);
int sumpy_qbx_lpot_helmholtz_f64(int order, int mode, int axis, double k, int64_t ntargets,
                                 const double *targets, int64_t target_stride,
                                 const double *centers, int64_t center_stride, int64_t nsources,
                                 const double *sources, int64_t source_stride,
                                 const double *source_dirs, int64_t dir_stride,
                                 const double *strength, double scale, double *result,
                                 void *stream);

/* The (ntargets, nsources) row-major matrix of pair values (unit strength). */
int sumpy_qbx_matrix_laplace_f64(int order, int mode, int axis, int64_t ntargets,
                                 const double *targets, int64_t target_stride,
                                 const double *centers, int64_t center_stride,
                                 int64_t nsources, const double *sources,
                                 int64_t source_stride, const double *source_dirs,
                                 int64_t dir_stride, double scale, double *result, void *stream);
int sumpy_qbx_matrix_helmholtz_f64(int order, int mode, int axis, double k, int64_t ntargets,
                                   const double *targets, int64_t target_stride,
                                   const double *centers, int64_t center_stride,
                                   int64_t nsources, const double *sources,
                                   int64_t source_stride, const double *source_dirs,
                                   int64_t dir_stride, double scale, double *result,
                                   void *stream);

/* Entries (tgtindices[m], srcindices[m]) of that matrix, m < nentries (DEVICE
 * int32 index arrays, in range: the caller checks). */
int sumpy_qbx_matrix_subset_laplace_f64(int order, int mode, int axis, int64_t nentries,
                                        const int32_t *tgtindices, const int32_t *srcindices,
                                        const double *targets, int64_t target_stride,
                                        const double *centers, int64_t center_stride,
                                        const double *sources, int64_t source_stride,
                                        const double *source_dirs, int64_t dir_stride,
                                        double scale, double *result, void *stream);
int sumpy_qbx_matrix_subset_helmholtz_f64(int order, int mode, int axis, double k,
                                          int64_t nentries, const int32_t *tgtindices,
                                          const int32_t *srcindices, const double *targets,
                                          int64_t target_stride, const double *centers,
                                          int64_t center_stride, const double *sources,
                                          int64_t source_stride, const double *source_dirs,
                                          int64_t dir_stride, double scale, double *result,
                                          void *stream);

#ifdef __cplusplus
}
#endif

#endif
