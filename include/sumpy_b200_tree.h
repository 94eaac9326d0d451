/*
 * sumpy_b200_tree.h -- host-side octree, interaction lists and translation
 * classes for 3D point sets.
 *
 * sumpy takes its tree, traversal and translation classes from boxtree
 * (TreeBuilder, FMMTraversalBuilder, TranslationClassesBuilder; called at
 * sumpy/fmm.py:356-363 and sumpy/test/test_fmm.py:182-189). boxtree is an
 * external dependency, not part of the sumpy sources, so this library
 * provides the same products under boxtree's array names: the arrays sumpy's
 * wrangler reads (sumpy/fmm.py:372-397, 413-418, 543-592, 752-754, 931-948).
 *
 * All arrays are host memory. The handle owns them until sumpy_tree_free.
 */
#ifndef SUMPY_B200_TREE_H
#define SUMPY_B200_TREE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SUMPY_TREE_OK = 0,
    SUMPY_TREE_EINVAL = 1,
    SUMPY_TREE_EINTERNAL = 2
};

/* Build tree + traversal + translation classes.
 * Replaces boxtree.TreeBuilder.__call__(actx, sources, targets=...,
 * max_particles_in_box=...) followed by FMMTraversalBuilder and
 * TranslationClassesBuilder(is_translation_per_level=True), as used at
 * sumpy/test/test_fmm.py:182-189 and sumpy/fmm.py:356-363.
 * Coordinates are SoA float64. Pass tx == NULL (or ntargets < 0) when the
 * targets are the sources; the tree then counts each particle once and
 * provides a target_to_source array for exclude_self.
 * Returns SUMPY_TREE_OK and an opaque handle in *handle_out. */
int sumpy_tree_build(int64_t nsources, const double *sx, const double *sy, const double *sz,
                     int64_t ntargets, const double *tx, const double *ty, const double *tz,
                     int max_particles_in_box, int max_levels, void **handle_out);

/* sumpy_tree_build with a caller-fixed root box [bbox_min, bbox_min + root_extent]^3
 * instead of the particles' bounding cube. Trees built in one box share their
 * box sizes, rscales and translation-class vectors level by level, which is
 * what lets sumpy_b200.forest merge many problems into one level-major box
 * numbering. boxtree's TreeBuilder takes the same option as its
 * bbox argument. Particles outside the box are an error (SUMPY_TREE_EINVAL);
 * a coordinate equal to the upper bound goes to the last cell. */
int sumpy_tree_build_in_box(int64_t nsources, const double *sx, const double *sy,
                            const double *sz, int64_t ntargets, const double *tx,
                            const double *ty, const double *tz, int max_particles_in_box,
                            int max_levels, const double *bbox_min, double root_extent,
                            void **handle_out);

/* Look up a named array: kind 0 = int32, 1 = float64; length in elements. */
int sumpy_tree_array_info(void *handle, const char *name, int *kind, int64_t *length);

/* Copy a named array into dst (capacity in bytes). */
int sumpy_tree_array_copy(void *handle, const char *name, void *dst, int64_t capacity_bytes);

void sumpy_tree_free(void *handle);

/* Next-fit packing of n sizes (in the given order) into items of total size
 * <= capacity and at most max_count entries each: item i holds entries
 * [item_first[i], item_first[i] + item_count[i]). The item arrays need room for
 * n entries; *nitems_out receives their number. Used to pack the partial
 * 32-target slots of the one-launch L2P (sumpy_e2p_from_single_box_packed_f64). */
int sumpy_pack_next_fit(int64_t n, const int32_t *sizes, int32_t capacity, int32_t max_count,
                        int32_t *item_first, int32_t *item_count, int64_t *nitems_out);

/* Message of the last failed call on this thread. */
const char *sumpy_tree_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
