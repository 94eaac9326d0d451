"""Adjoint (transpose) of the FMM and gradients with respect to positions.

For the symmetric Laplace kernel each transposed FMM stage is a forward
stage with the roles of sources and targets exchanged (derivation in the
comments of :func:`transpose_traversal`), so the exact transpose F^T of the
FMM operator F of a tree is the FMM run on the *transposed traversal* of the
same tree: sources and targets swapped, each interaction list transposed,
each translation class reversed. With strengths g at the targets it yields

    psi(x_s) = sum_t g_t G(x_t - x_s) / (4 pi)   at every source,

i.e. F^T g, and, with the gradient-form evaluation stages, grad psi(x_s).
For L = loss(phi), g = dL/dphi:
    dL/dq_s   = psi(x_s)
    dL/dx_s   = q_s * grad psi(x_s)
    dL/dx_t   = g_t * grad phi(x_t)   (gradient form of the forward FMM).

Stage by stage (S = diag((-1)^|mi|), which cancels in pairs):
    L2P^T = S P2M, L2L^T = S M2M S, M2L^T = S M2L S on reversed pairs
    (T_c is symmetric), P2L^T = M2P S, M2M^T = S L2L S, M2P^T = S P2L,
    P2M^T = L2P S, P2P^T = P2P on transposed List 1.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from sumpy_b200.tree import FMMTraversalInfo, FromSepSmallerCSR, TranslationClassesInfo


def _inverse_perm(p):
    inv = np.empty_like(p)
    inv[p] = np.arange(len(p), dtype=p.dtype)
    return inv


def _transpose_csr(row_boxes, starts, lists, new_row_boxes, nboxes, values=None):
    """Entries (row_box -> col_box) regrouped as (col_box -> row_box), rows
    ordered as new_row_boxes; within a row, entries keep ascending row_box."""
    starts = np.asarray(starts, dtype=np.int64)
    lists = np.asarray(lists, dtype=np.int64)
    counts = np.diff(starts)
    ent_row = np.repeat(np.asarray(row_boxes, dtype=np.int64), counts)
    ent_col = lists[starts[0]:starts[-1]]
    pos = np.full(nboxes, -1, dtype=np.int64)
    pos[np.asarray(new_row_boxes, dtype=np.int64)] = np.arange(len(new_row_boxes))
    new_row = pos[ent_col]
    if len(new_row) and new_row.min() < 0:
        raise ValueError("transposed list entry has no row in the new box set")
    order = np.lexsort((ent_row, new_row))
    new_starts = np.zeros(len(new_row_boxes) + 1, dtype=np.int64)
    np.add.at(new_starts, new_row + 1, 1)
    new_starts = np.cumsum(new_starts)
    out_lists = ent_row[order].astype(np.int32)
    out_vals = None if values is None else np.asarray(values)[starts[0]:starts[-1]][order]
    return new_starts.astype(np.int32), out_lists, out_vals, new_row[order]


def _level_starts(boxes, levels, nlevels):
    lv = levels[boxes] if len(boxes) else np.zeros(0, dtype=np.int32)
    return np.searchsorted(lv, np.arange(nlevels + 1), side="left").astype(np.int32)


def transpose_traversal(tree, trav, tcls):
    """Tree, traversal and translation classes of the transposed FMM.

    Derivation for one target/source pair of stages (a = center - source,
    b = target - center, D(x)[mi] = rscale^|mi| d^mi (1/|x|), D(-x) = S D(x)):
      * P2M^T: q_s' += sum (P Mbar)[mi] (a/r)^mi/mi! = L2P of S Mbar at the
        source (b = -a).
      * M2M(d)^T = S L2L(-d) S and L2L^T = S M2M S: the local shift matrix
        transposed is the multipole shift matrix, the compressions transpose
        into each other and commute with S (they preserve the degree).
      * M2L: T_c[t][s] = D_c[s+t] is symmetric and T_{-c} = S T_c S, so
        M2L^T for the pair (t <- s) is S M2L S for (s <- t) with class -c.
      * M2P^T = S P2L (sources := targets), P2L^T = M2P S.
    Writing the adjoint expansions as S-flipped vectors turns every stage
    into the forward kernel; this function only rearranges the lists.
    """
    nb = tree.nboxes
    nl = tree.nlevels
    levels = np.asarray(tree.box_levels)
    leaf = np.all(np.asarray(tree.box_child_ids) == 0, axis=0)

    # swapped particle roles
    tts = None
    if tree.target_to_source is not None:
        tts = np.full(tree.nsources, -1, dtype=np.int32)
        valid = tree.target_to_source >= 0
        tts[tree.target_to_source[valid]] = np.nonzero(valid)[0].astype(np.int32)
    tree_t = dataclasses.replace(
        tree,
        nsources=tree.ntargets, ntargets=tree.nsources,
        sources=tree.targets, targets=tree.sources,
        user_source_ids=_inverse_perm(tree.sorted_target_ids),
        sorted_target_ids=_inverse_perm(tree.user_source_ids),
        box_source_starts=tree.box_target_starts, box_target_starts=tree.box_source_starts,
        box_source_counts_cumul=tree.box_target_counts_cumul,
        box_target_counts_cumul=tree.box_source_counts_cumul,
        box_source_counts_nonchild=tree.box_target_counts_nonchild,
        box_target_counts_nonchild=tree.box_source_counts_nonchild,
        target_to_source=tts, _handle=tree._handle)

    has_src = tree.box_source_counts_cumul > 0
    has_tgt = tree.box_target_counts_cumul > 0
    src_boxes_t = np.asarray(trav.target_boxes)                       # leaves with targets
    tgt_boxes_t = np.asarray(trav.source_boxes)                       # leaves with sources
    src_parents_t = np.nonzero(~leaf & has_tgt)[0].astype(np.int32)
    ttp_t = np.nonzero(has_src)[0].astype(np.int32)

    # List 1^T: rows = source leaves
    l1s, l1l, _, _ = _transpose_csr(trav.target_boxes, trav.neighbor_source_boxes_starts,
                                    trav.neighbor_source_boxes_lists, tgt_boxes_t, nb)
    # List 2^T with reversed classes: rows = boxes with sources
    cls = np.asarray(tcls.from_sep_siblings_translation_classes)
    l2s, l2l, l2c, _ = _transpose_csr(trav.target_or_target_parent_boxes,
                                      trav.from_sep_siblings_starts,
                                      trav.from_sep_siblings_lists, ttp_t, nb, values=cls)
    vec = np.asarray(tcls.from_sep_siblings_translation_class_to_distance_vector)
    cls_ls = np.asarray(tcls.from_sep_siblings_translation_classes_level_starts)
    rev = np.arange(vec.shape[1], dtype=np.int32)
    for lev in range(nl):
        a, b = int(cls_ls[lev]), int(cls_ls[lev + 1])
        if a == b:
            continue
        h = tree.root_extent * 2.0 ** -lev
        key = {tuple(np.rint(vec[:, c] / h).astype(int)): c for c in range(a, b)}
        for c in range(a, b):
            rev[c] = key[tuple(-np.rint(vec[:, c] / h).astype(int))]
    l2c = rev[l2c] if len(l2c) else l2c

    # List 4^T -> List 3 of the adjoint (by level of the List-4 target box)
    l4_rows = trav.target_or_target_parent_boxes
    s4, l4, _, _ = _transpose_csr(l4_rows, trav.from_sep_bigger_starts,
                                  trav.from_sep_bigger_lists, tgt_boxes_t, nb)
    by_level_tb, by_level = [], []
    ent_lev = levels[l4] if len(l4) else np.zeros(0, dtype=np.int32)
    counts = np.diff(s4)
    ent_row = np.repeat(np.arange(len(tgt_boxes_t)), counts)
    for lev in range(nl):
        m = ent_lev == lev
        rows = ent_row[m]
        lst = l4[m]
        uniq, cnt = np.unique(rows, return_counts=True)
        st = np.zeros(len(uniq) + 1, dtype=np.int32)
        st[1:] = np.cumsum(cnt)
        by_level_tb.append(tgt_boxes_t[uniq].astype(np.int32))
        by_level.append(FromSepSmallerCSR(starts=st, lists=lst.astype(np.int32)))

    # List 3^T -> List 4 of the adjoint: rows = boxes with sources
    ent_t, ent_d = [], []
    for tbs, csr in zip(trav.target_boxes_sep_smaller_by_source_level,
                        trav.from_sep_smaller_by_level):
        cnt = np.diff(csr.starts)
        ent_t.append(np.repeat(np.asarray(tbs), cnt))
        ent_d.append(np.asarray(csr.lists[csr.starts[0]:csr.starts[-1]] if len(csr.starts) else []))
    ent_t = np.concatenate(ent_t) if ent_t else np.zeros(0, dtype=np.int64)
    ent_d = np.concatenate(ent_d) if ent_d else np.zeros(0, dtype=np.int64)
    pos = np.full(nb, -1, dtype=np.int64)
    pos[ttp_t] = np.arange(len(ttp_t))
    row = pos[ent_d.astype(np.int64)] if len(ent_d) else np.zeros(0, dtype=np.int64)
    order = np.lexsort((ent_t, row)) if len(row) else np.zeros(0, dtype=np.int64)
    s3 = np.zeros(len(ttp_t) + 1, dtype=np.int64)
    np.add.at(s3, row + 1, 1)
    s3 = np.cumsum(s3).astype(np.int32)
    l3 = ent_t[order].astype(np.int32)

    trav_t = FMMTraversalInfo(
        tree=tree_t,
        source_boxes=src_boxes_t, target_boxes=tgt_boxes_t,
        source_parent_boxes=src_parents_t, target_or_target_parent_boxes=ttp_t,
        level_start_source_box_nrs=np.asarray(trav.level_start_target_box_nrs),
        level_start_target_box_nrs=np.asarray(trav.level_start_source_box_nrs),
        level_start_source_parent_box_nrs=_level_starts(src_parents_t, levels, nl),
        level_start_target_or_target_parent_box_nrs=_level_starts(ttp_t, levels, nl),
        neighbor_source_boxes_starts=l1s, neighbor_source_boxes_lists=l1l,
        from_sep_siblings_starts=l2s, from_sep_siblings_lists=l2l,
        target_boxes_sep_smaller_by_source_level=by_level_tb,
        from_sep_smaller_by_level=by_level,
        from_sep_bigger_starts=s3, from_sep_bigger_lists=l3)
    tcls_t = TranslationClassesInfo(
        traversal=trav_t,
        from_sep_siblings_translation_classes=np.asarray(l2c, dtype=np.int32),
        from_sep_siblings_translation_class_to_distance_vector=vec,
        from_sep_siblings_translation_classes_level_starts=cls_ls)
    tree_t._traversal = trav_t
    tree_t._translation_classes = tcls_t
    return tree_t, trav_t, tcls_t
