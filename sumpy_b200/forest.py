"""Many independent FMM problems as one forest, evaluated by one ``drive_fmm``.

A batch of problems (each its own sources, targets and strengths) is built
tree by tree in a common root box (``build_all(..., bbox=...)``), so level
``l`` has the same box size, rscale and translation-class vectors in every
tree. The trees are then merged into one :class:`~sumpy_b200.tree.Tree`
whose level ``l`` holds the level-``l`` boxes of all problems (problem after
problem), with the interaction lists renumbered. Lists never cross problems,
so the merged traversal is the disjoint union of the per-problem ones and
sumpy's wrangler (``sumpy/fmm.py:609-1086``) runs every stage of every
level for the whole batch in one launch, with the storage layout unchanged
(``sumpy/fmm.py:399-485``: level-major flat arrays).

Particles are stored problem after problem (tree order inside a problem);
user order is the concatenation of the problems' user orders, so a batch's
strengths are ``torch.cat`` of the per-problem ones and its potentials split
at :attr:`Forest.target_starts`.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from sumpy_b200.tree import (
    FMMTraversalInfo,
    FromSepSmallerCSR,
    Tree,
    TranslationClassesInfo,
    build_all,
)


@dataclass
class Forest:
    """Where each problem lives in the merged arrays."""
    nproblems: int
    source_starts: np.ndarray   # [nproblems + 1], user and tree order alike
    target_starts: np.ndarray   # [nproblems + 1]
    box_maps: list              # per problem: merged box id of each of its boxes

    def split_targets(self, values):
        """Per-problem views of a merged ``[ntargets]`` result."""
        return [values[int(a):int(b)] for a, b in zip(self.target_starts[:-1],
                                                      self.target_starts[1:])]


def _cat(parts, dtype=np.int32):
    if not parts:
        return np.zeros(0, dtype=dtype)
    return np.concatenate(parts, dtype=dtype, casting="unsafe")


def _level_sorted(lists, level_starts, maps, nl):
    """Merge per-problem level-sorted box lists: level by level, problem
    after problem. Returns the merged list, its level starts and the row
    blocks ``(problem, begin, end)`` (per-problem row ranges) in merged
    order."""
    out, ls, blocks = [], np.zeros(nl + 1, dtype=np.int32), []
    n = 0
    for lev in range(nl):
        for i, (lst, st) in enumerate(zip(lists, level_starts)):
            if lev + 1 >= len(st):
                continue
            a, b = int(st[lev]), int(st[lev + 1])
            if a == b:
                continue
            out.append(maps[i][lst[a:b]])
            blocks.append((i, a, b))
            n += b - a
        ls[lev + 1] = n
    return _cat(out), ls, blocks


def _merge_csr(blocks, starts, lists, maps, values=None):
    """Merge per-problem CSR lists row block by row block (``blocks`` as
    returned by :func:`_level_sorted`); entries are box ids mapped by
    ``maps``; ``values`` ride along unchanged."""
    counts, out, vout = [], [], []
    for i, a, b in blocks:
        st = np.asarray(starts[i], dtype=np.int64)
        counts.append(np.diff(st[a:b + 1]))
        e0, e1 = int(st[a]), int(st[b])
        out.append(maps[i][np.asarray(lists[i])[e0:e1]])
        if values is not None:
            vout.append(np.asarray(values[i])[e0:e1])
    counts = _cat(counts, np.int64)
    new_starts = np.zeros(len(counts) + 1, dtype=np.int64)
    np.cumsum(counts, out=new_starts[1:])
    return (new_starts.astype(np.int32), _cat(out),
            None if values is None else _cat(vout))


def merge_trees(parts):
    """Merge ``[(tree, trav, tcls), ...]`` built in one root box into one
    forest ``(tree, trav, tcls, Forest)``."""
    if not parts:
        raise ValueError("empty batch")
    trees = [p[0] for p in parts]
    travs = [p[1] for p in parts]
    tclss = [p[2] for p in parts]
    ext = trees[0].root_extent
    bmin = np.asarray(trees[0].bounding_box[0])
    sat = trees[0].sources_are_targets
    for t in trees:
        if t.root_extent != ext or not np.array_equal(np.asarray(t.bounding_box[0]), bmin):
            raise ValueError("forest trees must share one root box (build them with bbox=)")
        if t.sources_are_targets != sat:
            raise ValueError("forest trees must all have (or all lack) separate targets")
    P = len(trees)
    nl = max(t.nlevels for t in trees)

    # {{{ box numbering: level by level, problem after problem

    cnt = np.zeros((P, nl), dtype=np.int64)
    for i, t in enumerate(trees):
        ls = np.asarray(t.level_start_box_nrs, dtype=np.int64)
        cnt[i, :t.nlevels] = np.diff(ls)
    level_tot = cnt.sum(axis=0)
    LS = np.zeros(nl + 1, dtype=np.int64)
    np.cumsum(level_tot, out=LS[1:])
    off = LS[:-1][None, :] + np.cumsum(cnt, axis=0) - cnt        # [P, nl]
    maps = []
    for i, t in enumerate(trees):
        lev = np.asarray(t.box_levels, dtype=np.int64)
        ls = np.asarray(t.level_start_box_nrs, dtype=np.int64)
        maps.append((off[i, lev] + np.arange(t.nboxes) - ls[lev]).astype(np.int32))
    NB = int(LS[-1])

    # }}}

    src_st = np.zeros(P + 1, dtype=np.int64)
    tgt_st = np.zeros(P + 1, dtype=np.int64)
    np.cumsum([t.nsources for t in trees], out=src_st[1:])
    np.cumsum([t.ntargets for t in trees], out=tgt_st[1:])

    centers = np.zeros((3, NB))
    levels = np.zeros(NB, dtype=np.int32)
    parent = np.zeros(NB, dtype=np.int32)
    child = np.zeros((8, NB), dtype=np.int32)
    coords = np.zeros((3, NB), dtype=np.int32)
    bss = np.zeros(NB, dtype=np.int32)
    bscc = np.zeros(NB, dtype=np.int32)
    bscn = np.zeros(NB, dtype=np.int32)
    bts = np.zeros(NB, dtype=np.int32)
    btcc = np.zeros(NB, dtype=np.int32)
    btcn = np.zeros(NB, dtype=np.int32)
    for i, t in enumerate(trees):
        m = maps[i]
        centers[:, m] = t.box_centers
        levels[m] = t.box_levels
        par = m[np.asarray(t.box_parent_ids, dtype=np.int64)]
        par[0] = m[0]                       # a root is its own parent
        parent[m] = par
        ch = np.asarray(t.box_child_ids, dtype=np.int64)
        child[:, m] = np.where(ch > 0, m[ch], 0)
        coords[:, m] = t.box_coords
        bss[m] = np.asarray(t.box_source_starts) + src_st[i]
        bscc[m] = t.box_source_counts_cumul
        bscn[m] = t.box_source_counts_nonchild
        bts[m] = np.asarray(t.box_target_starts) + tgt_st[i]
        btcc[m] = t.box_target_counts_cumul
        btcn[m] = t.box_target_counts_nonchild

    def ids(name, starts):
        return _cat([np.asarray(getattr(t, name)) + starts[i] for i, t in enumerate(trees)],
                    np.int32)

    tts = None
    if sat:
        tts = _cat([np.where(np.asarray(t.target_to_source) >= 0,
                             np.asarray(t.target_to_source) + src_st[i], -1)
                    for i, t in enumerate(trees)])
    tree = Tree(
        dimensions=3, nsources=int(src_st[-1]), ntargets=int(tgt_st[-1]), nboxes=NB,
        nlevels=nl, sources_are_targets=sat, root_extent=ext,
        bounding_box=(bmin, bmin + ext),
        sources=np.concatenate([t.sources for t in trees], axis=1),
        targets=np.concatenate([t.targets for t in trees], axis=1),
        user_source_ids=ids("user_source_ids", src_st),
        sorted_target_ids=ids("sorted_target_ids", tgt_st),
        level_start_box_nrs=LS.astype(np.int32),
        box_centers=centers, box_levels=levels, box_parent_ids=parent,
        box_child_ids=child, box_coords=coords,
        box_source_starts=bss, box_source_counts_cumul=bscc,
        box_source_counts_nonchild=bscn,
        box_target_starts=bts, box_target_counts_cumul=btcc,
        box_target_counts_nonchild=btcn,
        target_to_source=tts)

    # {{{ traversal

    def boxes(name, lsname):
        return _level_sorted([np.asarray(getattr(tr, name), dtype=np.int64) for tr in travs],
                             [np.asarray(getattr(tr, lsname)) for tr in travs], maps, nl)

    sb, sb_ls, _ = boxes("source_boxes", "level_start_source_box_nrs")
    tb, tb_ls, tb_blk = boxes("target_boxes", "level_start_target_box_nrs")
    spb, spb_ls, _ = boxes("source_parent_boxes", "level_start_source_parent_box_nrs")
    ttp, ttp_ls, ttp_blk = boxes("target_or_target_parent_boxes",
                                 "level_start_target_or_target_parent_box_nrs")

    l1s, l1l, _ = _merge_csr(tb_blk, [tr.neighbor_source_boxes_starts for tr in travs],
                             [tr.neighbor_source_boxes_lists for tr in travs], maps)
    l2s, l2l, l2c = _merge_csr(ttp_blk, [tr.from_sep_siblings_starts for tr in travs],
                               [tr.from_sep_siblings_lists for tr in travs], maps,
                               values=[tc.from_sep_siblings_translation_classes
                                       for tc in tclss])
    l4s, l4l, _ = _merge_csr(ttp_blk, [tr.from_sep_bigger_starts for tr in travs],
                             [tr.from_sep_bigger_lists for tr in travs], maps)

    by_level_tb, by_level = [], []
    for lev in range(nl):
        rows, blk = [], []
        for i, tr in enumerate(travs):
            if lev >= len(tr.from_sep_smaller_by_level):
                continue
            tbs = np.asarray(tr.target_boxes_sep_smaller_by_source_level[lev], dtype=np.int64)
            if len(tbs) == 0:
                continue
            rows.append(maps[i][tbs])
            blk.append((i, 0, len(tbs)))
        s3, l3, _ = _merge_csr(
            blk, [tr.from_sep_smaller_by_level[lev].starts if lev < len(
                tr.from_sep_smaller_by_level) else None for tr in travs],
            [tr.from_sep_smaller_by_level[lev].lists if lev < len(
                tr.from_sep_smaller_by_level) else None for tr in travs], maps)
        by_level_tb.append(_cat(rows))
        by_level.append(FromSepSmallerCSR(starts=s3, lists=l3))

    trav = FMMTraversalInfo(
        tree=tree, source_boxes=sb, target_boxes=tb, source_parent_boxes=spb,
        target_or_target_parent_boxes=ttp,
        level_start_source_box_nrs=sb_ls, level_start_target_box_nrs=tb_ls,
        level_start_source_parent_box_nrs=spb_ls,
        level_start_target_or_target_parent_box_nrs=ttp_ls,
        neighbor_source_boxes_starts=l1s, neighbor_source_boxes_lists=l1l,
        from_sep_siblings_starts=l2s, from_sep_siblings_lists=l2l,
        target_boxes_sep_smaller_by_source_level=by_level_tb,
        from_sep_smaller_by_level=by_level,
        from_sep_bigger_starts=l4s, from_sep_bigger_lists=l4l)

    # translation classes depend on the level and the root box only: take the
    # deepest tree's table
    deep = tclss[int(np.argmax([t.nlevels for t in trees]))]
    tcls = TranslationClassesInfo(
        traversal=trav,
        from_sep_siblings_translation_classes=l2c,
        from_sep_siblings_translation_class_to_distance_vector=(
            deep.from_sep_siblings_translation_class_to_distance_vector),
        from_sep_siblings_translation_classes_level_starts=(
            deep.from_sep_siblings_translation_classes_level_starts))

    # }}}

    tree._traversal = trav
    tree._translation_classes = tcls
    forest = Forest(nproblems=P, source_starts=src_st, target_starts=tgt_st, box_maps=maps)
    return tree, trav, tcls, forest


def build_forest(sources, targets=None, max_particles_in_box=30, bbox=None, max_levels=None,
                 threads=8, device=None):
    """Build one forest over a batch of problems.

    :arg sources: list of ``(3, n_i)`` arrays.
    :arg targets: ``None`` (every problem evaluates at its sources, with
        exclude_self available) or a list of ``(3, m_i)`` arrays.
    :arg bbox: the common root box as a ``(3, 2)`` array; default the
        bounding cube of all particles of the batch.
    :arg device: build the whole forest in one pass on this GPU
        (``sumpy_tree_gpu_build`` with one problem per root box); the same
        arrays, bit for bit, as per-problem host trees merged by
        :func:`merge_trees`. Default: host trees built in ``threads`` threads,
        then merged.
    """
    P = len(sources)
    if targets is not None and len(targets) != P:
        raise ValueError("one target array per problem")
    if bbox is None:
        allp = [np.asarray(s, dtype=np.float64) for s in sources]
        if targets is not None:
            allp += [np.asarray(t, dtype=np.float64) for t in targets]
        lo = np.min([a.min(axis=1) for a in allp if a.size], axis=0)
        hi = np.max([a.max(axis=1) for a in allp if a.size], axis=0)
        ext = float(np.max(hi - lo)) or 1.0
        ext *= 1 + 1e-9
        lo = lo - 0.5 * (ext - (hi - lo))
        bbox = np.stack([lo, lo + ext], axis=1)
    if device is not None:
        return build_forest_gpu(sources, targets, max_particles_in_box, bbox, max_levels, device)

    def one(i):
        return build_all(sources[i], None if targets is None else targets[i],
                         max_particles_in_box, max_levels, bbox=bbox)

    with ThreadPoolExecutor(max_workers=max(1, int(threads))) as ex:
        parts = list(ex.map(one, range(P)))
    return merge_trees(parts)


def build_forest_gpu(sources, targets, max_particles_in_box, bbox, max_levels, device):
    """The forest of :func:`build_forest` built on the GPU in one pass: all
    problems' particles concatenated, one root box per problem in the common
    root box ``bbox``."""
    import torch
    from sumpy_b200.tree import _objects, _root_box, gpu_tree_handle

    def cat(arrs):
        ts = [torch.as_tensor(a, dtype=torch.float64).reshape(3, -1) for a in arrs]
        return torch.cat(ts, dim=1).to(device).contiguous()

    P = len(sources)
    src = cat(sources)
    tgt = None if targets is None else cat(targets)
    src_st = np.zeros(P + 1, dtype=np.int64)
    np.cumsum([np.shape(s)[1] for s in sources], out=src_st[1:])
    if targets is None:
        tgt_st = src_st.copy()
    else:
        tgt_st = np.zeros(P + 1, dtype=np.int64)
        np.cumsum([np.shape(t)[1] for t in targets], out=tgt_st[1:])
    bmin, ext = _root_box(bbox)
    H = gpu_tree_handle(src, tgt, max_particles_in_box, max_levels, bmin, ext,
                        source_starts=src_st, target_starts=None if targets is None else tgt_st)
    tree, trav, tcls = _objects(H, keep_handle=False)
    prob = H.get("box_problem")
    del H
    order = np.argsort(prob, kind="stable").astype(np.int32)
    cuts = np.zeros(P + 1, dtype=np.int64)
    np.cumsum(np.bincount(prob, minlength=P), out=cuts[1:])
    maps = [order[cuts[i]:cuts[i + 1]] for i in range(P)]
    return tree, trav, tcls, Forest(nproblems=P, source_starts=src_st, target_starts=tgt_st,
                                    box_maps=maps)
