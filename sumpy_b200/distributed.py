"""Several GPUs of one node: process-group plumbing and the distributed FMM.

Two ways of using more than one GPU:

* independent problems -- replicas of one evaluation, or a batch of point
  sets split across ranks (:func:`shard_problems`, longest first to the
  least loaded rank); no data crosses between ranks;
* one problem split across ranks -- :class:`DistributedSumpyExpansionWrangler`
  and :class:`DistributedFMMRunner`, the counterparts of sumpy's
  ``DistributedSumpyExpansionWrangler`` (sumpy/distributed.py:38-113) and
  boxtree's ``DistributedFMMRunner`` (driven as in
  sumpy/test/test_distributed.py:60-146).

The distributed FMM partitions the *leaves* of the global tree: sorted along
the Morton curve and cut into contiguous ranges of equal estimated work
(:func:`partition_boxes`). Every rank keeps the whole tree and all source
strengths (the near field reads neighbours' particles) and evaluates, on its
own GPU with the ordinary wrangler, a *local traversal*
(:func:`local_traversal`): the global interaction lists restricted to

* upward pass: P2M of its own source leaves and M2M over their ancestors --
  partial multipoles, since M2M is linear;
* exchange: the multipoles summed over all ranks (one all-reduce of the
  ``[nboxes][ncoeff]`` array over NCCL: sumpy's
  ``communicate_mpoles_via_allreduce`` mode), after which every rank holds
  the global multipoles;
* downward pass: Lists 1 and 3 and L2P for its own target leaves, Lists 2
  and 4 and L2L for their ancestors (coarse ancestors shared by several
  ranks are evaluated by each of them, for their own leaves only);
* potentials: each rank's are zero outside its own targets; a reduction to
  the root rank gives the global result.

Every (target, source) interaction of the global FMM is evaluated by exactly
one rank, so the sum equals the single-rank result up to rounding.
"""
from __future__ import annotations

import dataclasses
import datetime
import os

import numpy as np
import torch
import torch.distributed as dist


def env_ranks():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=300):
    """Initialise the default process group when WORLD_SIZE > 1; return
    (rank, world_size, local_rank)."""
    rank, world, local = env_ranks()
    if world > 1 and not dist.is_initialized():
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def _active(group=None):
    return dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (identity on one rank)."""
    if not _active():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_problems(costs, world):
    """Assign independent problems to ranks: largest cost first, each to the
    currently least loaded rank. Returns a list of index lists, one per rank."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


# {{{ partition of the leaves

def leaf_boxes(tree):
    """Boxes without children (the boxes that hold particles)."""
    return np.nonzero((np.asarray(tree.box_child_ids) == 0).all(axis=0))[0]


def morton_keys(tree, boxes):
    """Morton keys of boxes at the finest level (their lower corners'
    integer coordinates, bits interleaved x, y, z from the top)."""
    boxes = np.asarray(boxes, dtype=np.int64)
    top = tree.nlevels - 1
    lev = np.asarray(tree.box_levels, dtype=np.int64)[boxes]
    c = np.asarray(tree.box_coords, dtype=np.int64)[:, boxes] << (top - lev)
    key = np.zeros(len(boxes), dtype=np.int64)
    for bit in range(top - 1, -1, -1):
        for d in range(3):
            key = (key << 1) | ((c[d] >> bit) & 1)
    return key


def leaf_costs(tree, trav, ncoeff=121):
    """Estimated work of every box as a partition unit (nonzero on leaves):
    near-field pairs (List 1), List-3 evaluations, L2P and P2M point work,
    List-2 entries at the leaf, and List-4 source points (weights in units of
    one near-field pair)."""
    nb = tree.nboxes
    bsc = np.asarray(tree.box_source_counts_nonchild, dtype=np.int64)
    btc = np.asarray(tree.box_target_counts_nonchild, dtype=np.int64)
    cost = np.zeros(nb, dtype=np.float64)
    w_exp = ncoeff / 6.0
    tb = np.asarray(trav.target_boxes, dtype=np.int64)
    st = np.asarray(trav.neighbor_source_boxes_starts, dtype=np.int64)
    ls = np.asarray(trav.neighbor_source_boxes_lists, dtype=np.int64)
    csum = np.concatenate([[0], np.cumsum(bsc[ls])])
    cost[tb] += btc[tb] * (csum[st[1:]] - csum[st[:-1]])
    for tbs, csr in zip(trav.target_boxes_sep_smaller_by_source_level,
                        trav.from_sep_smaller_by_level):
        tbs = np.asarray(tbs, dtype=np.int64)
        if len(tbs):
            cost[tbs] += btc[tbs] * np.diff(np.asarray(csr.starts, dtype=np.int64)) * w_exp
    cost += (btc + bsc) * w_exp
    ttp = np.asarray(trav.target_or_target_parent_boxes, dtype=np.int64)
    s2 = np.asarray(trav.from_sep_siblings_starts, dtype=np.int64)
    cost[ttp] += np.diff(s2) * ncoeff
    s4 = np.asarray(trav.from_sep_bigger_starts, dtype=np.int64)
    l4 = np.asarray(trav.from_sep_bigger_lists, dtype=np.int64)
    c4 = np.concatenate([[0], np.cumsum(bsc[l4])])
    cost[ttp] += (c4[s4[1:]] - c4[s4[:-1]]) * w_exp
    leaves = leaf_boxes(tree)
    out = np.zeros(nb, dtype=np.float64)
    out[leaves] = cost[leaves] + 1.0
    return out


def partition_boxes(tree, trav, nranks, costs=None):
    """Owner rank of every leaf box (-1 for boxes with children): the leaves
    in Morton order, cut into ``nranks`` contiguous ranges of about equal
    cost (:func:`leaf_costs` unless ``costs`` is given). Deterministic, so
    every rank computes the same partition."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    leaves = leaf_boxes(tree)
    if costs is None:
        costs = leaf_costs(tree, trav)
    order = leaves[np.argsort(morton_keys(tree, leaves), kind="stable")]
    c = np.asarray(costs, dtype=np.float64)[order]
    cum = np.cumsum(c) - 0.5 * c          # midpoint of each leaf's cost interval
    total = float(c.sum()) if len(c) else 1.0
    rank = np.minimum((cum / max(total, 1e-300) * nranks).astype(np.int64), nranks - 1)
    owner = np.full(tree.nboxes, -1, dtype=np.int32)
    owner[order] = rank.astype(np.int32)
    return owner

# }}}


# {{{ local traversals

def _ancestors_or_self(tree, mask):
    """Boolean mask of the boxes that are ``mask`` boxes or their ancestors."""
    parent = np.asarray(tree.box_parent_ids, dtype=np.int64)
    out = np.zeros(tree.nboxes, dtype=bool)
    cur = np.nonzero(mask)[0]
    while cur.size:
        cur = cur[~out[cur]]
        out[cur] = True
        cur = parent[cur[cur != 0]] if cur.size else cur
    return out


def _keep_sorted(boxes, level_starts, keep):
    """Level-sorted box array restricted to ``keep`` boxes: (boxes, level
    starts, kept positions)."""
    boxes = np.asarray(boxes)
    ls = np.asarray(level_starts, dtype=np.int64)
    sel = np.nonzero(keep[np.asarray(boxes, dtype=np.int64)])[0]
    new_ls = np.searchsorted(sel, ls).astype(ls.dtype)
    return boxes[sel], new_ls, sel


def _keep_rows(starts, lists, rows, *per_entry):
    """CSR restricted to ``rows``: (starts, lists, *per_entry arrays)."""
    st = np.asarray(starts, dtype=np.int64)
    rows = np.asarray(rows, dtype=np.int64)
    cnt = np.diff(st)[rows]
    new_st = np.concatenate([[0], np.cumsum(cnt)])
    ent = np.repeat(st[rows] - new_st[:-1], cnt) + np.arange(int(new_st[-1]), dtype=np.int64)
    out = [new_st.astype(np.asarray(starts).dtype), np.asarray(lists)[ent]]
    out += [np.asarray(a)[ent] for a in per_entry]
    return out


def local_traversal(tree, trav, tcls, owner, rank, restrict_sources=True,
                    restrict_targets=True):
    """The global traversal restricted to one rank's share (see the module
    docstring): returns (traversal, translation classes) with the global
    tree. ``restrict_sources`` / ``restrict_targets`` switch off either half
    of the restriction (the other ranks' sources, or targets, are then
    included; useful to check the two halves separately)."""
    own = np.asarray(owner) == rank
    full = np.ones(tree.nboxes, dtype=bool)
    src_leaf = own if restrict_sources else full
    tgt_leaf = own if restrict_targets else full
    src_anc = _ancestors_or_self(tree, src_leaf) if restrict_sources else full
    tgt_anc = _ancestors_or_self(tree, tgt_leaf) if restrict_targets else full

    sb, sb_ls, _ = _keep_sorted(trav.source_boxes, trav.level_start_source_box_nrs, src_leaf)
    spb, spb_ls, _ = _keep_sorted(trav.source_parent_boxes,
                                  trav.level_start_source_parent_box_nrs, src_anc)
    tb, tb_ls, tsel = _keep_sorted(trav.target_boxes, trav.level_start_target_box_nrs,
                                   tgt_leaf)
    n1_st, n1_ls = _keep_rows(trav.neighbor_source_boxes_starts,
                              trav.neighbor_source_boxes_lists, tsel)
    ttp, ttp_ls, psel = _keep_sorted(trav.target_or_target_parent_boxes,
                                     trav.level_start_target_or_target_parent_box_nrs,
                                     tgt_anc)
    s2_st, s2_ls, s2_cls = _keep_rows(trav.from_sep_siblings_starts,
                                      trav.from_sep_siblings_lists, psel,
                                      tcls.from_sep_siblings_translation_classes)
    s4_st, s4_ls = _keep_rows(trav.from_sep_bigger_starts, trav.from_sep_bigger_lists, psel)
    by_tb, by_csr = [], []
    for tbs, csr in zip(trav.target_boxes_sep_smaller_by_source_level,
                        trav.from_sep_smaller_by_level):
        tbs = np.asarray(tbs)
        rows = np.nonzero(tgt_leaf[tbs.astype(np.int64)])[0] if len(tbs) else \
            np.zeros(0, dtype=np.int64)
        st3, ls3 = _keep_rows(csr.starts, csr.lists, rows)
        by_tb.append(tbs[rows])
        by_csr.append(type(csr)(starts=st3, lists=ls3))
    loc = dataclasses.replace(
        trav, source_boxes=sb, level_start_source_box_nrs=sb_ls,
        source_parent_boxes=spb, level_start_source_parent_box_nrs=spb_ls,
        target_boxes=tb, level_start_target_box_nrs=tb_ls,
        neighbor_source_boxes_starts=n1_st, neighbor_source_boxes_lists=n1_ls,
        target_or_target_parent_boxes=ttp,
        level_start_target_or_target_parent_box_nrs=ttp_ls,
        from_sep_siblings_starts=s2_st, from_sep_siblings_lists=s2_ls,
        from_sep_bigger_starts=s4_st, from_sep_bigger_lists=s4_ls,
        target_boxes_sep_smaller_by_source_level=by_tb, from_sep_smaller_by_level=by_csr)
    loc_cls = dataclasses.replace(tcls, traversal=loc,
                                  from_sep_siblings_translation_classes=s2_cls)
    loc._translation_classes = loc_cls
    return loc, loc_cls

# }}}


# {{{ collectives

def allreduce_sum_(tensor, group=None):
    """In-place sum over the ranks of ``group`` (complex tensors as their
    real views); a no-op on one rank."""
    if not _active(group):
        return tensor
    dist.all_reduce(torch.view_as_real(tensor) if tensor.is_complex() else tensor,
                    op=dist.ReduceOp.SUM, group=group)
    return tensor


def reduce_sum_to_root_(tensor, group=None, root=0):
    """In-place sum onto rank ``root`` of ``group``; a no-op on one rank."""
    if not _active(group):
        return tensor
    dist.reduce(torch.view_as_real(tensor) if tensor.is_complex() else tensor,
                dst=dist.get_global_rank(group, root) if group is not None else root,
                op=dist.ReduceOp.SUM, group=group)
    return tensor


def broadcast_(tensor, group=None, root=0):
    if not _active(group):
        return tensor
    dist.broadcast(torch.view_as_real(tensor) if tensor.is_complex() else tensor,
                   src=dist.get_global_rank(group, root) if group is not None else root,
                   group=group)
    return tensor


def _rank(group=None):
    return dist.get_rank(group) if dist.is_available() and dist.is_initialized() else 0


def _world(group=None):
    return dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1

# }}}


# {{{ tree transport

def _fields(obj, skip):
    return {f.name: getattr(obj, f.name) for f in dataclasses.fields(obj)
            if f.name not in skip and not f.name.startswith("_")}


def pack_tree(tree, trav, tcls):
    """The tree, traversal and translation classes as plain data (numpy
    arrays and scalars) for sending to other ranks."""
    t = _fields(tree, ())
    v = _fields(trav, ("tree",))
    v["from_sep_smaller_by_level"] = [(c.starts, c.lists) for c in trav.from_sep_smaller_by_level]
    c = _fields(tcls, ("traversal",))
    return {"tree": t, "trav": v, "tcls": c}


def unpack_tree(data):
    from sumpy_b200.tree import FMMTraversalInfo, FromSepSmallerCSR, TranslationClassesInfo, Tree
    tree = Tree(**data["tree"])
    v = dict(data["trav"])
    v["from_sep_smaller_by_level"] = [FromSepSmallerCSR(starts=s, lists=l)
                                      for s, l in v["from_sep_smaller_by_level"]]
    trav = FMMTraversalInfo(tree=tree, **v)
    tcls = TranslationClassesInfo(traversal=trav, **data["tcls"])
    tree._traversal = trav
    tree._translation_classes = tcls
    return tree, trav, tcls


def broadcast_tree(tree, group=None, root=0):
    """(tree, traversal, translation classes) of ``root`` on every rank of
    ``group`` (``tree`` is ignored on the other ranks)."""
    if not _active(group):
        return tree, tree._traversal, tree._translation_classes
    payload = [pack_tree(tree, tree._traversal, tree._translation_classes)
               if _rank(group) == root else None]
    dist.broadcast_object_list(
        payload, src=dist.get_global_rank(group, root) if group is not None else root,
        group=group)
    return unpack_tree(payload[0])

# }}}


# {{{ wrangler and runner

def _wrangler_base():
    from sumpy_b200.fmm import SumpyExpansionWrangler
    return SumpyExpansionWrangler


class DistributedSumpyExpansionWrangler(_wrangler_base()):
    """``sumpy.distributed.DistributedSumpyExpansionWrangler``
    (sumpy/distributed.py:38-113): the expansion wrangler of one rank,
    evaluating its local traversal (:func:`local_traversal`) on this
    process's GPU. ``comm`` is a ``torch.distributed`` process group (None:
    the default group). Multipoles are exchanged with one all-reduce after
    the upward pass (``communicate_mpoles_via_allreduce``, the only mode
    here); the point-to-point exchange of sumpy's other mode is not built.
    Evaluation is eager (no CUDA-graph capture around the collectives)."""

    def __init__(self, actx, comm, tree_indep, local_traversal, global_traversal, dtype,
                 fmm_level_to_order, communicate_mpoles_via_allreduce=True, **kwargs):
        if not communicate_mpoles_via_allreduce:
            raise NotImplementedError(
                "only communicate_mpoles_via_allreduce=True is implemented")
        kwargs["cuda_graph"] = False
        super().__init__(tree_indep, local_traversal, dtype, fmm_level_to_order, **kwargs)
        self.comm = comm
        self.global_traversal = global_traversal
        self.communicate_mpoles_via_allreduce = True
        self.traversal_in_device_memory = True

    @property
    def is_mpi_root(self):
        return _rank(self.comm) == 0

    def communicate_mpoles(self, actx, mpole_exps, return_stats=False):
        """Sum the partial multipoles of all ranks in place (NCCL all-reduce
        on the current stream's device)."""
        allreduce_sum_(mpole_exps, self.comm)
        return {"bytes": mpole_exps.numel() * mpole_exps.element_size()} \
            if return_stats else None

    def distribute_source_weights(self, src_weight_vecs, src_idx_all_ranks=None):
        """Strengths are replicated: every rank's near field reads sources of
        other ranks' boxes (the runner broadcasts them before evaluating)."""
        return src_weight_vecs

    def gather_potential_results(self, potentials, tgt_idx_all_ranks=None):
        """Sum of all ranks' potentials on the root rank (each rank's are zero
        outside its own targets); None on the other ranks."""
        for p in potentials:
            reduce_sum_to_root_(p, self.comm)
        return potentials if self.is_mpi_root else None


class DistributedFMMRunner:
    """``boxtree.distributed.DistributedFMMRunner`` as sumpy's test drives it
    (sumpy/test/test_distributed.py:127-136): ``global_tree`` on the root
    rank (ignored elsewhere), a traversal builder, and
    ``wrangler_factory(local_traversal, global_traversal)`` returning a
    :class:`DistributedSumpyExpansionWrangler`. The tree is sent from the
    root to every rank, each rank computes the same leaf partition and its
    local traversal; :meth:`drive_dfmm` broadcasts the strengths, evaluates
    and returns the potentials on the root (None elsewhere)."""

    def __init__(self, actx, global_tree, traversal_builder, wrangler_factory, comm=None,
                 costs=None):
        self.comm = comm
        tree, trav, tcls = broadcast_tree(global_tree, comm)
        if traversal_builder is not None:
            trav, _ = traversal_builder(actx, tree)
        self.global_tree, self.global_traversal = tree, trav
        self.nranks = _world(comm)
        self.rank = _rank(comm)
        self.owner = partition_boxes(tree, trav, self.nranks, costs)
        self.local_traversal, self.local_translation_classes = local_traversal(
            tree, trav, tcls, self.owner, self.rank)
        self.wrangler = wrangler_factory(self.local_traversal, self.global_traversal)

    def drive_dfmm(self, actx, source_weights, timing_data=None):
        from sumpy_b200.drive import drive_fmm
        w = self.wrangler
        vecs = []
        for x in source_weights:
            t = torch.as_tensor(x, device=w.device)
            if t.numel() != self.global_tree.nsources:
                t = torch.empty(self.global_tree.nsources, dtype=w._tdtype, device=w.device)
            t = t.to(w._tdtype).contiguous()
            vecs.append(broadcast_(t, self.comm))
        pot = drive_fmm(actx, w, vecs)
        return w.gather_potential_results(pot)

# }}}
