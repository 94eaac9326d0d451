"""Expansion wrangler with sumpy's interface, running the B200 kernels.

``SumpyTreeIndependentDataForWrangler`` and ``SumpyExpansionWrangler`` keep
the constructor and method signatures of sumpy/fmm.py:99-252 and 264-1086,
so a boxtree-style ``drive_fmm`` (here :func:`sumpy_b200.drive.drive_fmm`)
runs unchanged. Arrays are torch CUDA tensors; the ``actx`` arguments are
accepted for call compatibility and ignored. Each method launches one C-ABI
entry point (``include/sumpy_b200.h``) per tree level on the current torch
stream, without host synchronisation.

Storage is sumpy's (sumpy/fmm.py:399-485, 1093-1115): one flat FP64 array
per expansion kind, level-major, each level a row-major
``(nboxes_level, ncoeff)`` block.

Beyond sumpy's knobs, the wrangler takes ``precision``: ``"fp64"`` (every
stage in FP64) or ``"mixed"`` (FP32 near field, M2P and P2L with FP64
offsets and sums; M2L and M2M as split-FP32 (3xTF32) GEMMs on the tcgen05
tensor cores with FP32 accumulation and FP64 results; the other stages FP64), ``gradient`` (also
return the potential's gradient at the targets), ``m2l_item_groups`` (class
groups per M2L work item, one CTA each; :mod:`sumpy_b200.autotune` picks it)
and ``cuda_graph`` (``drive_fmm`` replays the evaluation from a captured CUDA
graph).
"""
from __future__ import annotations

import math
from functools import cached_property

import numpy as np
import torch

from sumpy_b200 import _capi
from sumpy_b200._capi import call, dptr, stream_ptr
from sumpy_b200.expansion import (
    helmholtz_m2l_class_matrices,
    l2l_operator,
    m2l_class_matrices,
    m2m_operator,
    octant_offsets,
    real_embedding,
)
from sumpy_b200.kernel import HelmholtzKernel, helmholtz_k, is_scale_invariant

_i32 = _capi.i32
_i64 = _capi.i64
_c = _capi.cint
_d = _capi.dbl

M2L_TILE = 64          # FP64 GEMM tile (target boxes)
M2L_TILE_TC = 128      # tensor-core tile (MMA N)
M2L_ITEM_GROUPS = 192  # class groups per tensor-core work item (one CTA)
ITEM_ROUNDS = 16       # rounds (one source box / 32 sources each) per mixed M2P / P2L item
M2P_ITEM_GROUPS = 8    # lane groups per warp in the M2P item kernel (fixed by the kernel)
L2P_ITEM_SLOTS = 4     # boxes per packed L2P item (fixed by the kernel)
HL2P_ITEM_SLOTS = 4    # the same for the Helmholtz packed L2P


def _npad(order):
    """Row stride of the FP32 multipole copy (sumpy_mpoles_to_f32)."""
    return ((order + 1) ** 2 + 3) & ~3


def _expand_ranges(starts, counts):
    """Concatenation of range(starts[i], starts[i] + counts[i]) over i."""
    counts = np.asarray(counts, dtype=np.int64)
    total = int(counts.sum())
    if total == 0:
        return np.zeros(0, dtype=np.int64)
    first = np.cumsum(counts) - counts
    return np.repeat(np.asarray(starts, dtype=np.int64) - first, counts) + np.arange(total)


def m2p_items(tree, target_boxes_by_source_level, source_boxes_by_level,
              rounds=ITEM_ROUNDS, groups=M2P_ITEM_GROUPS):
    """Work items of the one-launch mixed M2P (sumpy_e2p_from_items_mixed).

    Each target box's targets go 32 per chunk; a chunk of ntc targets runs on
    lane groups of g = max(32 / groups, next_pow2(ntc)) lanes, 32 / g source
    boxes per round, and an item takes ``rounds`` rounds of its chunk's
    List-3 boxes. Returns (items int32 [n, 4] longest first, the levels'
    source box lists concatenated)."""
    bts = np.asarray(tree.box_target_starts, dtype=np.int64)
    btc = np.asarray(tree.box_target_counts_nonchild, dtype=np.int64)
    out, cost, lists = [], [], []
    off = 0
    for lev, ssn in enumerate(source_boxes_by_level):
        tb = np.asarray(target_boxes_by_source_level[lev], dtype=np.int64)
        lst = np.asarray(ssn.lists, dtype=np.int32)
        if len(tb) == 0:
            lists.append(lst)
            off += len(lst)
            continue
        starts = np.asarray(ssn.starts, dtype=np.int64)
        ln = np.diff(starts)[:len(tb)]
        nt = btc[tb]
        nch = np.where((ln > 0) & (nt > 0), (nt + 31) // 32, 0)
        cb = np.repeat(np.arange(len(tb)), nch)
        ci = _expand_ranges(np.zeros(len(tb), dtype=np.int64), nch)
        ntc = np.minimum(32, nt[cb] - 32 * ci)
        t0 = bts[tb][cb] + 32 * ci
        g = np.full(len(ntc), 32 // groups, dtype=np.int64)
        while (g < ntc).any():
            g = np.where(g < ntc, 2 * g, g)
        nph = 32 // g
        per = nph * rounds
        lnc = ln[cb]
        nit = (lnc + per - 1) // per
        ic = np.repeat(np.arange(len(ntc)), nit)
        j = _expand_ranges(np.zeros(len(ntc), dtype=np.int64), nit)
        nb = np.minimum(per[ic], lnc[ic] - j * per[ic])
        l0 = starts[cb][ic] + off + j * per[ic]
        out.append(np.stack([t0[ic], l0, nb, ntc[ic] | (lev << 8)], axis=1))
        cost.append((nb + nph[ic] - 1) // nph[ic])
        lists.append(lst)
        off += len(lst)
    if not out:
        return np.zeros((0, 4), np.int32), np.concatenate(lists) if lists else np.zeros(0, np.int32)
    items = np.concatenate(out)
    order = np.argsort(-np.concatenate(cost), kind="stable")
    return np.ascontiguousarray(items[order], dtype=np.int32), np.concatenate(lists)


def _box_levels(level_starts, n):
    return np.repeat(np.arange(len(level_starts) - 1),
                     np.diff(np.asarray(level_starts, dtype=np.int64)))[:n]


def l2p_items(tree, level_starts, target_boxes, max_slots=L2P_ITEM_SLOTS):
    """Packed work items of the one-launch L2P
    (sumpy_e2p_from_single_box_packed_f64): a box's targets go 32 per slot;
    slots of fewer than 32 targets share an item (next fit, largest first)
    up to 32 targets and ``max_slots`` slots. Returns (items int32 [n, 2] =
    first slot, number of slots; slots int32 [m, 4] = box, first target,
    number of targets, level)."""
    bts = np.asarray(tree.box_target_starts, dtype=np.int64)
    btc = np.asarray(tree.box_target_counts_nonchild, dtype=np.int64)
    tb = np.asarray(target_boxes, dtype=np.int64)
    lev = _box_levels(level_starts, len(tb))
    nt = btc[tb]
    nfull = nt // 32
    fb = np.repeat(np.arange(len(tb)), nfull)
    fc = _expand_ranges(np.zeros(len(tb), dtype=np.int64), nfull)
    full = np.stack([tb[fb], bts[tb][fb] + 32 * fc, np.full(len(fb), 32), lev[fb]], axis=1)
    rem = nt - 32 * nfull
    rb = np.nonzero(rem > 0)[0]
    rb = rb[np.argsort(-rem[rb], kind="stable")]
    part = np.stack([tb[rb], bts[tb][rb] + 32 * nfull[rb], rem[rb], lev[rb]], axis=1)
    slots = np.concatenate([full.reshape(-1, 4), part.reshape(-1, 4)]).astype(np.int32)
    first, cnt = _pack_next_fit(part[:, 2].astype(np.int32), 32, max_slots)
    items = np.concatenate([
        np.stack([np.arange(len(full)), np.ones(len(full), dtype=np.int64)], axis=1),
        np.stack([first.astype(np.int64) + len(full), cnt.astype(np.int64)], axis=1)])
    return (np.ascontiguousarray(items.reshape(-1, 2), dtype=np.int32),
            np.ascontiguousarray(slots))


def _pack_next_fit(sizes, capacity, max_count):
    """Next-fit packing (host library sumpy_pack_next_fit): (first, count)
    of each item, entries in the given order."""
    import ctypes

    from sumpy_b200._lib import load_tree_library
    lib = load_tree_library()
    n = len(sizes)
    sizes = np.ascontiguousarray(sizes, dtype=np.int32)
    first = np.empty(max(n, 1), dtype=np.int32)
    cnt = np.empty(max(n, 1), dtype=np.int32)
    ni = ctypes.c_int64(0)
    rc = lib.sumpy_pack_next_fit(
        ctypes.c_int64(n), sizes.ctypes.data_as(ctypes.c_void_p), ctypes.c_int32(capacity),
        ctypes.c_int32(max_count), first.ctypes.data_as(ctypes.c_void_p),
        cnt.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ni))
    if rc:
        raise RuntimeError(lib.sumpy_tree_last_error().decode())
    return first[:ni.value], cnt[:ni.value]


def p2l_items(tree, level_starts, target_boxes, starts, lists, rounds=ITEM_ROUNDS):
    """Work items of the one-launch mixed P2L (sumpy_p2e_from_items_mixed):
    the sources of each target box's List-4 boxes as one flat index array,
    cut into items of at most 32 * ``rounds`` sources. Returns (items int32
    [n, 4] longest first, source index int32)."""
    bss = np.asarray(tree.box_source_starts, dtype=np.int64)
    bsc = np.asarray(tree.box_source_counts_nonchild, dtype=np.int64)
    starts = np.asarray(starts, dtype=np.int64)
    lists = np.asarray(lists, dtype=np.int64)
    cnt = bsc[lists]
    src_index = _expand_ranges(bss[lists], cnt)
    F = np.concatenate([[0], np.cumsum(cnt)])
    ntb = len(starts) - 1
    f0 = F[starts[:-1]]
    n = F[starts[1:]] - f0
    lev_of = _box_levels(level_starts, ntb)
    per = 32 * rounds
    nit = (n + per - 1) // per
    it = np.repeat(np.arange(ntb), nit)
    j = _expand_ranges(np.zeros(ntb, dtype=np.int64), nit)
    c = np.minimum(per, n[it] - j * per)
    items = np.stack([np.asarray(target_boxes, dtype=np.int64)[it], f0[it] + j * per, c,
                      lev_of[it]], axis=1)
    order = np.argsort(-c, kind="stable")
    return np.ascontiguousarray(items[order], dtype=np.int32), src_index.astype(np.int32)


def _np_i32(a):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(a, dtype=np.int32)


class SumpyTreeIndependentDataForWrangler:
    """Code-side data of the wrangler (sumpy/fmm.py:99-252)."""

    def __init__(self, array_context, multipole_expansion_factory,
                 local_expansion_factory, target_kernels, exclude_self=False,
                 use_rscale=None, strength_usage=None, source_kernels=None):
        if len(target_kernels) != 1:
            raise NotImplementedError("exactly one target kernel is supported")
        if source_kernels is not None and list(source_kernels) != list(target_kernels):
            raise NotImplementedError("source kernels must equal the target kernel")
        if strength_usage is not None and list(strength_usage) != [0]:
            raise NotImplementedError("a single strength vector is supported")
        self._setup_actx = array_context
        self.multipole_expansion_factory = multipole_expansion_factory
        self.local_expansion_factory = local_expansion_factory
        self.target_kernels = list(target_kernels)
        self.source_kernels = source_kernels
        self.exclude_self = exclude_self
        self.use_rscale = use_rscale
        self.strength_usage = strength_usage
        self._mexp = {}
        self._lexp = {}

    def get_base_kernel(self):
        return self.target_kernels[0].get_base_kernel()

    def multipole_expansion(self, order):
        if order not in self._mexp:
            self._mexp[order] = (self.multipole_expansion_factory(order)
                                 if self.use_rscale is None else
                                 self.multipole_expansion_factory(order, use_rscale=self.use_rscale))
        return self._mexp[order]

    def local_expansion(self, order):
        if order not in self._lexp:
            self._lexp[order] = (self.local_expansion_factory(order)
                                 if self.use_rscale is None else
                                 self.local_expansion_factory(order, use_rscale=self.use_rscale))
        return self._lexp[order]


class SumpyExpansionWrangler:
    """B200 implementation of boxtree's ExpansionWranglerInterface with
    sumpy's constructor (sumpy/fmm.py:304-367)."""

    def __init__(self, tree_indep, traversal, dtype, fmm_level_to_order,
                 source_extra_kwargs=None, kernel_extra_kwargs=None,
                 self_extra_kwargs=None, translation_classes_data=None,
                 preprocessed_mpole_dtype=None, *, _disable_translation_classes=False,
                 precision="fp64", device=None, gradient=False, m2l_item_groups=None,
                 cuda_graph=False):
        if not callable(fmm_level_to_order):
            raise TypeError("fmm_level_to_order not passed")
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
        self.tree_indep = tree_indep
        self.traversal = traversal
        self.tree = traversal.tree
        self.dtype = np.dtype(dtype)
        self.precision = precision
        self.gradient = bool(gradient)
        self.source_extra_kwargs = source_extra_kwargs or {}
        self.kernel_extra_kwargs = kernel_extra_kwargs or {}
        self.self_extra_kwargs = self_extra_kwargs or {}
        self.device = torch.device(device if device is not None else "cuda")

        base_kernel = tree_indep.get_base_kernel()
        self.helmholtz = isinstance(base_kernel, HelmholtzKernel)
        if self.helmholtz:
            if np.dtype(dtype) != np.complex128:
                raise NotImplementedError("the 3D Helmholtz wrangler computes in complex128")
            if self.gradient:
                raise NotImplementedError("gradient outputs are implemented for Laplace only")
            self.k = helmholtz_k(base_kernel, self.kernel_extra_kwargs)
        elif np.dtype(dtype) != np.float64:
            raise NotImplementedError("the 3D Laplace wrangler computes in float64")
        self._tdtype = torch.complex128 if self.helmholtz else torch.float64
        kernel_arg_set = frozenset(self.kernel_extra_kwargs.items())
        self.level_orders = [fmm_level_to_order(base_kernel, kernel_arg_set, self.tree, lev)
                             for lev in range(self.tree.nlevels)]
        for o in self.level_orders:
            if not 0 <= o <= 16:
                raise ValueError(f"expansion order {o} outside [0, 16]")

        if _disable_translation_classes:
            raise NotImplementedError("M2L always uses translation classes on the B200 path")
        if translation_classes_data is None:
            from sumpy_b200.tree import TranslationClassesBuilder
            translation_classes_data, _ = TranslationClassesBuilder()(
                None, traversal, self.tree, is_translation_per_level=True)
        self.translation_classes_data = translation_classes_data
        self.supports_translation_classes = True

        self._devcache = {}
        self._m2l_plans = {}
        self._m2l_mats = {}
        self._m2l_tc_mats = {}
        self._m2l_ws = None
        self._status = torch.zeros(1, dtype=torch.int32, device=self.device)
        # drive_fmm runs List 1, 3 and 4 on a second stream (sumpy_b200.drive)
        self.concurrent_stages = True
        # one order on every level: M2M and L2L as eight dense maps per level
        # applied as grouped GEMMs. Laplace: both as FP64 GEMMs with K split
        # over CTAs on small levels (on the 1M-point benchmark the FP64 M2M,
        # 0.21 ms, beats the 3xTF32 tensor-core M2M, 0.29 ms, whose per-level
        # TF32 split adds a launch to the level-serial chain; the 3xTF32 L2L
        # also compounds its FP32 group sums down the levels: ~3x the mixed
        # form's error). Helmholtz mixed: M2M on the tensor cores.
        self.tc_m2m = self.helmholtz
        self.tc_l2l = False
        # operand format of the tensor-core GEMMs (mixed form): "f16" splits
        # every operand row into two f16 halves after scaling it by a power
        # of two (row max in [2^13, 2^14)), the scales undone in the FP64
        # epilogue; "tf32" splits into two TF32 values. Both keep ~22 bits
        # per operand with FP32 sums per class group; f16 runs at twice the
        # tensor rate with half the operand bytes.
        self.tc_format = "f16"
        self.gemm_l2l = True
        self.gemm_m2m = True
        # FP64 octant GEMMs of all levels in one persistent launch (a device
        # work queue in chain order with bounded per-level waits) instead of
        # one launch per level. Off: on the 1M-point workload the chained
        # launch takes M2M 0.46 ms and L2L 0.59 ms against 0.21 and 0.23 ms
        # for the per-level launches replayed from a CUDA graph (each level
        # waits for the whole previous one either way, and the persistent
        # CTAs add a queue round trip and L2-only source loads per unit)
        self.chain_levels = False
        # mixed List 3 / List 4: all levels in one launch over host-cut work
        # items (False: one launch per level, a warp per target box)
        self.item_kernels = True
        # P2M and L2P of all levels in one launch (one order on every level)
        self.merge_levels = True
        # Helmholtz L2P over packed items (False: one warp per box, all levels)
        self.packed_l2p = True
        # drive_fmm replays the whole evaluation from a CUDA graph (one host
        # call per evaluation instead of one per kernel launch)
        self.cuda_graph = bool(cuda_graph)
        self.m2l_item_groups = int(m2l_item_groups or M2L_ITEM_GROUPS)
        if self.m2l_item_groups < 1:
            raise ValueError("m2l_item_groups must be >= 1")
        # rounds (one source box / 32 sources each) per List-3 / List-4 item
        self.item_rounds = ITEM_ROUNDS
        # the octant (M2M / L2L) GEMMs of a level are cut into enough items
        # and K parts to cover the SMs this many times
        self.octant_split = 1

    SCHEDULE_KNOBS = ("m2l_item_groups", "item_rounds", "octant_split", "chain_levels",
                      "concurrent_stages")

    def set_schedule(self, **knobs):
        """Change schedule knobs (:attr:`SCHEDULE_KNOBS`); work plans are
        cached per knob value, and a captured CUDA graph of the evaluation is
        dropped so that the next call captures the new schedule."""
        for k, v in knobs.items():
            if k not in self.SCHEDULE_KNOBS:
                raise ValueError(f"unknown schedule knob {k!r}")
            if k in ("m2l_item_groups", "item_rounds", "octant_split") and int(v) < 1:
                raise ValueError(f"{k} must be >= 1")
            setattr(self, k, type(getattr(self, k))(v))
        self._graph_cache = None

    def schedule(self):
        return {k: getattr(self, k) for k in self.SCHEDULE_KNOBS}

    # {{{ geometry, storage

    def level_to_rscale(self, level):
        """sumpy/fmm.py:369-386: rscale = root_extent * 2^-level * 2 / order."""
        return self.tree.root_extent * (2 ** -level) * 2 / self.level_orders[level]

    @cached_property
    def tree_level_start_box_nrs(self):
        return np.asarray(self.tree.level_start_box_nrs, dtype=np.int64)

    def _expansions_level_starts(self, order_to_size):
        lsb = self.tree_level_start_box_nrs
        res = [0]
        for lev in range(self.tree.nlevels):
            res.append(res[-1] + order_to_size(self.level_orders[lev]) * int(lsb[lev + 1] - lsb[lev]))
        return res

    @cached_property
    def _mpole_level_starts(self):
        return self._expansions_level_starts(
            lambda o: len(self.tree_indep.multipole_expansion(o)))

    @cached_property
    def _local_level_starts(self):
        return self._expansions_level_starts(
            lambda o: len(self.tree_indep.local_expansion(o)))

    def multipole_expansions_level_starts(self):
        return self._mpole_level_starts

    def local_expansions_level_starts(self):
        return self._local_level_starts

    def multipole_expansion_zeros(self, actx=None):
        return torch.zeros(self._mpole_level_starts[-1], dtype=self._tdtype, device=self.device)

    def local_expansion_zeros(self, actx=None):
        return torch.zeros(self._local_level_starts[-1], dtype=self._tdtype, device=self.device)

    def output_zeros(self, actx=None):
        """Potential per target kernel; with ``gradient=True`` the potential
        and its three target-coordinate derivatives (rows of one (4, n)
        buffer, so the derivative rows form a contiguous [3][n] block)."""
        if self.gradient:
            buf = torch.zeros((4, self.tree.ntargets), dtype=torch.float64, device=self.device)
            return [buf[0], buf[1], buf[2], buf[3]]
        return [torch.zeros(self.tree.ntargets, dtype=self._tdtype, device=self.device)
                for _ in self.tree_indep.target_kernels]

    def _view(self, exps, level, starts):
        a, b = starts[level], starts[level + 1]
        lsb = self.tree_level_start_box_nrs
        nb = int(lsb[level + 1] - lsb[level])
        return int(lsb[level]), exps[a:b].view(nb, -1) if nb else exps[a:b]

    def multipole_expansions_view(self, mpole_exps, level):
        return self._view(mpole_exps, level, self._mpole_level_starts)

    def local_expansions_view(self, local_exps, level):
        return self._view(local_exps, level, self._local_level_starts)

    def _dev(self, arr, dtype=torch.int32):
        """Device copy of a host array (cached per array object and dtype)."""
        if isinstance(arr, torch.Tensor):
            if arr.device.type == "cuda":
                return arr if arr.dtype == dtype else arr.to(dtype)
            return arr.to(self.device, dtype)
        key = (id(arr), dtype)
        hit = self._devcache.get(key)
        if hit is not None and hit[0] is arr:
            return hit[1]
        t = torch.as_tensor(np.ascontiguousarray(arr)).to(self.device, dtype)
        self._devcache[key] = (arr, t)
        return t

    @cached_property
    def _geom(self):
        t = self.tree
        f64 = torch.float64
        g = {
            "centers": self._dev(t.box_centers, f64),
            "sources": self._dev(t.sources, f64),
            "targets": self._dev(t.targets, f64),
            "bss": self._dev(t.box_source_starts),
            "bsc": self._dev(t.box_source_counts_nonchild),
            "bts": self._dev(t.box_target_starts),
            "btc": self._dev(t.box_target_counts_nonchild),
            "child": self._dev(t.box_child_ids),
            "parent": self._dev(t.box_parent_ids),
            "tts": (self._dev(t.target_to_source)
                    if self.tree_indep.exclude_self else None),
        }
        if self.tree_indep.exclude_self and t.target_to_source is None:
            raise ValueError("exclude_self needs a tree whose sources are its targets")
        return g

    def set_positions(self, sources=None, targets=None):
        """Overwrite the device coordinates of the sources and/or targets in
        place ((3, n) float64 tensors in tree order). Every stage reads the
        coordinates from these buffers, and the work plans, operator tables
        and a captured CUDA graph depend only on the boxes, so they stay
        valid as long as each point stays inside the box it was sorted
        into; the caller checks that (see :mod:`sumpy_b200.autograd`)."""
        g = self._geom
        for key, new in (("sources", sources), ("targets", targets)):
            if new is None:
                continue
            if tuple(new.shape) != tuple(g[key].shape):
                raise ValueError(f"{key}: shape {tuple(new.shape)}, tree has "
                                 f"{tuple(g[key].shape)}")
            g[key].copy_(new)

    @property
    def _scale(self):
        return self.tree_indep.target_kernels[0].global_scaling_const

    # }}}

    def reorder_sources(self, source_array):
        idx = self._dev(self.tree.user_source_ids, torch.int64)
        return source_array[idx]

    def reorder_potentials(self, potentials):
        idx = self._dev(self.tree.sorted_target_ids, torch.int64)
        return [p[idx] for p in potentials]

    def distribute_source_weights(self, src_weight_vecs, src_idx_all_ranks=None):
        return src_weight_vecs

    def gather_potential_results(self, potentials, tgt_idx_all_ranks=None):
        return potentials

    def communicate_mpoles(self, actx, mpole_exps, return_stats=False):
        """Exchange of the upward pass's multipoles between ranks (boxtree's
        distributed hook, called by drive_fmm after coarsen_multipoles);
        nothing to exchange on one rank."""
        return None

    def finalize_potentials(self, actx, potentials):
        return potentials

    def _weights(self, src_weight_vecs):
        (w,) = src_weight_vecs
        if w.dtype != self._tdtype or not w.is_contiguous():
            w = w.to(self._tdtype).contiguous()
        return w

    def _entry(self, name):
        """C-ABI entry point name of a stage for this wrangler's kernel."""
        return name.replace("sumpy_", "sumpy_helmholtz_", 1) if self.helmholtz else name

    @property
    def _kargs(self):
        """The wave number argument of the Helmholtz entry points."""
        return [_d(self.k)] if self.helmholtz else []

    # {{{ stages

    def form_multipoles(self, actx, level_start_source_box_nrs, source_boxes, src_weight_vecs):
        mpoles = self.multipole_expansion_zeros(actx)
        g = self._geom
        w = self._weights(src_weight_vecs)
        st = stream_ptr()
        if self._merged_levels and not isinstance(source_boxes, torch.Tensor):
            def build():
                sb = np.asarray(source_boxes, dtype=np.int64)
                lev = _box_levels(level_start_source_box_nrs, len(sb))
                order = np.argsort(-np.asarray(self.tree.box_source_counts_nonchild)[sb],
                                   kind="stable")
                return (torch.as_tensor(sb[order].astype(np.int32)).to(self.device),
                        torch.as_tensor(lev[order].astype(np.int32)).to(self.device))
            boxes, levs = self._cached_items(
                "p2m_boxes", (level_start_source_box_nrs, source_boxes), build)
            if boxes.numel():
                call(self._entry("sumpy_p2e_from_single_box_levels_f64"),
                     _c(self.level_orders[0]), *self._kargs,
                     _i32(boxes.numel()), dptr(boxes), dptr(levs), dptr(self._level_rscales),
                     dptr(g["centers"]), _i64(self.tree.nboxes), dptr(g["bss"]), dptr(g["bsc"]),
                     dptr(g["sources"]), _i64(self.tree.nsources), dptr(w), dptr(mpoles), st)
            return mpoles
        lss = _np_i32(level_start_source_box_nrs)
        boxes = self._dev(source_boxes)
        for lev in range(self.tree.nlevels):
            a, b = int(lss[lev]), int(lss[lev + 1])
            if a == b:
                continue
            base, view = self.multipole_expansions_view(mpoles, lev)
            call(self._entry("sumpy_p2e_from_single_box_f64"), _c(self.level_orders[lev]),
                 _d(self.level_to_rscale(lev)), *self._kargs, _i32(b - a), dptr(boxes[a:b]),
                 dptr(g["centers"]), _i64(self.tree.nboxes), dptr(g["bss"]), dptr(g["bsc"]),
                 dptr(g["sources"]), _i64(self.tree.nsources), dptr(w), _i32(base),
                 dptr(view), st)
        return mpoles

    def coarsen_multipoles(self, actx, level_start_source_parent_box_nrs,
                           source_parent_boxes, mpoles):
        if self._tc_translations and self.tc_m2m:
            return self._coarsen_tc(level_start_source_parent_box_nrs, source_parent_boxes,
                                    mpoles)
        if self.gemm_m2m and self._gemm_fp64_ok:
            return self._coarsen_tc(level_start_source_parent_box_nrs, source_parent_boxes,
                                    mpoles, fp64=True)
        lsp = _np_i32(level_start_source_parent_box_nrs)
        boxes = self._dev(source_parent_boxes)
        g = self._geom
        st = stream_ptr()
        for src_lev in range(self.tree.nlevels - 1, 2, -1):
            tgt_lev = src_lev - 1
            a, b = int(lsp[tgt_lev]), int(lsp[tgt_lev + 1])
            if a == b:
                continue
            sbase, sview = self.multipole_expansions_view(mpoles, src_lev)
            tbase, tview = self.multipole_expansions_view(mpoles, tgt_lev)
            call(self._entry("sumpy_e2e_from_children_f64"), _c(self.level_orders[src_lev]),
                 _c(self.level_orders[tgt_lev]), _d(self.level_to_rscale(src_lev)),
                 _d(self.level_to_rscale(tgt_lev)), *self._kargs, _i32(b - a),
                 dptr(boxes[a:b]),
                 dptr(g["child"]), _i64(self.tree.nboxes), dptr(g["centers"]),
                 _i64(self.tree.nboxes), _i32(sbase), dptr(sview), _i32(tbase), dptr(tview), st)
        return mpoles

    def _cost_sorted_csr(self, target_boxes, starts, lists):
        """The List-1 CSR with its target boxes in decreasing order of
        pairs (targets x list sources): warps of similar length share a CTA
        and the longest start first. Results are per target, so the order
        does not change them."""
        def build():
            # on the device (the forest's lists are long)
            dev, i64 = self.device, torch.int64
            tb = torch.as_tensor(np.asarray(target_boxes, dtype=np.int64), device=dev)
            st = torch.as_tensor(np.asarray(starts, dtype=np.int64), device=dev)
            ls = torch.as_tensor(np.asarray(lists, dtype=np.int64), device=dev)
            nent = len(lists)
            cnt = st[1:] - st[:-1]
            bsc = self._dev(self.tree.box_source_counts_nonchild, i64)
            btc = self._dev(self.tree.box_target_counts_nonchild, i64)
            csum = torch.cat([torch.zeros(1, dtype=i64, device=dev), torch.cumsum(bsc[ls], 0)])
            pairs = btc[tb] * (csum[st[1:]] - csum[st[:-1]])
            order = torch.sort(-pairs, stable=True).indices
            ncnt = cnt[order]
            nst = torch.cat([torch.zeros(1, dtype=i64, device=dev), torch.cumsum(ncnt, 0)])
            # entries of each reordered row: its old start plus 0 .. count - 1
            row = torch.repeat_interleave(torch.arange(len(ncnt), device=dev), ncnt,
                                          output_size=nent)
            ent = st[:-1][order][row] + torch.arange(nent, device=dev) - nst[:-1][row]
            return tuple(a.to(torch.int32) for a in (tb[order], nst, ls[ent]))
        return self._cached_items(("p2p_sorted", id(lists)), (target_boxes, starts, lists),
                                  build)

    def eval_direct(self, actx, target_boxes, source_box_starts, source_box_lists,
                    src_weight_vecs):
        pot = self.output_zeros(actx)
        tb = self._dev(target_boxes)
        if tb.numel() == 0:
            return pot
        g = self._geom
        w = self._weights(src_weight_vecs)
        if not any(isinstance(a, torch.Tensor)
                   for a in (target_boxes, source_box_starts, source_box_lists)):
            tb, st_d, ls_d = self._cost_sorted_csr(target_boxes, source_box_starts,
                                                   source_box_lists)
        else:
            st_d, ls_d = self._dev(source_box_starts), self._dev(source_box_lists)
        args = (_i32(tb.numel()), dptr(tb), dptr(st_d), dptr(ls_d), dptr(g["bss"]), dptr(g["bsc"]),
                dptr(g["bts"]), dptr(g["btc"]), dptr(g["sources"]), _i64(self.tree.nsources),
                *self._kargs, dptr(w), dptr(g["targets"]), _i64(self.tree.ntargets),
                dptr(g["tts"]), _d(self._scale), dptr(pot[0]))
        mixed = self.precision == "mixed"
        if self.helmholtz:
            call("sumpy_helmholtz_p2p_from_csr_mixed" if mixed
                 else "sumpy_helmholtz_p2p_from_csr_f64", *args, stream_ptr())
            return pot
        if self.gradient:
            call("sumpy_p2p_from_csr_grad_mixed" if mixed else "sumpy_p2p_from_csr_grad_f64",
                 *args, dptr(pot[1]), stream_ptr())
        else:
            call("sumpy_p2p_from_csr_mixed" if mixed else "sumpy_p2p_from_csr_f64",
                 *args, stream_ptr())
        return pot

    # {{{ M2L

    def _m2l_matrices(self, lev):
        """Device tensor [nclasses, n, n] and the level's scalar factor."""
        order = self.level_orders[lev]
        kernel = self.tree_indep.get_base_kernel()
        rscale = self.level_to_rscale(lev)
        tc = self.translation_classes_data
        ls = tc.from_sep_siblings_translation_classes_level_starts
        vecs = tc.from_sep_siblings_translation_class_to_distance_vector[:, ls[lev]:ls[lev + 1]]
        if self.helmholtz:
            # complex operators per level, applied as their real embedding
            key = ("helmholtz", lev, order)
            if key not in self._m2l_mats:
                T = helmholtz_m2l_class_matrices(order, vecs, rscale, rscale, self.k)
                self._m2l_mats[key] = torch.as_tensor(real_embedding(T)).to(self.device)
            return self._m2l_mats[key], 1.0
        if is_scale_invariant(kernel):
            # rscale^|mi| d^mi (1/r) at d = v*h with rscale = 2h/p equals
            # (1/rscale) times the same derivatives at v*(h/rscale) with unit rscale
            h = self.tree.root_extent * 2.0 ** -lev
            key = (order, tuple(np.round(vecs[:, :].ravel() / h, 12)))
            if key not in self._m2l_mats:
                unit = m2l_class_matrices(order, vecs / rscale, 1.0, 1.0)
                self._m2l_mats[key] = torch.as_tensor(unit).to(self.device)
            return self._m2l_mats[key], 1.0 / rscale
        key = ("level", lev)
        if key not in self._m2l_mats:
            mats = m2l_class_matrices(order, vecs, rscale, rscale)
            self._m2l_mats[key] = torch.as_tensor(mats).to(self.device)
        return self._m2l_mats[key], 1.0

    def _m2l_plan(self, lev, tgt_boxes, starts, lists, tile=M2L_TILE):
        """Regroup one level's List-2 CSR into (tile, class) GEMM groups.

        Targets are ordered by their octant in the parent (then by box
        number), so a tile's targets share the same set of valid classes;
        target rank r goes to tile r // tile, slot r % tile, and the groups
        are the distinct (tile, class) pairs in increasing order. Built on
        the device (sorts, unique and scatters over the level's entries)."""
        key = (lev, id(lists), tile)
        if key in self._m2l_plans:
            return self._m2l_plans[key]
        tc = self.translation_classes_data
        cls_ls = tc.from_sep_siblings_translation_classes_level_starts
        c0 = int(cls_ls[lev])
        ncls = int(cls_ls[lev + 1]) - c0
        dev = self.device
        i64 = torch.int64
        starts_h = np.asarray(starts, dtype=np.int64)
        st = torch.as_tensor(starts_h, device=dev)
        tb = torch.as_tensor(np.asarray(tgt_boxes, dtype=np.int64), device=dev)
        counts = st[1:] - st[:-1]
        tpos = torch.nonzero(counts > 0).flatten()
        if tpos.numel() == 0:
            self._m2l_plans[key] = None
            return None
        coords = self._dev(self.tree.box_coords, i64)[:, tb[tpos]]
        octant = (coords[0] & 1) * 4 + (coords[1] & 1) * 2 + (coords[2] & 1)
        order = torch.sort(octant * (self.tree.nboxes + 1) + tb[tpos]).indices
        tpos = tpos[order]
        nt = tpos.numel()
        ntiles = (nt + tile - 1) // tile
        tile_targets = torch.full((ntiles * tile,), -1, dtype=torch.int32, device=dev)
        tile_targets[:nt] = tb[tpos].to(torch.int32)
        rank = torch.empty(tb.numel(), dtype=i64, device=dev)
        rank[tpos] = torch.arange(nt, dtype=i64, device=dev)
        e0, e1 = int(starts_h[0]), int(starts_h[-1])
        # (the output size is known on the host: no device round trip)
        ent_tgt = torch.repeat_interleave(torch.arange(tb.numel(), device=dev), counts,
                                          output_size=e1 - e0)
        ent_src = self._dev(lists, torch.int32)[e0:e1]
        ent_cls = self._dev(tc.from_sep_siblings_translation_classes, i64)[e0:e1] - c0
        if ent_cls.numel() and bool((ent_cls.min() < 0) | (ent_cls.max() >= ncls)):
            raise ValueError(f"translation class out of range on level {lev}")
        r = rank[ent_tgt]
        slot = r % tile
        gkey = (r // tile) * ncls + ent_cls
        uniq, inv = torch.unique(gkey, sorted=True, return_inverse=True)
        ngroups = uniq.numel()
        group_sources = torch.full((ngroups, tile), -1, dtype=torch.int32, device=dev)
        group_sources[inv, slot] = ent_src
        group_tile = uniq // ncls
        tile_group_starts = torch.searchsorted(
            group_tile, torch.arange(ntiles + 1, dtype=i64, device=dev)).to(torch.int32)
        plan = {
            "ntiles": ntiles,
            "ngroups": ngroups,
            "nentries": e1 - e0,
            "nclasses": ncls,
            "tile_targets": tile_targets,
            "tile_group_starts": tile_group_starts,
            "group_class": (uniq % ncls).to(torch.int32),
            "group_sources": group_sources.reshape(-1),
        }
        self._m2l_plans[key] = plan
        return plan

    def multipole_to_local(self, actx, level_start_target_box_nrs, target_boxes,
                           src_box_starts, src_box_lists, mpole_exps):
        local_exps = self.local_expansion_zeros(actx)
        ltb = _np_i32(level_start_target_box_nrs)
        tboxes = _np_i32(target_boxes)
        starts = np.asarray(src_box_starts if not isinstance(src_box_starts, torch.Tensor)
                            else src_box_starts.cpu().numpy())
        st = stream_ptr()
        levels = [lev for lev in range(self.tree.nlevels)
                  if ltb[lev] != ltb[lev + 1] and starts[ltb[lev]] != starts[ltb[lev + 1]]]
        tc = self.precision == "mixed"
        tile = M2L_TILE_TC if tc else M2L_TILE
        if len({self.level_orders[lev] for lev in levels}) == 1 \
                and len(set(self.level_orders)) == 1:
            # every level in one launch (uniform expansion size: the flat
            # level-major arrays are [nboxes][ncoeff])
            plan = self._m2l_merged_plan(tuple(levels), ltb, tboxes, starts, src_box_lists, tile)
            if plan is not None:
                if tc:
                    self._launch_m2l_tc_merged(plan, mpole_exps, local_exps, st)
                else:
                    self._call_m2l_f64(self.level_orders[0], plan, plan["mats"], 0, mpole_exps,
                                       0, local_exps, st)
            return local_exps
        for lev in levels:
            a, b = int(ltb[lev]), int(ltb[lev + 1])
            plan = self._m2l_plan(lev, tboxes[a:b], starts[a:b + 1], src_box_lists, tile)
            if plan is None:
                continue
            mats, mscale = self._m2l_matrices(lev)
            sbase, sview = self.multipole_expansions_view(mpole_exps, lev)
            tbase, tview = self.local_expansions_view(local_exps, lev)
            items = self._level_items(lev, plan, mscale)
            if tc:
                self._launch_m2l_tc_level(lev, items, mats, sbase, sview, tbase, tview, st)
            else:
                self._call_m2l_f64(self.level_orders[lev], items, mats, sbase, sview, tbase,
                                   tview, st)
        return local_exps

    def _tc_items(self, tiles, groups_per_item=None):
        """Split tiles (group ranges ``[(g0, g1), ...]`` or an ``(n, 2)``
        array) into work items of at most ``groups_per_item`` (default
        ``m2l_item_groups``) groups, in tile order, then longest first (stable:
        CTAs start roughly in launch order). The same schedule serves the FP64
        and the tensor-core GEMMs."""
        gpi = int(groups_per_item or self.m2l_item_groups)
        t = np.asarray(tiles, dtype=np.int64).reshape(-1, 2)
        g0, g1 = t[:, 0], t[:, 1]
        nit = np.maximum(g1 - g0 + gpi - 1, 0) // gpi
        it_tile = np.repeat(np.arange(len(t), dtype=np.int64), nit)
        j = _expand_ranges(np.zeros(len(t), dtype=np.int64), nit)
        it_g0 = g0[it_tile] + j * gpi
        it_g1 = np.minimum(g1[it_tile], it_g0 + gpi)
        order = np.argsort(-(it_g1 - it_g0), kind="stable")
        return (it_tile[order].astype(np.int32), it_g0[order].astype(np.int32),
                it_g1[order].astype(np.int32))

    def _m2l_merged_plan(self, levels, ltb, tboxes, starts, lists, tile):
        """One GEMM schedule over all M2L levels: the per-level (tile, class)
        groups concatenated, class ids offset into a stacked operator set,
        one scale per tile, work items over the groups."""
        key = ("merged", levels, id(lists), tile, self.m2l_item_groups)
        if key in self._m2l_plans:
            return self._m2l_plans[key]
        tt, tsc, gcl, gsrc, tiles = [], [], [], [], []
        mats_list, mats_index = [], {}
        ntiles = ngroups = 0
        dev = self.device
        for lev in levels:
            a, b = int(ltb[lev]), int(ltb[lev + 1])
            p = self._m2l_plan(lev, tboxes[a:b], starts[a:b + 1], lists, tile)
            if p is None:
                continue
            mats, mscale = self._m2l_matrices(lev)
            mkey = mats.data_ptr()
            if mkey not in mats_index:
                mats_index[mkey] = sum(m.shape[0] for m in mats_list)
                mats_list.append(mats)
            tgs = p["tile_group_starts"].cpu().numpy().astype(np.int64) + ngroups
            tiles.append(np.stack([tgs[:-1], tgs[1:]], axis=1))
            tt.append(p["tile_targets"])
            tsc.append(torch.full((p["ntiles"],), mscale, dtype=torch.float64, device=dev))
            gcl.append(p["group_class"] + mats_index[mkey])
            gsrc.append(p["group_sources"])
            ntiles += p["ntiles"]
            ngroups += p["ngroups"]
        if ntiles == 0:
            self._m2l_plans[key] = None
            return None
        it_tile, it_g0, it_g1 = self._tc_items(np.concatenate(tiles))
        mats = mats_list[0] if len(mats_list) == 1 else torch.cat(mats_list)
        plan = {
            "nitems": len(it_tile), "ntiles": ntiles, "ngroups": ngroups,
            "nclasses": int(mats.shape[0]), "mats": mats,
            "item_tile": torch.as_tensor(it_tile).to(dev),
            "item_g0": torch.as_tensor(it_g0).to(dev),
            "item_g1": torch.as_tensor(it_g1).to(dev),
            "tile_targets": torch.cat(tt),
            "tile_scale": torch.cat(tsc),
            "group_class": torch.cat(gcl).to(torch.int32),
            "group_sources": torch.cat(gsrc),
        }
        self._m2l_plans[key] = plan
        return plan

    def _level_items(self, lev, plan, mscale):
        """Work items of one level's plan (levels of different expansion sizes
        run one launch each)."""
        key = ("items", lev, id(plan), self.m2l_item_groups)
        if key not in self._m2l_plans:
            tgs = plan["tile_group_starts"].cpu().numpy().astype(np.int64)
            it_tile, it_g0, it_g1 = self._tc_items(np.stack([tgs[:-1], tgs[1:]], axis=1))
            dev = self.device
            self._m2l_plans[key] = dict(
                plan, nitems=len(it_tile), item_tile=torch.as_tensor(it_tile).to(dev),
                item_g0=torch.as_tensor(it_g0).to(dev), item_g1=torch.as_tensor(it_g1).to(dev),
                tile_scale=torch.full((plan["ntiles"],), mscale, dtype=torch.float64, device=dev))
        return self._m2l_plans[key]

    def _call_m2l_f64(self, order, plan, mats, sbase, src, tbase, tgt, st):
        call(self._entry("sumpy_m2l_translation_classes_f64"), _c(order), _i32(plan["nitems"]),
             dptr(plan["item_tile"]), dptr(plan["item_g0"]), dptr(plan["item_g1"]),
             _i32(M2L_TILE), dptr(plan["tile_targets"]), dptr(plan["tile_scale"]),
             dptr(plan["group_class"]), dptr(plan["group_sources"]), _i32(mats.shape[0]),
             dptr(mats), _i32(sbase), dptr(src), _i32(tbase), dptr(tgt), st)

    @property
    def _tc_f16(self):
        if self.tc_format not in ("f16", "tf32"):
            raise ValueError(f"tc_format must be 'f16' or 'tf32', got {self.tc_format!r}")
        return self.tc_format == "f16"

    @staticmethod
    def _tc_pads(n, f16=False):
        """Padded rows (MMA M) and K: K is a whole number of 128-byte rows
        (32 tf32 or 64 f16)."""
        kq = 64 if f16 else 32
        return (n + 127) // 128 * 128, (n + kq - 1) // kq * kq

    def _m2l_tc_operands(self, mats):
        """Split planes [nclasses][rows_pad][k_pad] of a class-operator set:
        (hi, lo, rows_pad, k_pad, row scales) -- f16 halves with a power-of-two
        scale per operator row ([nclasses][rows_pad], the inverse scales), or
        TF32 halves (row scales None)."""
        f16 = self._tc_f16
        key = (mats.data_ptr(), f16)
        hit = self._m2l_tc_mats.get(key)
        if hit is not None:
            return hit
        ncls, n, _ = mats.shape
        rp, kp = self._tc_pads(n, f16)
        if f16:
            hi = torch.empty((ncls, rp, kp), dtype=torch.float16, device=self.device)
            lo = torch.empty_like(hi)
            rinv = torch.empty((ncls, rp), dtype=torch.float32, device=self.device)
            call("sumpy_split_f16x2_rowscale", _i64(ncls), _i32(n), _i32(n), dptr(mats),
                 _i32(rp), _i32(kp), dptr(hi), dptr(lo), dptr(rinv), stream_ptr())
        else:
            hi = torch.empty((ncls, rp, kp), dtype=torch.float32, device=self.device)
            lo = torch.empty_like(hi)
            rinv = None
            call("sumpy_split_tf32x2", _i64(ncls), _i32(n), _i32(n), dptr(mats), _i32(rp),
                 _i32(kp), dptr(hi), dptr(lo), stream_ptr())
        self._m2l_tc_mats[key] = (hi, lo, rp, kp, rinv)
        return self._m2l_tc_mats[key]

    def _m2l_workspace(self, nrows, kp):
        """Split planes of the source multipoles, [nrows + 1][kp], and (f16)
        their row scales; the extra last row stays zero (it stands in for
        empty tile slots)."""
        f16 = self._tc_f16
        dt = torch.float16 if f16 else torch.float32
        need = (nrows + 1) * kp
        ws = self._m2l_ws
        if ws is None or ws[0].dtype != dt or ws[0].numel() < need or ws[2].numel() < nrows + 1:
            rows = max(nrows, self.tree.nboxes) + 1
            self._m2l_ws = (torch.empty(rows * kp, dtype=dt, device=self.device),
                            torch.empty(rows * kp, dtype=dt, device=self.device),
                            torch.empty(rows, dtype=torch.float32, device=self.device))
        hi, lo, rinv = self._m2l_ws
        zero = slice(nrows * kp, (nrows + 1) * kp)
        hi[zero].zero_()
        lo[zero].zero_()
        rinv[nrows:nrows + 1].zero_()
        return hi, lo, rinv

    def _split_sources(self, nb, n, src, kp, ws, st):
        """M2L pre-processing: every source expansion (row = box) as split planes."""
        hi, lo, rinv = ws
        if self._tc_f16:
            call("sumpy_split_f16x2_rowscale", _i64(nb), _i32(1), _i32(n), dptr(src), _i32(1),
                 _i32(kp), dptr(hi), dptr(lo), dptr(rinv), st)
        else:
            call("sumpy_split_tf32x2", _i64(nb), _i32(1), _i32(n), dptr(src), _i32(1),
                 _i32(kp), dptr(hi), dptr(lo), st)

    def _launch_m2l_tc_merged(self, plan, mpole_exps, local_exps, st):
        ops = self._m2l_tc_operands(plan["mats"])
        n = plan["mats"].shape[1]
        nb = self.tree.nboxes
        ws = self._m2l_workspace(nb, ops[3])
        self._split_sources(nb, n, mpole_exps, ops[3], ws, st)
        self._call_m2l_tc(self.level_orders[0], plan, ops, nb + 1, 0, ws, 0, local_exps, st)

    def _call_m2l_tc(self, order, plan, ops, src_nrows, sbase, ws, tbase, tgt, st):
        hi, lo, rp, kp, rinv = ops
        ws_hi, ws_lo, ws_rinv = ws
        head = [_c(order), _i32(plan["nitems"]),
                dptr(plan["item_tile"]), dptr(plan["item_g0"]), dptr(plan["item_g1"]),
                _i32(M2L_TILE_TC), dptr(plan["tile_targets"]), dptr(plan["tile_scale"]),
                dptr(plan["group_class"]), dptr(plan["group_sources"]), _i32(plan["nclasses"])]
        tail = [_i32(tbase), dptr(tgt), dptr(self._status), st]
        if self._tc_f16:
            call(self._entry("sumpy_m2l_translation_classes_f16x3"), *head,
                 dptr(hi), dptr(lo), dptr(rinv), _i32(rp), _i32(kp), _i32(src_nrows),
                 _i32(sbase), dptr(ws_hi), dptr(ws_lo), dptr(ws_rinv), *tail)
        else:
            call(self._entry("sumpy_m2l_translation_classes_tf32x3"), *head,
                 dptr(hi), dptr(lo), _i32(rp), _i32(kp), _i32(src_nrows), _i32(sbase),
                 dptr(ws_hi), dptr(ws_lo), *tail)

    def _launch_m2l_tc_level(self, lev, items, mats, sbase, sview, tbase, tview, st):
        ops = self._m2l_tc_operands(mats)
        nb, n = sview.shape[0], mats.shape[1]   # real values per box
        ws = self._m2l_workspace(nb, ops[3])
        self._split_sources(nb, n, sview, ops[3], ws, st)
        self._call_m2l_tc(self.level_orders[lev], items, ops, nb + 1, sbase, ws, tbase, tview,
                          st)

    # {{{ M2M / L2L as per-octant GEMMs on the tensor cores (mixed form)

    @cached_property
    def _tc_translations(self):
        """Mixed form with one order on every level: M2M (and optionally L2L)
        as eight dense maps per level (one per child octant), applied as
        grouped GEMMs by the tensor-core kernel. For Laplace the maps are the
        same on every level (rscale ratio 1/2 and offset/rscale = order/8 do
        not depend on it); for Helmholtz they depend on the level through
        k^2 rscale^2 and act on the interleaved complex coefficients as their
        block-diagonal real embedding."""
        return self.precision == "mixed" and len(set(self.level_orders)) == 1

    def _octant_operator_planes(self, kind, parent_level=2):
        # Laplace: any level pair gives the same maps (take levels 2 -> 3)
        lev = parent_level if self.helmholtz else 2
        key = ("octant-ops", kind, lev, self._tc_f16)
        if key not in self._m2l_tc_mats:
            order = self.level_orders[0]
            # rscale as level_to_rscale (sumpy/fmm.py:369-386)
            r_par = self.tree.root_extent * 2.0 ** -lev * 2 / order
            r_ch = self.tree.root_extent * 2.0 ** -(lev + 1) * 2 / order
            h_ch = self.tree.root_extent * 2.0 ** -(lev + 1)
            offs = octant_offsets(h_ch)          # child center - parent center
            k2 = self.k ** 2 if self.helmholtz else 0.0
            if kind == "m2m":
                ops = [m2m_operator(order, r_ch, r_par, -offs[o], k2 * r_par ** 2)
                       for o in range(8)]
            else:
                ops = [l2l_operator(order, r_par, r_ch, offs[o], k2 * r_par ** 2)
                       for o in range(8)]
            ops = np.stack(ops)
            if self.helmholtz:
                # real maps on interleaved (re, im): rows/cols 2t + a, a in {0, 1}
                n = ops.shape[1]
                emb = np.zeros((8, n, 2, n, 2))
                emb[:, :, 0, :, 0] = ops
                emb[:, :, 1, :, 1] = ops
                ops = emb.reshape(8, 2 * n, 2 * n)
            mats = torch.as_tensor(ops).to(self.device)
            self._m2l_tc_mats[key] = (mats,) + self._m2l_tc_operands(mats)
        return self._m2l_tc_mats[key]

    def _octants(self, boxes):
        c = self.tree.box_coords[:, boxes]
        return ((c[0] & 1) * 4 + (c[1] & 1) * 2 + (c[2] & 1)).astype(np.int32)

    def _octant_plan(self, key, targets, sources, tw=M2L_TILE_TC):
        """GEMM schedule for per-octant maps: ``targets`` (box ids) in tiles of
        ``tw`` (128 for the tensor cores, 64 for the FP64 GEMM), one group per
        octant present in a tile, ``sources[o][i]`` the source box of target i
        for octant o (-1 = none)."""
        if key in self._m2l_plans:
            return self._m2l_plans[key]
        nt = len(targets)
        ntiles = (nt + tw - 1) // tw
        tile_targets = np.full(ntiles * tw, -1, dtype=np.int32)
        tile_targets[:nt] = targets
        src = np.full((8, ntiles * tw), -1, dtype=np.int32)
        src[:, :nt] = sources
        # one group per (tile, octant) with a source, tile-major
        blk = src.reshape(8, ntiles, tw)
        present = (blk >= 0).any(axis=2)                        # [8, ntiles]
        tile_of, oct_of = np.nonzero(present.T)                 # tile-major order
        groups = blk[oct_of, tile_of]                           # [ngroups, tw]
        classes = oct_of.astype(np.int32)
        gcount = present.sum(axis=0)
        gend = np.cumsum(gcount)
        tiles = list(zip((gend - gcount).tolist(), gend.tolist()))
        # a level's octant GEMM is on the level-serial M2M / L2L chain: cut
        # it into enough items (CTAs) to cover the GPU twice, down to one
        # octant group per item, so few tiles do not leave one CTA pipelining
        # all eight groups
        gpi = min(8, max(1, -(-len(groups) // (self.octant_split * self._sm_count))))
        it_tile, it_g0, it_g1 = self._tc_items(tiles, gpi)
        dev = self.device
        plan = {
            "nitems": len(it_tile), "nclasses": 8,
            "item_tile": torch.as_tensor(it_tile).to(dev),
            "item_g0": torch.as_tensor(it_g0).to(dev),
            "item_g1": torch.as_tensor(it_g1).to(dev),
            "tile_targets": torch.as_tensor(tile_targets).to(dev),
            "tile_scale": torch.ones(ntiles, dtype=torch.float64, device=dev),
            "group_class": torch.as_tensor(classes).to(dev),
            "group_sources": torch.as_tensor(
                np.ascontiguousarray(groups, dtype=np.int32).ravel()).to(dev),
        }
        self._m2l_plans[key] = plan
        return plan

    def _octant_gemm(self, kind, plan, sview, sbase, tview, tbase, st, fp64=False,
                     parent_level=2):
        mats, hi, lo, rp, kp, rinv = self._octant_operator_planes(kind, parent_level)
        n = mats.shape[1]   # real values per box

        def k_split(row_tiles, nkc, cap):
            # a level's octant GEMM is on the level-serial chain: few items
            # also split K (partial sums meet in the FP64 atomic epilogue)
            want = -(-self.octant_split * self._sm_count // max(1, plan["nitems"] * row_tiles))
            return int(max(1, min(nkc, cap, want)))

        if fp64:
            ks = k_split(1 if n <= 64 else -(-n // 128), -(-n // 8), 8)
            call("sumpy_class_gemm_f64", _i32(n), _i32(ks), _i32(plan["nitems"]),
                 dptr(plan["item_tile"]), dptr(plan["item_g0"]), dptr(plan["item_g1"]),
                 _i32(M2L_TILE), dptr(plan["tile_targets"]), dptr(plan["tile_scale"]),
                 dptr(plan["group_class"]), dptr(plan["group_sources"]), _i32(mats.shape[0]),
                 dptr(mats), _i32(sbase), dptr(sview), _i32(tbase), dptr(tview), st)
            return
        nb = sview.shape[0]
        ws = self._m2l_workspace(nb, kp)
        self._split_sources(nb, n, sview, kp, ws, st)
        f16 = self._tc_f16
        ks = k_split(rp // 128, kp // (64 if f16 else 32), 4)
        head = [_i32(n), _i32(ks), _i32(plan["nitems"]),
                dptr(plan["item_tile"]), dptr(plan["item_g0"]), dptr(plan["item_g1"]),
                _i32(M2L_TILE_TC), dptr(plan["tile_targets"]), dptr(plan["tile_scale"]),
                dptr(plan["group_class"]), dptr(plan["group_sources"]), _i32(plan["nclasses"])]
        tail = [_i32(tbase), dptr(tview), dptr(self._status), st]
        if f16:
            call("sumpy_class_gemm_f16x3", *head, dptr(hi), dptr(lo), dptr(rinv), _i32(rp),
                 _i32(kp), _i32(nb + 1), _i32(sbase), dptr(ws[0]), dptr(ws[1]), dptr(ws[2]),
                 *tail)
        else:
            call("sumpy_class_gemm_tf32x3", *head, dptr(hi), dptr(lo), _i32(rp), _i32(kp),
                 _i32(nb + 1), _i32(sbase), dptr(ws[0]), dptr(ws[1]), *tail)

    @property
    def _gemm_fp64_ok(self):
        """M2M / L2L as FP64 octant GEMMs: Laplace, one order on every level."""
        return not self.helmholtz and len(set(self.level_orders)) == 1

    def _coarsen_tc(self, level_start_source_parent_box_nrs, source_parent_boxes, mpoles,
                    fp64=False):
        lsp = _np_i32(level_start_source_parent_box_nrs)
        parents_all = _np_i32(source_parent_boxes)
        child = np.asarray(self.tree.box_child_ids)
        st = stream_ptr()
        chain = []
        for src_lev in range(self.tree.nlevels - 1, 2, -1):
            tgt_lev = src_lev - 1
            a, b = int(lsp[tgt_lev]), int(lsp[tgt_lev + 1])
            if a == b:
                continue
            key = ("m2m-plan", tgt_lev, id(source_parent_boxes), fp64, self.octant_split)
            if key not in self._m2l_plans:
                parents = parents_all[a:b]
                kids = child[:, parents]                       # [slot][parent]
                srcs = np.full((8, len(parents)), -1, dtype=np.int32)
                for slot in range(kids.shape[0]):
                    ch = kids[slot]
                    has = ch > 0
                    oc = self._octants(ch[has])
                    srcs[oc, np.nonzero(has)[0]] = ch[has]
                self._octant_plan(key, parents, srcs, M2L_TILE if fp64 else M2L_TILE_TC)
            plan = self._m2l_plans[key]
            if fp64 and self.chain_levels:
                chain.append(plan)
                continue
            sbase, sview = self.multipole_expansions_view(mpoles, src_lev)
            tbase, tview = self.multipole_expansions_view(mpoles, tgt_lev)
            self._octant_gemm("m2m", plan, sview, sbase, tview, tbase, st, fp64=fp64,
                              parent_level=tgt_lev)
        if chain:
            self._octant_chain("m2m", chain, mpoles, st)
        return mpoles

    def _refine_tc(self, level_start_target_or_target_parent_box_nrs,
                   target_or_target_parent_boxes, local_exps, fp64=False):
        lt = _np_i32(level_start_target_or_target_parent_box_nrs)
        boxes_all = _np_i32(target_or_target_parent_boxes)
        parent = np.asarray(self.tree.box_parent_ids)
        st = stream_ptr()
        chain = []
        for tgt_lev in range(1, self.tree.nlevels):
            a, b = int(lt[tgt_lev]), int(lt[tgt_lev + 1])
            if a == b:
                continue
            key = ("l2l-plan", tgt_lev, id(target_or_target_parent_boxes), fp64,
                   self.octant_split)
            if key not in self._m2l_plans:
                kids = boxes_all[a:b]
                oc = self._octants(kids)
                order = np.argsort(oc, kind="stable")   # octant-pure tiles
                kids, oc = kids[order], oc[order]
                srcs = np.full((8, len(kids)), -1, dtype=np.int32)
                srcs[oc, np.arange(len(kids))] = parent[kids]
                self._octant_plan(key, kids, srcs, M2L_TILE if fp64 else M2L_TILE_TC)
            plan = self._m2l_plans[key]
            if fp64 and self.chain_levels:
                chain.append(plan)
                continue
            src_lev = tgt_lev - 1
            sbase, sview = self.local_expansions_view(local_exps, src_lev)
            tbase, tview = self.local_expansions_view(local_exps, tgt_lev)
            self._octant_gemm("l2l", plan, sview, sbase, tview, tbase, st, fp64=fp64,
                              parent_level=src_lev)
        if chain:
            self._octant_chain("l2l", chain, local_exps, st)
        return local_exps

    # }}}

    def _octant_chain(self, kind, plans, expansions, st):
        """The FP64 octant GEMMs of several levels (``plans`` in chain order:
        each level's sources are the previous level's targets) as one
        persistent launch of ``sumpy_class_gemm_chain_f64``. Same work items
        and K splits as the level-by-level launches; the expansions of all
        levels are rows of one flat [nboxes][n] array."""
        mats = self._octant_operator_planes(kind)[0]
        n = mats.shape[1]
        key = ("chain", kind, tuple(id(p) for p in plans))
        ch = self._m2l_plans.get(key)
        if ch is None:
            dev = self.device
            row_tiles = 1 if n <= 64 else -(-n // 128)
            nkc = -(-n // 8)
            it_t, it_a, it_b, tt, tsc, gcl, gsrc = [], [], [], [], [], [], []
            unit_start, item_start, ksplit = [0], [], []
            ntiles = ngroups = nitems = 0
            for p in plans:
                want = -(-self.octant_split * self._sm_count // max(1, p["nitems"] * row_tiles))
                ks = int(max(1, min(nkc, 8, want)))
                it_t.append(p["item_tile"] + ntiles)
                it_a.append(p["item_g0"] + ngroups)
                it_b.append(p["item_g1"] + ngroups)
                tt.append(p["tile_targets"])
                tsc.append(p["tile_scale"])
                gcl.append(p["group_class"])
                gsrc.append(p["group_sources"])
                item_start.append(nitems)
                ksplit.append(ks)
                unit_start.append(unit_start[-1] + p["nitems"] * row_tiles * ks)
                nitems += p["nitems"]
                ntiles += p["tile_scale"].numel()
                ngroups += p["group_class"].numel()

            def i32(x):
                return torch.as_tensor(np.asarray(x, dtype=np.int32)).to(dev)

            ch = {
                "nsteps": len(plans), "total": unit_start[-1],
                "unit_start": i32(unit_start), "item_start": i32(item_start),
                "ksplit": i32(ksplit),
                "item_tile": torch.cat(it_t).to(torch.int32),
                "item_g0": torch.cat(it_a).to(torch.int32),
                "item_g1": torch.cat(it_b).to(torch.int32),
                "tile_targets": torch.cat(tt), "tile_scale": torch.cat(tsc),
                "group_class": torch.cat(gcl), "group_sources": torch.cat(gsrc),
                "queue": torch.zeros(1 + len(plans), dtype=torch.int32, device=dev),
            }
            self._m2l_plans[key] = ch
        call("sumpy_class_gemm_chain_f64", _i32(n), _i32(ch["nsteps"]), dptr(ch["unit_start"]),
             dptr(ch["item_start"]), dptr(ch["ksplit"]), _i32(ch["total"]),
             dptr(ch["item_tile"]), dptr(ch["item_g0"]), dptr(ch["item_g1"]), _i32(M2L_TILE),
             dptr(ch["tile_targets"]), dptr(ch["tile_scale"]), dptr(ch["group_class"]),
             dptr(ch["group_sources"]), dptr(mats), dptr(expansions), dptr(ch["queue"]),
             dptr(self._status), st)

    def check_status(self):
        """Raise if a kernel reported an internal error (synchronises); the
        status is cleared, so the next evaluation starts clean."""
        code = int(self._status.item())
        if code:
            self._status.zero_()
            what = {1: "a tensor-core barrier wait", 2: "a level-chain wait"}.get(code, "a wait")
            raise RuntimeError(f"{what} expired in a kernel (status {code})")

    # }}}

    @cached_property
    def _sm_count(self):
        return torch.cuda.get_device_properties(self.device).multi_processor_count

    @property
    def _merged_levels(self):
        return self.merge_levels and len(set(self.level_orders)) == 1

    @property
    def _items_path(self):
        """List 3 / List 4 through the one-launch item kernels (Laplace mixed:
        FP32 arithmetic on FP64 offsets; Laplace FP64 and Helmholtz: FP64
        arithmetic); needs one order on every level (flat [nboxes][ncoeff]
        storage)."""
        return self.item_kernels and len(set(self.level_orders)) == 1

    @cached_property
    def _level_rscales(self):
        return torch.tensor([self.level_to_rscale(lev) if self.level_orders[lev] else 1.0
                             for lev in range(self.tree.nlevels)],
                            dtype=torch.float64, device=self.device)

    @property
    def _m2p_f32(self):
        """Laplace mixed form: the M2P items read an FP32 copy of the
        multipoles (lane groups of at least 32 / M2P_ITEM_GROUPS lanes)."""
        return self.precision == "mixed" and not self.helmholtz

    def _cached_items(self, key, objs, build):
        hit = self._devcache.get(key)
        if hit is not None and all(a is b for a, b in zip(hit[0], objs)):
            return hit[1]
        val = build()
        self._devcache[key] = (objs, val)
        return val

    def _eval_multipoles_items(self, target_boxes_by_source_level, source_boxes_by_level,
                               mpole_exps, pot):
        def build():
            items, lists = m2p_items(self.tree, target_boxes_by_source_level,
                                     source_boxes_by_level, rounds=self.item_rounds,
                                     groups=M2P_ITEM_GROUPS if self._m2p_f32 else 32)
            return (torch.as_tensor(items).to(self.device),
                    torch.as_tensor(lists).to(self.device))
        items, lists = self._cached_items(
            ("m2p_items", self.item_rounds),
            (target_boxes_by_source_level, source_boxes_by_level), build)
        if items.shape[0] == 0:
            return pot
        order = self.level_orders[0]
        g = self._geom
        st = stream_ptr()
        if self.helmholtz:
            call("sumpy_helmholtz_e2p_from_items_f64", _c(order), _d(self.k),
                 _i32(items.shape[0]), dptr(items), dptr(self._level_rscales), dptr(lists),
                 dptr(g["centers"]), _i64(self.tree.nboxes), dptr(mpole_exps),
                 dptr(g["targets"]), _i64(self.tree.ntargets), _d(self._scale), dptr(pot[0]), st)
            return pot
        if not self._m2p_f32:
            args = (_c(order), _i32(items.shape[0]), dptr(items), dptr(self._level_rscales),
                    dptr(lists), dptr(g["centers"]), _i64(self.tree.nboxes), dptr(mpole_exps),
                    dptr(g["targets"]), _i64(self.tree.ntargets), _d(self._scale), dptr(pot[0]))
            if self.gradient:
                call("sumpy_e2p_from_items_grad_f64", *args, dptr(pot[1]), st)
            else:
                call("sumpy_e2p_from_items_f64", *args, st)
            return pot
        mp32 = torch.empty(self.tree.nboxes * _npad(order), dtype=torch.float32,
                           device=self.device)
        call("sumpy_mpoles_to_f32", _c(order), _i64(self.tree.nboxes), dptr(mpole_exps),
             dptr(mp32), st)
        args = (_c(order), _i32(items.shape[0]), dptr(items), dptr(self._level_rscales),
                dptr(lists), dptr(g["centers"]), _i64(self.tree.nboxes), dptr(mp32),
                dptr(g["targets"]), _i64(self.tree.ntargets), _d(self._scale), dptr(pot[0]))
        if self.gradient:
            call("sumpy_e2p_from_items_grad_mixed", *args, dptr(pot[1]), st)
        else:
            call("sumpy_e2p_from_items_mixed", *args, st)
        return pot

    def eval_multipoles(self, actx, target_boxes_by_source_level, source_boxes_by_level,
                        mpole_exps):
        pot = self.output_zeros(actx)
        if self._items_path:
            return self._eval_multipoles_items(target_boxes_by_source_level,
                                               source_boxes_by_level, mpole_exps, pot)
        g = self._geom
        st = stream_ptr()
        for lev, ssn in enumerate(source_boxes_by_level):
            tb = target_boxes_by_source_level[lev]
            if len(tb) == 0:
                continue
            sbase, sview = self.multipole_expansions_view(mpole_exps, lev)
            tbd = self._dev(tb)
            args = (_c(self.level_orders[lev]), _d(self.level_to_rscale(lev)), *self._kargs,
                    _i32(tbd.numel()), dptr(tbd), dptr(self._dev(ssn.starts)),
                    dptr(self._dev(ssn.lists)), dptr(g["centers"]), _i64(self.tree.nboxes),
                    _i32(sbase), dptr(sview), dptr(g["bts"]), dptr(g["btc"]),
                    dptr(g["targets"]), _i64(self.tree.ntargets), _d(self._scale),
                    dptr(pot[0]))
            if self.gradient:
                call("sumpy_e2p_from_csr_grad_f64", *args, dptr(pot[1]), st)
            elif self.precision == "mixed" and not self.helmholtz:
                call("sumpy_e2p_from_csr_mixed", *args, st)
            else:
                call(self._entry("sumpy_e2p_from_csr_f64"), *args, st)
        return pot

    def form_locals(self, actx, level_start_target_or_target_parent_box_nrs,
                    target_or_target_parent_boxes, starts, lists, src_weight_vecs):
        local_exps = self.local_expansion_zeros(actx)
        if self._items_path and not isinstance(starts, torch.Tensor) \
                and not isinstance(lists, torch.Tensor):
            def build():
                items, sidx = p2l_items(self.tree, level_start_target_or_target_parent_box_nrs,
                                        target_or_target_parent_boxes, starts, lists,
                                        rounds=self.item_rounds)
                return (torch.as_tensor(items).to(self.device),
                        torch.as_tensor(sidx).to(self.device))
            items, sidx = self._cached_items(
                ("p2l_items", self.item_rounds), (level_start_target_or_target_parent_box_nrs,
                              target_or_target_parent_boxes, starts, lists), build)
            if items.shape[0]:
                g = self._geom
                w = self._weights(src_weight_vecs)
                name = ("sumpy_helmholtz_p2e_from_items_f64" if self.helmholtz
                        else "sumpy_p2e_from_items_mixed" if self.precision == "mixed"
                        else "sumpy_p2e_from_items_f64")
                call(name, _c(self.level_orders[0]), *self._kargs,
                     _i32(items.shape[0]), dptr(items), dptr(self._level_rscales), dptr(sidx),
                     dptr(g["centers"]), _i64(self.tree.nboxes), dptr(g["sources"]),
                     _i64(self.tree.nsources), dptr(w), dptr(local_exps), stream_ptr())
            return local_exps
        lt = _np_i32(level_start_target_or_target_parent_box_nrs)
        starts_h = np.asarray(starts if not isinstance(starts, torch.Tensor)
                              else starts.cpu().numpy())
        boxes = self._dev(target_or_target_parent_boxes)
        starts_d = self._dev(starts)
        lists_d = self._dev(lists)
        g = self._geom
        w = self._weights(src_weight_vecs)
        st = stream_ptr()
        for lev in range(self.tree.nlevels):
            a, b = int(lt[lev]), int(lt[lev + 1])
            if a == b or starts_h[a] == starts_h[b]:
                continue
            tbase, tview = self.local_expansions_view(local_exps, lev)
            name = ("sumpy_p2e_from_csr_mixed" if self.precision == "mixed" and not self.helmholtz
                    else self._entry("sumpy_p2e_from_csr_f64"))
            call(name, _c(self.level_orders[lev]),
                 _d(self.level_to_rscale(lev)), *self._kargs, _i32(b - a), dptr(boxes[a:b]),
                 dptr(starts_d[a:b + 1]), dptr(lists_d), dptr(g["centers"]),
                 _i64(self.tree.nboxes), dptr(g["bss"]), dptr(g["bsc"]), dptr(g["sources"]),
                 _i64(self.tree.nsources), dptr(w), _i32(tbase), dptr(tview), st)
        return local_exps

    def refine_locals(self, actx, level_start_target_or_target_parent_box_nrs,
                      target_or_target_parent_boxes, local_exps):
        tc = self._tc_translations and self.tc_l2l
        if tc or (self.gemm_l2l and self._gemm_fp64_ok):
            return self._refine_tc(level_start_target_or_target_parent_box_nrs,
                                   target_or_target_parent_boxes, local_exps, fp64=not tc)
        lt = _np_i32(level_start_target_or_target_parent_box_nrs)
        boxes = self._dev(target_or_target_parent_boxes)
        g = self._geom
        st = stream_ptr()
        for tgt_lev in range(1, self.tree.nlevels):
            a, b = int(lt[tgt_lev]), int(lt[tgt_lev + 1])
            if a == b:
                continue
            src_lev = tgt_lev - 1
            sbase, sview = self.local_expansions_view(local_exps, src_lev)
            tbase, tview = self.local_expansions_view(local_exps, tgt_lev)
            call(self._entry("sumpy_e2e_from_parent_f64"), _c(self.level_orders[src_lev]),
                 _c(self.level_orders[tgt_lev]), _d(self.level_to_rscale(src_lev)),
                 _d(self.level_to_rscale(tgt_lev)), *self._kargs, _i32(b - a),
                 dptr(boxes[a:b]),
                 dptr(g["parent"]), dptr(g["centers"]), _i64(self.tree.nboxes),
                 _i32(sbase), dptr(sview), _i32(tbase), dptr(tview), st)
        return local_exps

    def eval_locals(self, actx, level_start_target_box_nrs, target_boxes, local_exps):
        pot = self.output_zeros(actx)
        g = self._geom
        st = stream_ptr()
        if self._merged_levels and self.helmholtz and self.packed_l2p \
                and not isinstance(target_boxes, torch.Tensor):
            def build_hp():
                items, slots = l2p_items(self.tree, level_start_target_box_nrs, target_boxes,
                                         max_slots=HL2P_ITEM_SLOTS)
                return (torch.as_tensor(items).to(self.device),
                        torch.as_tensor(slots).to(self.device))
            items, slots = self._cached_items(
                "hl2p_items", (level_start_target_box_nrs, target_boxes), build_hp)
            if items.shape[0]:
                call("sumpy_helmholtz_e2p_from_single_box_packed_f64", _c(self.level_orders[0]),
                     _d(self.k), _i32(items.shape[0]), dptr(items), dptr(slots),
                     dptr(self._level_rscales), dptr(g["centers"]), _i64(self.tree.nboxes),
                     dptr(local_exps), dptr(g["targets"]), _i64(self.tree.ntargets),
                     _d(self._scale), dptr(pot[0]), st)
            return pot
        if self._merged_levels and self.helmholtz and not isinstance(target_boxes, torch.Tensor):
            def build_h():
                tb = np.asarray(target_boxes, dtype=np.int64)
                lev = _box_levels(level_start_target_box_nrs, len(tb))
                order = np.argsort(-np.asarray(self.tree.box_target_counts_nonchild)[tb],
                                   kind="stable")
                return (torch.as_tensor(tb[order].astype(np.int32)).to(self.device),
                        torch.as_tensor(lev[order].astype(np.int32)).to(self.device))
            boxes, levs = self._cached_items(
                "hl2p_boxes", (level_start_target_box_nrs, target_boxes), build_h)
            if boxes.numel():
                call("sumpy_helmholtz_e2p_from_single_box_levels_f64", _c(self.level_orders[0]),
                     _d(self.k), _i32(boxes.numel()), dptr(boxes), dptr(levs),
                     dptr(self._level_rscales), dptr(g["centers"]), _i64(self.tree.nboxes),
                     dptr(local_exps), dptr(g["bts"]), dptr(g["btc"]), dptr(g["targets"]),
                     _i64(self.tree.ntargets), _d(self._scale), dptr(pot[0]), st)
            return pot
        if self._merged_levels and not isinstance(target_boxes, torch.Tensor):
            def build():
                items, slots = l2p_items(self.tree, level_start_target_box_nrs, target_boxes,
                                         max_slots=L2P_ITEM_SLOTS)
                return (torch.as_tensor(items).to(self.device),
                        torch.as_tensor(slots).to(self.device))
            items, slots = self._cached_items(
                "l2p_items", (level_start_target_box_nrs, target_boxes), build)
            if items.shape[0]:
                args = (_c(self.level_orders[0]), _i32(items.shape[0]), dptr(items),
                        dptr(slots), dptr(self._level_rscales), dptr(g["centers"]),
                        _i64(self.tree.nboxes), dptr(local_exps), dptr(g["targets"]),
                        _i64(self.tree.ntargets), _d(self._scale), dptr(pot[0]))
                if self.gradient:
                    call("sumpy_e2p_from_single_box_packed_grad_f64", *args, dptr(pot[1]), st)
                else:
                    call("sumpy_e2p_from_single_box_packed_f64", *args, st)
            return pot
        ltb = _np_i32(level_start_target_box_nrs)
        boxes = self._dev(target_boxes)
        for lev in range(self.tree.nlevels):
            a, b = int(ltb[lev]), int(ltb[lev + 1])
            if a == b:
                continue
            sbase, sview = self.local_expansions_view(local_exps, lev)
            args = (_c(self.level_orders[lev]), _d(self.level_to_rscale(lev)), *self._kargs,
                    _i32(b - a), dptr(boxes[a:b]), dptr(g["centers"]), _i64(self.tree.nboxes), _i32(sbase),
                    dptr(sview), dptr(g["bts"]), dptr(g["btc"]), dptr(g["targets"]),
                    _i64(self.tree.ntargets), _d(self._scale), dptr(pot[0]))
            if self.gradient:
                call("sumpy_e2p_from_single_box_grad_f64", *args, dptr(pot[1]), st)
            else:
                call(self._entry("sumpy_e2p_from_single_box_f64"), *args, st)
        return pot

    # }}}
