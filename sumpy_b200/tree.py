"""Tree, traversal and translation classes under boxtree's names.

sumpy reads its tree and interaction lists from boxtree objects
(``sumpy/fmm.py:356-363, 372-397, 543-592, 752-754, 931-948``). boxtree is an
external dependency of sumpy, so this module provides builders with the same
call shapes -- ``TreeBuilder()(actx, sources, targets=..., max_particles_in_box=...)``,
``FMMTraversalBuilder()(actx, tree)``,
``TranslationClassesBuilder()(actx, trav, tree, is_translation_per_level=True)`` --
backed by the host C++ library ``libsumpy_b200_tree.so`` (source
``sumpy_b200/csrc/tree.cpp``, interface ``include/sumpy_b200_tree.h``).

Objects hold host numpy arrays; :meth:`Tree.to_device` etc. make torch CUDA
copies for the wrangler. Index arrays are int32, coordinates float64, SoA
``[3][n]`` as in boxtree.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from sumpy_b200 import _lib


def _tree_lib():
    lib = _lib.load_tree_library()
    return lib


class _Handle:
    def __init__(self, h):
        self.h = h

    def get(self, name):
        lib = _tree_lib()
        kind = ctypes.c_int()
        n = ctypes.c_int64()
        rc = lib.sumpy_tree_array_info(self.h, name.encode(), ctypes.byref(kind),
                                       ctypes.byref(n))
        if rc != 0:
            raise RuntimeError(lib.sumpy_tree_last_error().decode())
        arr = np.empty(n.value, dtype=np.int32 if kind.value == 0 else np.float64)
        rc = lib.sumpy_tree_array_copy(self.h, name.encode(),
                                       arr.ctypes.data_as(ctypes.c_void_p),
                                       ctypes.c_int64(arr.nbytes))
        if rc != 0:
            raise RuntimeError(lib.sumpy_tree_last_error().decode())
        return arr

    def __del__(self):
        if self.h:
            try:
                _tree_lib().sumpy_tree_free(self.h)
            except Exception:  # noqa: BLE001 (interpreter shutdown)
                pass
            self.h = None


def _soa(points, name):
    if isinstance(points, (list, tuple)):
        points = np.stack([np.asarray(p, dtype=np.float64) for p in points])
    if hasattr(points, "detach"):
        points = points.detach().cpu().numpy()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    if pts.ndim != 2 or pts.shape[0] != 3:
        raise ValueError(f"{name} must have shape (3, n); got {pts.shape}")
    return pts


@dataclass
class Tree:
    """Octree with boxtree's field names (``boxtree.Tree``)."""
    dimensions: int
    nsources: int
    ntargets: int
    nboxes: int
    nlevels: int
    sources_are_targets: bool
    root_extent: float
    bounding_box: tuple
    sources: np.ndarray
    targets: np.ndarray
    user_source_ids: np.ndarray
    sorted_target_ids: np.ndarray
    level_start_box_nrs: np.ndarray
    box_centers: np.ndarray
    box_levels: np.ndarray
    box_parent_ids: np.ndarray
    box_child_ids: np.ndarray
    box_coords: np.ndarray
    box_source_starts: np.ndarray
    box_source_counts_cumul: np.ndarray
    box_source_counts_nonchild: np.ndarray
    box_target_starts: np.ndarray
    box_target_counts_cumul: np.ndarray
    box_target_counts_nonchild: np.ndarray
    target_to_source: np.ndarray | None
    stick_out_factor: float = 0.0
    _handle: Any = field(default=None, repr=False)

    @property
    def aligned_nboxes(self):
        return self.nboxes

    @property
    def max_nsources_in_one_box(self):
        return int(self.box_source_counts_nonchild.max()) if self.nboxes else 0

    @property
    def max_ntargets_in_one_box(self):
        return int(self.box_target_counts_nonchild.max()) if self.nboxes else 0


@dataclass
class FromSepSmallerCSR:
    starts: np.ndarray
    lists: np.ndarray


@dataclass
class FMMTraversalInfo:
    """Interaction lists with boxtree's field names (``boxtree.traversal``)."""
    tree: Tree
    source_boxes: np.ndarray
    target_boxes: np.ndarray
    source_parent_boxes: np.ndarray
    target_or_target_parent_boxes: np.ndarray
    level_start_source_box_nrs: np.ndarray
    level_start_target_box_nrs: np.ndarray
    level_start_source_parent_box_nrs: np.ndarray
    level_start_target_or_target_parent_box_nrs: np.ndarray
    neighbor_source_boxes_starts: np.ndarray
    neighbor_source_boxes_lists: np.ndarray
    from_sep_siblings_starts: np.ndarray
    from_sep_siblings_lists: np.ndarray
    target_boxes_sep_smaller_by_source_level: list
    from_sep_smaller_by_level: list
    from_sep_bigger_starts: np.ndarray
    from_sep_bigger_lists: np.ndarray
    # no targets with extent: these lists do not exist
    from_sep_close_smaller_starts: Any = None
    from_sep_close_smaller_lists: Any = None
    from_sep_close_bigger_starts: Any = None
    from_sep_close_bigger_lists: Any = None
    well_sep_is_n_away: int = 1


@dataclass
class TranslationClassesInfo:
    """M2L translation classes (``boxtree.translation_classes``)."""
    traversal: FMMTraversalInfo
    from_sep_siblings_translation_classes: np.ndarray
    from_sep_siblings_translation_class_to_distance_vector: np.ndarray
    from_sep_siblings_translation_classes_level_starts: np.ndarray


def _root_box(bbox):
    """(bbox_min, root_extent) of a ``(3, 2)`` per-axis [min, max] box, as
    boxtree's ``TreeBuilder(..., bbox=...)``: the cube at ``min`` with the
    largest side."""
    bb = np.asarray(bbox, dtype=np.float64).reshape(3, 2)
    return np.ascontiguousarray(bb[:, 0]), float(np.max(bb[:, 1] - bb[:, 0]))


def _is_cuda(a):
    return hasattr(a, "is_cuda") and a.is_cuda


def build_all(sources, targets=None, max_particles_in_box=30, max_levels=None, bbox=None,
              device=None):
    """Build :class:`Tree`, :class:`FMMTraversalInfo` and
    :class:`TranslationClassesInfo` in one native call.

    ``bbox``, as boxtree's ``TreeBuilder(..., bbox=...)``: a ``(3, 2)`` array
    of per-axis ``[min, max]``; the root box is the cube at ``min`` with the
    largest side. Without it the root box is the particles' bounding cube.

    ``device`` (or sources given as a CUDA tensor): build on that GPU
    (``sumpy_tree_gpu_build``, the same arrays bit for bit); otherwise on the
    host (``sumpy_tree_build_in_box``). The returned objects hold host arrays
    either way."""
    if device is None and _is_cuda(sources):
        device = sources.device
    if device is not None:
        return build_all_gpu(sources, targets, max_particles_in_box, max_levels, bbox, device)
    H = _host_handle(sources, targets, max_particles_in_box, max_levels, bbox)
    return _objects(H)


def _host_handle(sources, targets, max_particles_in_box, max_levels, bbox):
    src = _soa(sources, "sources")
    tgt = None if targets is None else _soa(targets, "targets")
    lib = _tree_lib()
    h = ctypes.c_void_p()
    ptr = ctypes.c_void_p

    def p(a):
        return a.ctypes.data_as(ptr)

    sx, sy, sz = (np.ascontiguousarray(src[i]) for i in range(3))
    if tgt is None:
        tx = ty = tz = None
        ntgt = -1
    else:
        tx, ty, tz = (np.ascontiguousarray(tgt[i]) for i in range(3))
        ntgt = tgt.shape[1]
    if bbox is None:
        bmin, ext = None, 0.0
    else:
        bmin, ext = _root_box(bbox)
    rc = lib.sumpy_tree_build_in_box(
        ctypes.c_int64(src.shape[1]), p(sx), p(sy), p(sz),
        ctypes.c_int64(ntgt),
        None if tx is None else p(tx), None if ty is None else p(ty),
        None if tz is None else p(tz),
        ctypes.c_int(int(max_particles_in_box)),
        ctypes.c_int(0 if max_levels is None else int(max_levels)),
        None if bmin is None else p(bmin), ctypes.c_double(ext),
        ctypes.byref(h))
    if rc != 0:
        raise ValueError(lib.sumpy_tree_last_error().decode())
    return _Handle(h)


class _GpuHandle:
    """Result arrays of ``sumpy_tree_gpu_build`` (device memory owned by the
    native handle until this object goes)."""

    def __init__(self, h):
        self.h = h

    def _lib(self):
        from sumpy_b200 import _lib as L
        return L.load_cuda_library()

    def info(self, name):
        lib = self._lib()
        kind = ctypes.c_int()
        n = ctypes.c_int64()
        rc = lib.sumpy_tree_gpu_array_info(self.h, name.encode(), ctypes.byref(kind),
                                           ctypes.byref(n))
        if rc != 0:
            raise RuntimeError(lib.sumpy_last_error().decode())
        return kind.value, n.value

    def get(self, name):
        """Host copy."""
        from sumpy_b200._capi import stream_ptr
        kind, n = self.info(name)
        arr = np.empty(n, dtype=np.int32 if kind == 0 else np.float64)
        lib = self._lib()
        rc = lib.sumpy_tree_gpu_array_copy(self.h, name.encode(),
                                           arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes, 0,
                                           stream_ptr())
        if rc != 0:
            raise RuntimeError(lib.sumpy_last_error().decode())
        return arr

    def __del__(self):
        if self.h:
            try:
                self._lib().sumpy_tree_gpu_free(self.h)
            except Exception:  # noqa: BLE001 (interpreter shutdown)
                pass
            self.h = None


def _dev_soa(points, name, device):
    """(3, n) float64 contiguous CUDA tensor of host or device points."""
    import torch
    if isinstance(points, (list, tuple)):
        points = np.stack([np.asarray(p, dtype=np.float64) for p in points])
    t = torch.as_tensor(points, dtype=torch.float64, device=device).contiguous()
    if t.ndim != 2 or t.shape[0] != 3:
        raise ValueError(f"{name} must have shape (3, n); got {tuple(t.shape)}")
    return t


def gpu_tree_handle(src, tgt, max_particles_in_box, max_levels, bmin, ext,
                    source_starts=None, target_starts=None):
    """Run ``sumpy_tree_gpu_build`` on (3, n) CUDA tensors (problems given by
    their int64 start arrays) on the current stream."""
    import torch
    from sumpy_b200 import _lib as L
    from sumpy_b200._capi import stream_ptr
    lib = L.load_cuda_library()
    with torch.cuda.device(src.device):
        nprob = 1 if source_starts is None else len(source_starts) - 1
        sst = None if source_starts is None else np.ascontiguousarray(source_starts, np.int64)
        tst = None if target_starts is None else np.ascontiguousarray(target_starts, np.int64)
        vp = ctypes.c_void_p
        h = ctypes.c_void_p()
        rc = lib.sumpy_tree_gpu_build(
            ctypes.c_int64(src.shape[1]), vp(src[0].data_ptr()), vp(src[1].data_ptr()),
            vp(src[2].data_ptr()),
            ctypes.c_int64(-1 if tgt is None else tgt.shape[1]),
            None if tgt is None else vp(tgt[0].data_ptr()),
            None if tgt is None else vp(tgt[1].data_ptr()),
            None if tgt is None else vp(tgt[2].data_ptr()),
            ctypes.c_int32(nprob),
            None if sst is None else sst.ctypes.data_as(vp),
            None if tst is None else tst.ctypes.data_as(vp),
            ctypes.c_int(int(max_particles_in_box)),
            ctypes.c_int(0 if max_levels is None else int(max_levels)),
            None if bmin is None else np.ascontiguousarray(bmin, np.float64).ctypes.data_as(vp),
            ctypes.c_double(ext), stream_ptr(), ctypes.byref(h))
        if rc != 0:
            raise ValueError(lib.sumpy_last_error().decode())
    return _GpuHandle(h)


def build_all_gpu(sources, targets=None, max_particles_in_box=30, max_levels=None, bbox=None,
                  device="cuda"):
    """:func:`build_all` on the GPU (``sumpy_tree_gpu_build``): the same
    arrays, bit for bit, as the host builder; returned as host arrays."""
    src = _dev_soa(sources, "sources", device)
    tgt = None if targets is None else _dev_soa(targets, "targets", device)
    bmin, ext = (None, 0.0) if bbox is None else _root_box(bbox)
    H = gpu_tree_handle(src, tgt, max_particles_in_box, max_levels, bmin, ext)
    out = _objects(H, keep_handle=False)
    del H
    return out


def _objects(H, keep_handle=True):
    """Tree, traversal and translation classes from a builder handle (host
    arrays; ``keep_handle``: the tree keeps the handle alive)."""
    nb, nl, ns, nt, sat = (int(x) for x in H.get("scalars"))
    g = H.get

    def s3(name, n):
        return g(name).reshape(3, n)

    bbox_min = g("bbox_min")
    root_extent = float(g("root_extent")[0])
    tree = Tree(
        dimensions=3, nsources=ns, ntargets=nt, nboxes=nb, nlevels=nl,
        sources_are_targets=bool(sat), root_extent=root_extent,
        bounding_box=(bbox_min, bbox_min + root_extent),
        sources=s3("sources", ns), targets=s3("targets", nt),
        user_source_ids=g("user_source_ids"), sorted_target_ids=g("sorted_target_ids"),
        level_start_box_nrs=g("level_start_box_nrs"),
        box_centers=s3("box_centers", nb), box_levels=g("box_levels"),
        box_parent_ids=g("box_parent_ids"),
        box_child_ids=g("box_child_ids").reshape(8, nb),
        box_coords=g("box_coords").reshape(3, nb),
        box_source_starts=g("box_source_starts"),
        box_source_counts_cumul=g("box_source_counts_cumul"),
        box_source_counts_nonchild=g("box_source_counts_nonchild"),
        box_target_starts=g("box_target_starts"),
        box_target_counts_cumul=g("box_target_counts_cumul"),
        box_target_counts_nonchild=g("box_target_counts_nonchild"),
        target_to_source=g("target_to_source") if sat else None,
        _handle=H if keep_handle else None)

    tb_all = g("sep_smaller_target_boxes")
    tb_ls = g("sep_smaller_target_boxes_level_starts")
    st_all = g("sep_smaller_starts")
    st_off = g("sep_smaller_starts_level_offsets")
    li_all = g("sep_smaller_lists")
    li_off = g("sep_smaller_lists_level_offsets")
    by_level_tb, by_level = [], []
    for lev in range(nl):
        by_level_tb.append(tb_all[tb_ls[lev]:tb_ls[lev + 1]])
        by_level.append(FromSepSmallerCSR(
            starts=st_all[st_off[lev]:st_off[lev + 1]],
            lists=li_all[li_off[lev]:li_off[lev + 1]]))

    trav = FMMTraversalInfo(
        tree=tree,
        source_boxes=g("source_boxes"), target_boxes=g("target_boxes"),
        source_parent_boxes=g("source_parent_boxes"),
        target_or_target_parent_boxes=g("target_or_target_parent_boxes"),
        level_start_source_box_nrs=g("level_start_source_box_nrs"),
        level_start_target_box_nrs=g("level_start_target_box_nrs"),
        level_start_source_parent_box_nrs=g("level_start_source_parent_box_nrs"),
        level_start_target_or_target_parent_box_nrs=g(
            "level_start_target_or_target_parent_box_nrs"),
        neighbor_source_boxes_starts=g("neighbor_source_boxes_starts"),
        neighbor_source_boxes_lists=g("neighbor_source_boxes_lists"),
        from_sep_siblings_starts=g("from_sep_siblings_starts"),
        from_sep_siblings_lists=g("from_sep_siblings_lists"),
        target_boxes_sep_smaller_by_source_level=by_level_tb,
        from_sep_smaller_by_level=by_level,
        from_sep_bigger_starts=g("from_sep_bigger_starts"),
        from_sep_bigger_lists=g("from_sep_bigger_lists"))

    cls_ls = g("from_sep_siblings_translation_classes_level_starts")
    tcls = TranslationClassesInfo(
        traversal=trav,
        from_sep_siblings_translation_classes=g("from_sep_siblings_translation_classes"),
        from_sep_siblings_translation_class_to_distance_vector=s3(
            "from_sep_siblings_translation_class_to_distance_vector", int(cls_ls[-1])),
        from_sep_siblings_translation_classes_level_starts=cls_ls)
    tree._traversal = trav
    tree._translation_classes = tcls
    return tree, trav, tcls


# {{{ boxtree-shaped builders

class TreeBuilder:
    """``boxtree.TreeBuilder`` call shape. The traversal and translation
    classes are built in the same native call and cached on the tree."""

    def __init__(self, actx=None):
        self.actx = actx

    def __call__(self, actx, particles, targets=None, max_particles_in_box=None,
                 max_levels=None, debug=False, kind="adaptive", bbox=None, **kwargs):
        if max_particles_in_box is None:
            raise TypeError("max_particles_in_box must be given")
        if kind not in ("adaptive", "adaptive-level-restricted") and kind is not None:
            raise NotImplementedError(f"tree kind '{kind}'")
        tree, _, _ = build_all(particles, targets, max_particles_in_box, max_levels, bbox=bbox)
        return tree, None


class FMMTraversalBuilder:
    """``boxtree.traversal.FMMTraversalBuilder`` call shape."""

    def __init__(self, actx=None, well_sep_is_n_away=1):
        if well_sep_is_n_away != 1:
            raise NotImplementedError("only well_sep_is_n_away=1 is supported")

    def __call__(self, actx, tree, debug=False, **kwargs):
        return tree._traversal, None


class TranslationClassesBuilder:
    """``boxtree.translation_classes.TranslationClassesBuilder`` call shape."""

    def __init__(self, actx=None):
        pass

    def __call__(self, actx, trav, tree, is_translation_per_level=True):
        if not is_translation_per_level:
            raise NotImplementedError("translation classes are built per level")
        # a traversal restricted to part of the tree (sumpy_b200.distributed)
        # carries the classes of its own List-2 entries
        own = getattr(trav, "_translation_classes", None)
        return (own if own is not None else tree._translation_classes), None

# }}}
