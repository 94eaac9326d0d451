"""Batched evaluation of many independent 3D Laplace FMM problems.

sumpy evaluates one problem per ``drive_fmm`` call (``sumpy/fmm.py:609-1086``
under boxtree's driver), one kernel per level and stage. For a batch of
small problems that is launch-bound: a 10k-point problem has ~25 launches of
a few microseconds of work each. :class:`BatchedLaplaceFMM` instead

1. builds all problems as one forest in a common root box
   (:func:`sumpy_b200.forest.build_forest`), so every stage of every level
   runs for the whole batch in one launch;
2. records the whole evaluation (reorder, P2M ... L2P, reorder back) as one
   CUDA graph after a warm-up, and replays it per call with the batch's
   strengths copied into the graph's input buffer;
3. optionally picks the M2L work-item size by measurement
   (:mod:`sumpy_b200.autotune`).
"""
from __future__ import annotations

import numpy as np
import torch

from sumpy_b200.drive import drive_fmm
from sumpy_b200.expansion import (
    LinearPDEConformingVolumeTaylorLocalExpansion,
    LinearPDEConformingVolumeTaylorMultipoleExpansion,
)
from sumpy_b200.fmm import SumpyExpansionWrangler, SumpyTreeIndependentDataForWrangler
from sumpy_b200.forest import build_forest
from sumpy_b200.kernel import LaplaceKernel


class BatchedLaplaceFMM:
    """Potentials of a batch of problems with fixed geometry.

    :arg sources: list of ``(3, n_i)`` float64 arrays.
    :arg targets: ``None`` (evaluate at the sources, self-interaction
        excluded) or a list of ``(3, m_i)`` arrays.
    :arg order: expansion order on every level.
    :arg precision: ``"fp64"`` or ``"mixed"`` (see :class:`SumpyExpansionWrangler`).
    :arg bbox: common root box, ``(3, 2)``; default the batch's bounding cube.
    :arg use_graph: replay a captured CUDA graph (True) or launch eagerly.
    :arg autotune: choose the schedule knobs by timing (coordinate descent,
        cached on disk; :func:`sumpy_b200.autotune.tune_schedule`).
    :arg gpu_tree: build the forest on the GPU in one pass (default) instead
        of host trees merged on the host (the same arrays either way).
    """

    def __init__(self, sources, targets=None, order=8, max_particles_in_box=32,
                 precision="mixed", bbox=None, device="cuda", use_graph=True,
                 autotune=False, m2l_item_groups=None, autotune_cache=None, gpu_tree=True):
        import time
        self.device = torch.device(device)
        t0 = time.perf_counter()
        tree, trav, tcls, forest = build_forest(
            sources, targets, max_particles_in_box, bbox,
            device=self.device if gpu_tree and self.device.type == "cuda" else None)
        # wall times of the set-up steps (seconds)
        self.timings = {"forest_s": time.perf_counter() - t0}
        self.tree, self.traversal, self.forest = tree, trav, forest
        knl = LaplaceKernel(3)
        exclude_self = targets is None
        ti = SumpyTreeIndependentDataForWrangler(
            None, lambda o, **kw: LinearPDEConformingVolumeTaylorMultipoleExpansion(knl, o),
            lambda o, **kw: LinearPDEConformingVolumeTaylorLocalExpansion(knl, o), [knl],
            exclude_self=exclude_self)
        self.wrangler = SumpyExpansionWrangler(
            ti, trav, np.float64, lambda k, a, t, lev: int(order),
            translation_classes_data=tcls, precision=precision, device=self.device,
            m2l_item_groups=m2l_item_groups)
        self.use_graph = bool(use_graph)
        self._w = torch.zeros(tree.nsources, dtype=torch.float64, device=self.device)
        self._graph = None
        self._out = None
        self.schedule = self.wrangler.schedule()
        if autotune:
            from sumpy_b200.autotune import tune_schedule
            t0 = time.perf_counter()
            self.schedule = tune_schedule(self.wrangler, lambda: self._eager(self._w),
                                          path=autotune_cache)
            self.timings["autotune_s"] = time.perf_counter() - t0

    @property
    def nsources(self):
        return self.tree.nsources

    @property
    def ntargets(self):
        return self.tree.ntargets

    def _eager(self, w):
        (pot,) = drive_fmm(None, self.wrangler, [w])
        return pot

    def capture(self):
        """Warm up (builds every schedule and operator table) on a side
        stream, then record one evaluation as a CUDA graph."""
        cur = torch.cuda.current_stream(self.device)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(cur)
        with torch.cuda.stream(side):
            for _ in range(2):
                self._eager(self._w)
        cur.wait_stream(side)
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self._out = self._eager(self._w)
        self._graph = graph
        return graph

    def _strengths(self, strengths):
        if isinstance(strengths, (list, tuple)):
            strengths = torch.cat([torch.as_tensor(s, dtype=torch.float64).reshape(-1)
                                   for s in strengths])
        w = torch.as_tensor(strengths, dtype=torch.float64)
        if w.numel() != self.nsources:
            raise ValueError(f"expected {self.nsources} strengths in total, got {w.numel()}")
        return w.reshape(-1)

    def evaluate(self, strengths):
        """Concatenated potentials of all problems (``[ntargets]`` float64 on
        the device, user order, problem after problem). Accepts one
        concatenated strength vector or a list of per-problem vectors, on
        the host or the device."""
        w = self._strengths(strengths)
        if not self.use_graph:
            return self._eager(w.to(self.device).contiguous())
        if self._graph is None:
            self.capture()
        self._w.copy_(w, non_blocking=True)
        self._graph.replay()
        return self._out.clone()

    def __call__(self, strengths):
        """Per-problem potentials (list of device tensors)."""
        return self.forest.split_targets(self.evaluate(strengths))

    def check_status(self):
        self.wrangler.check_status()
