"""The distributed FMM's ranks emulated one after another on one GPU (no
kernel waits for another rank's): each rank's GPU wrangler evaluates its
local traversal; the partial multipoles of all ranks, summed, are the global
multipoles, and with them each rank's potentials -- on its own targets --
sum to the single-rank GPU FMM (FP64 to 1e-12, mixed to the mixed form's
accuracy), as sumpy/test/test_distributed.py:107-146 checks a distributed
run against a single-rank one. Also the runner end to end on a one-rank
process group."""
import os
import socket

import numpy as np
import pytest
import torch

from sumpy_b200 import (
    LaplaceKernel,
    LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
    LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp,
    SumpyExpansionWrangler,
    SumpyTreeIndependentDataForWrangler,
    drive_fmm,
)
from sumpy_b200 import distributed as D
from sumpy_b200.tree import build_all
from tests._pointsets import sphere_plummer

pytestmark = pytest.mark.gpu

ORDER = 8


def _tree_indep():
    knl = LaplaceKernel(3)
    return SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)


class _EmulatedRank(D.DistributedSumpyExpansionWrangler):
    """One rank of an emulated group: its exchange installs the precomputed
    sum of every rank's partial multipoles."""
    global_mpoles = None

    def communicate_mpoles(self, actx, mpole_exps, return_stats=False):
        mpole_exps.copy_(self.global_mpoles)


def _relerr(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nranks", [2, 5])
def test_emulated_ranks_match_single_rank(cuda_device, precision, nranks):
    src = sphere_plummer(60000, 31)
    tree, trav, tcls = build_all(src, None, 40)
    q = torch.as_tensor(np.random.default_rng(9).standard_normal(src.shape[1]),
                        device=cuda_device)
    ti = _tree_indep()
    glob = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: ORDER,
                                  translation_classes_data=tcls, precision=precision,
                                  device=cuda_device)
    ref = drive_fmm(None, glob, [q])[0]
    qs = glob.reorder_sources(q)
    mp_ref = glob.coarsen_multipoles(
        None, trav.level_start_source_parent_box_nrs, trav.source_parent_boxes,
        glob.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs]))
    owner = D.partition_boxes(tree, trav, nranks)
    ranks = []
    msum = torch.zeros_like(mp_ref)
    for r in range(nranks):
        lt, lc = D.local_traversal(tree, trav, tcls, owner, r)
        w = _EmulatedRank(None, None, ti, lt, trav, np.float64, lambda *a: ORDER,
                          translation_classes_data=lc, precision=precision,
                          device=cuda_device)
        m = w.coarsen_multipoles(
            None, lt.level_start_source_parent_box_nrs, lt.source_parent_boxes,
            w.form_multipoles(None, lt.level_start_source_box_nrs, lt.source_boxes, [qs]))
        msum += m
        ranks.append(w)
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert _relerr(msum, mp_ref) < tol
    pot = torch.zeros_like(ref)
    for w in ranks:
        w.global_mpoles = msum
        (p,) = drive_fmm(None, w, [q])
        (p,) = w.gather_potential_results([p])     # one-rank group: unchanged
        w.check_status()
        pot += p
    assert _relerr(pot, ref) < tol


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_runner_on_one_rank_group(cuda_device):
    import datetime
    import torch.distributed as dist
    if dist.is_initialized():
        pytest.skip("a process group already exists")
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}",
                            rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        src = sphere_plummer(30000, 32)
        tree, trav, tcls = build_all(src, None, 40)
        q = np.random.default_rng(3).standard_normal(src.shape[1])
        ti = _tree_indep()

        def factory(local_trav, global_trav):
            return D.DistributedSumpyExpansionWrangler(
                None, None, ti, local_trav, global_trav, np.float64, lambda *a: ORDER,
                device=cuda_device)

        runner = D.DistributedFMMRunner(None, tree, None, factory)
        (pot,) = runner.drive_dfmm(None, [q])
        glob = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: ORDER,
                                      device=cuda_device)
        (ref,) = drive_fmm(None, glob, [torch.as_tensor(q, device=cuda_device)])
        assert _relerr(pot, ref) < 1e-13
        with pytest.raises(NotImplementedError):
            D.DistributedSumpyExpansionWrangler(
                None, None, ti, trav, trav, np.float64, lambda *a: ORDER,
                communicate_mpoles_via_allreduce=False, device=cuda_device)
    finally:
        dist.destroy_process_group()
