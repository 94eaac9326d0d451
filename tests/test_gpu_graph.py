"""drive_fmm replaying a CUDA graph (wrangler ``cuda_graph=True``) against the
eager launch sequence: same potentials for new strengths on every call,
host or device strengths, results that later calls do not overwrite."""
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
from sumpy_b200._capi import launch_counter
from sumpy_b200.tree import build_all
from tests._pointsets import sphere_plummer

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_graph_replay_matches_eager(cuda_device, precision):
    src = sphere_plummer(40000, 21)
    tree, trav, tcls = build_all(src, None, 48)
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)

    def wr(graph):
        return SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: 8,
                                      translation_classes_data=tcls, precision=precision,
                                      cuda_graph=graph)

    we, wg = wr(False), wr(True)
    rng = np.random.default_rng(4)
    outs = []
    for it in range(3):
        q = rng.standard_normal(src.shape[1])
        ref = drive_fmm(None, we, [torch.as_tensor(q, device=cuda_device)])[0].cpu().numpy()
        qin = torch.as_tensor(q).pin_memory() if it == 2 else torch.as_tensor(q, device=cuda_device)
        n0 = launch_counter.value
        (got,) = drive_fmm(None, wg, [qin])
        if it > 0:   # a replay counts the captured launches
            assert launch_counter.value - n0 == wg._graph_cache[-1] > 0
        outs.append((got, ref))
    wg.check_status()
    for got, ref in outs:   # earlier results survive later replays
        assert relerr(got.cpu().numpy(), ref) < 1e-12
