"""Benchmark: 3D Laplace FMM evaluation throughput on one B200 (or N replicas).

Workload (one step = one full FMM evaluation, ``drive_fmm``): 1,000,000
points that are both sources and targets (exclude_self), 50% on the unit
sphere surface and 50% Plummer (scale 0.1), strengths N(0, 1), expansion
order 10, max_particles_in_box 32. Synthetic, seeded inputs; the tree,
interaction lists and M2L tables are built once before timing (reported
separately). ``value`` is Mpts/s of the mixed-precision form with inputs
resident in HBM; the FP64 form is timed the same way for the ratio; the
accuracy of both is the relative L2 error on 4,096 sampled targets against
an FP64 direct sum. ``e2e`` runs the public API with host buffers (H2D of the
strengths, D2H of the potentials inside the timed region).

``--impl reference`` times the FP64 CPU restatement of sumpy's algorithm
(the oracle, C + OpenMP on all host cores) on a bounded sample of the same
workload and prints the same metric.

Multi-GPU (torchrun): each rank evaluates its own replica; no collective on
the data path (the problem does not shard in this build); value = points of
all ranks / max over ranks of the step time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "3D Laplace FMM Mpts/s @ relL2<=1e-6 (mixed vs FP64 GPU); adjoint/forward ratio"
NPOINTS = 1_000_000
ORDER = 10
# max_particles_in_box of the 1M-point workload (the workload leaves it open): the fastest
# mixed form in a sweep over 32..192 on this GPU (32: 11.0 ms, 64: 10.1, 96: 9.6, 128: 10.0,
# 192: 13.7 ms; accuracy against the direct sum 3.5e-6 for all). The FP64 form is timed on
# the same tree (like for like) and, separately, on its own fastest tree (FP64_MAX_PARTICLES).
MAX_PARTICLES = 96
FP64_MAX_PARTICLES = 128
HELMHOLTZ_MAX_PARTICLES = 64   # same sweep for the Helmholtz workload: 32: 46 ms, 64: 21 ms
BATCH_MAX_PARTICLES = 32       # the batched workload's own setting
ADJOINT_MAX_PARTICLES = 32
ACCURACY_MAX_PARTICLES = 128   # the order sweep toward relL2 <= 1e-6 (p = 11..13)
NSAMPLE = 4096


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--npoints", type=int, default=NPOINTS)
    ap.add_argument("--order", type=int, default=ORDER)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip timing the FP64 form")
    ap.add_argument("--stage-times", action="store_true", help="print per-stage times")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-problem batch")
    ap.add_argument("--no-helmholtz", action="store_true",
                    help="skip the 500k-point Helmholtz workload")
    ap.add_argument("--only", choices=["mixed", "fp64", "batch", "helmholtz", "uniform",
                                       "matrix"],
                    help="run one workload alone (--steps/--warmup apply) and print its result; "
                         "for profiling")
    ap.add_argument("--eager", action="store_true",
                    help="with --only: launch kernel by kernel instead of replaying a CUDA graph")
    ap.add_argument("--helmholtz-npoints", type=int, default=500_000)
    ap.add_argument("--helmholtz-precision", choices=["mixed", "fp64", "both"], default="both")
    return ap.parse_args()


def workload(npoints, seed=2024):
    from tests._pointsets import sphere_plummer
    pts = sphere_plummer(npoints, seed)
    q = np.random.default_rng(44).standard_normal(npoints)
    return pts, q


# {{{ reference arm / CPU baseline (oracle)

def cpu_fmm_rate(npoints, order, seed=2024, target_seconds=10.0, min_points=5000):
    """Time the oracle FMM on a sample sized to take about target_seconds."""
    from oracle import oracle as O
    from sumpy_b200.tree import build_all
    n = max(min_points, min(npoints, 20000))
    while True:
        pts, q = workload(n, seed)
        tree, trav, tcls = build_all(pts, None, MAX_PARTICLES)
        t0 = time.perf_counter()
        O.run_fmm(tree, trav, tcls, order, q, exclude_self=True)
        dt = time.perf_counter() - t0
        if dt > 0.3 * target_seconds or n >= npoints:
            return n, dt
        n = min(npoints, int(n * min(8.0, target_seconds / max(dt, 1e-3))))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from sumpy_b200.tree import build_all
    n, _ = cpu_fmm_rate(args.npoints, args.order, target_seconds=4.0)
    pts, q = workload(n)
    tree, trav, tcls = build_all(pts, None, MAX_PARTICLES)
    for _ in range(args.warmup):
        O.run_fmm(tree, trav, tcls, args.order, q, exclude_self=True)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.run_fmm(tree, trav, tcls, args.order, q, exclude_self=True)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = n * args.steps / tot / 1e6
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpts/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"laplace3d_fmm_sphere_plummer_n{args.npoints}_p{args.order}",
                   "sample_points": n, "order": args.order,
                   "max_particles_in_box": MAX_PARTICLES, "exclude_self": True},
        "cpu_baseline": {"value": value, "unit": "Mpts/s", "cores": cores, "kind": "port",
                         "sample": f"{n}-point sample of the same distribution, p={args.order}, "
                                   f"FP64 C/OpenMP oracle (sumpy's algorithm restated), "
                                   f"{cores} threads"},
        "e2e": {"value": value, "unit": "Mpts/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)

# }}}


class ClockSampler:
    """SM clock and clock-event reasons sampled DURING a timed region: an NVML
    thread polling every 5 ms (read-only queries), so that even a region of a
    few tens of milliseconds gets samples; nvidia-smi at its 100 ms floor as
    the fallback when NVML is unavailable."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index, period_s=0.005):
        self.gpu = gpu_index
        self.period = period_s
        self.proc = None
        self.thread = None
        self.samples = []
        self.max_mhz = None
        self.out = ""

    def _nvml_loop(self, nv, h, bits):
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), [n for n, b in bits if rs & b]))
            except Exception:  # noqa: BLE001 (a failed read is skipped)
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            import torch
            uuid = None
            try:
                uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            except Exception:  # noqa: BLE001
                uuid = None
            h = None
            if uuid:
                for cand in (uuid, "GPU-" + uuid):
                    try:
                        h = nv.nvmlDeviceGetHandleByUUID(cand)
                        break
                    except Exception:  # noqa: BLE001
                        h = None
            if h is None:
                h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            bits = [("hw_slowdown", nv.nvmlClocksEventReasonHwSlowdown),
                    ("hw_thermal_slowdown", nv.nvmlClocksEventReasonHwThermalSlowdown),
                    ("sw_thermal_slowdown", nv.nvmlClocksEventReasonSwThermalSlowdown),
                    ("sw_power_cap", nv.nvmlClocksEventReasonSwPowerCap)]
            self._stop = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h, bits),
                                           daemon=True)
            self.thread.start()
            return self
        except Exception:  # noqa: BLE001 (no NVML: fall back to nvidia-smi)
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self._stop.set()
            self.thread.join(timeout=2)
            return
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()
            for r in (self.out or "").strip().splitlines():
                r = [x.strip() for x in r.split(",")]
                if len(r) < 9:
                    continue
                try:
                    sm = float(r[1])
                    self.max_mhz = float(r[2])
                except ValueError:
                    continue
                self.samples.append(
                    (sm, [nm for nm, v in zip(self.NAMES, r[5:9]) if v.lower() == "active"]))

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        reasons = sorted({n for _, rs in self.samples for n in rs})
        return {"sm_mhz": float(np.median([s for s, _ in self.samples])),
                "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples),
                "source": "nvml" if self.thread is not None else "nvidia-smi"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    from sumpy_b200.distributed import init as dist_init, max_over_ranks
    rank, world, local_rank = dist_init("nccl", timeout_s=300)
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)

    from sumpy_b200 import (
        P2P, LaplaceKernel, SumpyExpansionWrangler, SumpyTreeIndependentDataForWrangler,
        drive_fmm)
    from sumpy_b200 import _capi
    from sumpy_b200.expansion import (
        LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
        LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp)
    from sumpy_b200.tree import build_all

    if args.only in ("batch", "helmholtz", "uniform", "matrix"):
        if args.only == "batch":
            res = batched_bench(dev, steps=args.steps, warmup=args.warmup)
        elif args.only == "matrix":
            res = matrix_bench(dev, steps=args.steps, warmup=args.warmup)
        elif args.only == "helmholtz":
            precs = (("mixed", "fp64") if args.helmholtz_precision == "both"
                     else (args.helmholtz_precision,))
            res = helmholtz_bench(dev, steps=args.steps, warmup=args.warmup,
                                  npoints=args.helmholtz_npoints, precisions=precs)
        else:
            res = uniform_bench(dev, steps=args.steps, warmup=args.warmup, cpu=False)
        if rank == 0:
            print(json.dumps({"only": args.only, "result": res}), flush=True)
        return

    # cpu baseline first, before any process pool / GPU work competes for the host
    cpu_line = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.only is None:
        n, dt = cpu_fmm_rate(args.npoints, args.order, target_seconds=12.0)
        cores = os.cpu_count()
        cpu_line = {"value": n / dt / 1e6, "unit": "Mpts/s", "cores": cores, "kind": "port",
                    "sample": f"{n}-point sample of the same distribution, p={args.order}, "
                              f"FP64 C/OpenMP oracle, {cores} threads, {dt:.1f} s"}

    pts, q = workload(args.npoints)
    t0 = time.perf_counter()
    tree, trav, tcls = build_all(pts, None, MAX_PARTICLES)
    t_tree = time.perf_counter() - t0
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)

    def wrangler(precision, graph=True):
        # graph: drive_fmm replays the evaluation from a CUDA graph (one host
        # call per step); the eager form launches each kernel from Python
        return SumpyExpansionWrangler(ti, trav, np.float64, lambda k, a, t, lev: args.order,
                                      precision=precision, device=dev, cuda_graph=graph)

    q_dev = torch.as_tensor(q, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, steps):
        """Per-step CUDA-event times with an L2 flush between steps."""
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        torch.cuda.synchronize()
        barrier()
        for i in range(steps):
            flush.fill_(float(i))
            evs[i][0].record()
            fn()
            evs[i][1].record()
        torch.cuda.synchronize()
        barrier()
        ms = [a.elapsed_time(b) for a, b in evs]
        return max_over_ranks(sum(ms), device=dev) / steps, ms

    if args.only in ("mixed", "fp64"):
        w = wrangler(args.only, graph=not args.eager)
        for _ in range(max(1, args.warmup)):
            drive_fmm(None, w, [q_dev])
        ms, _ = timed(lambda: drive_fmm(None, w, [q_dev]), args.steps)
        if rank == 0:
            print(json.dumps({"only": args.only, "result": {
                "ms_per_step": ms, "Mpts_s": args.npoints / (ms * 1e-3) / 1e6}}), flush=True)
        return

    # setup (plans, tables, graph capture) outside timing
    t0 = time.perf_counter()
    w_mx = wrangler("mixed")
    drive_fmm(None, w_mx, [q_dev])
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0

    # the same evaluation launched kernel by kernel from Python
    w_mx.cuda_graph = False
    for _ in range(max(1, args.warmup)):
        drive_fmm(None, w_mx, [q_dev])
    ms_eager, _ = timed(lambda: drive_fmm(None, w_mx, [q_dev]), args.steps)
    w_mx.cuda_graph = True

    for _ in range(args.warmup):
        drive_fmm(None, w_mx, [q_dev])
    _capi.launch_counter.reset()
    with ClockSampler(local_rank) as clk:
        ms_mx, _ = timed(lambda: drive_fmm(None, w_mx, [q_dev]), args.steps)
    launches = _capi.launch_counter.value
    clocks = clk.summary()

    # e2e through the public API with host buffers
    q_host = torch.as_tensor(q).pin_memory()
    pot_host = torch.empty(args.npoints, dtype=torch.float64).pin_memory()

    def e2e_step():
        # strengths copied from pinned host memory into the graph's input
        (pot,) = drive_fmm(None, w_mx, [q_host])
        pot_host.copy_(pot, non_blocking=True)

    for _ in range(2):
        e2e_step()
    ms_e2e, _ = timed(e2e_step, args.steps)

    # FP64 form
    ms_64 = None
    w_64 = None
    if not args.no_fp64:
        w_64 = wrangler("fp64")
        for _ in range(max(1, args.warmup)):
            drive_fmm(None, w_64, [q_dev])
        ms_64, _ = timed(lambda: drive_fmm(None, w_64, [q_dev]), args.steps)

    # FP64 on its own fastest tree (larger leaves favour the slower FP64 M2L)
    fp64_best = None
    if not args.no_fp64 and args.npoints == NPOINTS and args.order == ORDER:
        tree_b, trav_b, tcls_b = build_all(pts, None, FP64_MAX_PARTICLES)
        w_b = SumpyExpansionWrangler(ti, trav_b, np.float64, lambda k, a, t, lev: args.order,
                                     translation_classes_data=tcls_b, precision="fp64",
                                     device=dev, cuda_graph=True)
        for _ in range(max(1, args.warmup)):
            drive_fmm(None, w_b, [q_dev])
        ms_b, _ = timed(lambda: drive_fmm(None, w_b, [q_dev]), args.steps)
        fp64_best = {"max_particles_in_box": FP64_MAX_PARTICLES, "ms_per_step": ms_b,
                     "value": world * args.npoints / (ms_b * 1e-3) / 1e6}
        del w_b, tree_b, trav_b, tcls_b

    # accuracy on sampled targets against the FP64 direct sum
    rng = np.random.default_rng(99)
    sample = rng.choice(args.npoints, size=min(NSAMPLE, args.npoints), replace=False)
    (ref,) = P2P([knl], exclude_self=True)(None, pts[:, sample], pts, (q,),
                                           target_to_source=sample, device=dev)
    (pot_mx,) = drive_fmm(None, w_mx, [q_dev])
    ref = ref.cpu().numpy()

    def rel(p):
        return float(np.linalg.norm(p[sample] - ref) / np.linalg.norm(ref))

    err_mx = rel(pot_mx.cpu().numpy())
    err_64 = rel(drive_fmm(None, w_64, [q_dev])[0].cpu().numpy()) if w_64 is not None else None

    # the metric's accuracy target (relL2 <= 1e-6) is out of reach at p = 10
    # for this algorithm (the FP64 form gives 3.4e-6); the same workload at
    # the orders around the target, mixed form, same tree
    # (leaf size 128: the errors are the same as at 96 within 1 %, the time lower)
    at_target = None
    if args.npoints == NPOINTS and args.order == ORDER and not args.only and world == 1:
        at_target = []
        tree_a, trav_a, tcls_a = build_all(pts, None, ACCURACY_MAX_PARTICLES)
        for p_hi in (11, 12, 13):
            w_p = SumpyExpansionWrangler(ti, trav_a, np.float64, lambda k, a, t, lev, p=p_hi: p,
                                         translation_classes_data=tcls_a, precision="mixed",
                                         device=dev, cuda_graph=True)
            for _ in range(max(1, args.warmup)):
                drive_fmm(None, w_p, [q_dev])
            ms_p, _ = timed(lambda: drive_fmm(None, w_p, [q_dev]), args.steps)
            e_p = rel(drive_fmm(None, w_p, [q_dev])[0].cpu().numpy())
            w_p.check_status()
            at_target.append({"order": p_hi, "max_particles_in_box": ACCURACY_MAX_PARTICLES,
                              "ms_per_step": ms_p,
                              "value": args.npoints / (ms_p * 1e-3) / 1e6, "relL2_mixed": e_p,
                              "meets_1e-6": e_p <= 1e-6})
            del w_p
            if e_p <= 1e-6:
                break
        if at_target[-1]["meets_1e-6"] and not args.no_fp64:
            # the FP64 form at the same order and on the same tree: the
            # metric's mixed-vs-FP64 comparison at relL2 <= 1e-6
            p_hi = at_target[-1]["order"]
            w_f = SumpyExpansionWrangler(ti, trav_a, np.float64, lambda k, a, t, lev, p=p_hi: p,
                                         translation_classes_data=tcls_a, precision="fp64",
                                         device=dev, cuda_graph=True)
            for _ in range(max(1, args.warmup)):
                drive_fmm(None, w_f, [q_dev])
            ms_f, _ = timed(lambda: drive_fmm(None, w_f, [q_dev]), args.steps)
            e_f = rel(drive_fmm(None, w_f, [q_dev])[0].cpu().numpy())
            at_target[-1].update({
                "fp64_ms_per_step": ms_f, "fp64_value": args.npoints / (ms_f * 1e-3) / 1e6,
                "relL2_fp64": e_f,
                "mixed_over_fp64": ms_f / at_target[-1]["ms_per_step"]})
            del w_f
        del tree_a, trav_a, tcls_a

    pipes = pipe_peaks_measured(dev)
    stage_ms, roof, roof_m2l = stage_breakdown(w_mx, trav, q_dev, dev, pipe_peaks=pipes)
    adj = adjoint_bench(dev) if world == 1 else None
    batch = batched_bench(dev) if world == 1 and not args.no_batch else None
    helm = helmholtz_bench(dev) if world == 1 and not args.no_helmholtz else None
    import gc
    gc.collect()
    uni = uniform_bench(dev, cpu=not args.no_cpu_baseline) if world == 1 else None
    mat = matrix_bench(dev) if world == 1 else None

    value = world * args.npoints / (ms_mx * 1e-3) / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": "Mpts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mx,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {
            "workload": f"laplace3d_fmm_sphere_plummer_n{args.npoints}_p{args.order}",
            "npoints": args.npoints, "order": args.order,
            "max_particles_in_box": MAX_PARTICLES, "exclude_self": True,
            "precision": "mixed (FP32 near field, M2P, P2L with FP64 offsets and sums; "
                         "3xTF32 tensor-core M2L and M2M; FP64 elsewhere)",
            "l2": "flushed between steps (256 MB write outside the timed events)",
            "parallelism": f"replicas x{world}",
            "launch": "drive_fmm replaying a CUDA graph of the whole evaluation "
                      "(wrangler cuda_graph=True); eager timing beside it",
            "tree_build_s": round(t_tree, 3), "setup_s": round(t_setup, 3),
        },
        "eager": {"ms_per_step": ms_eager,
                  "value": world * args.npoints / (ms_eager * 1e-3) / 1e6},
        "accuracy": {"relL2_mixed": err_mx, "relL2_fp64": err_64, "targets_sampled": len(sample),
                     "reference": "FP64 direct sum (GPU kernel sumpy_p2p_direct_f64)"},
        "fp64": {"value": (world * args.npoints / (ms_64 * 1e-3) / 1e6) if ms_64 else None,
                 "ms_per_step": ms_64},
        "mixed_over_fp64": (ms_64 / ms_mx) if ms_64 else None,
        "fp64_own_best_tree": fp64_best,
        "order_for_accuracy_target": at_target,
        "mixed_over_fp64_own_best": (fp64_best["ms_per_step"] / ms_mx) if fp64_best else None,
        "mixed_over_fp64_at_accuracy_target": (at_target[-1].get("mixed_over_fp64")
                                               if at_target else None),
        "adjoint_forward_ratio": adj["ratio"] if adj else None,
        "adjoint": adj,
        "batched": batch,
        "helmholtz": helm,
        "uniform_p6": uni,
        "p2p_matrix": mat,
        "stage_ms": stage_ms,
        "roofline": roof,
        "roofline_m2l": roof_m2l,
        "measured_pipe_peaks": pipes,
        "cpu_baseline": cpu_line,
        "e2e": {"value": world * args.npoints / (ms_e2e * 1e-3) / 1e6, "unit": "Mpts/s",
                "h2d_bytes_per_step": 8 * args.npoints, "d2h_bytes_per_step": 8 * args.npoints},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def adjoint_bench(dev, steps=3, ns=200_000, nt=50_000, order=8):
    """Backward/forward time ratio of the differentiable potential: 200k
    sources on the unit sphere perturbed radially by 0.05*N(0,1), 50k
    targets uniform in the shell 2 <= r <= 3, p = 8, mixed precision, loss
    0.5*|phi - phi_ref|^2 with phi_ref the FP64 direct sum at the unperturbed
    positions. Forward = one FMM; backward = transposed-traversal FMM with
    gradient-form evaluation (strength and source-position gradients). Trees
    and schedules are built before timing; times are CUDA events."""
    import torch
    from sumpy_b200 import P2P, LaplaceKernel, drive_fmm
    from sumpy_b200.adjoint import transpose_traversal
    from sumpy_b200.autograd import _Config, _wrangler
    from sumpy_b200.tree import build_all
    rng = np.random.default_rng(7)
    g = rng.standard_normal((3, ns))
    u = g / np.linalg.norm(g, axis=0)
    src = (1 + 0.05 * rng.standard_normal(ns)) * u
    d = rng.standard_normal((3, nt))
    d /= np.linalg.norm(d, axis=0)
    tgt = np.cbrt(8 + 19 * rng.random(nt)) * d
    q = rng.standard_normal(ns)
    knl = [LaplaceKernel(3)]
    (phi_ref,) = P2P(knl)(None, tgt, u, (q,), device=dev)
    cfg = _Config(order, ADJOINT_MAX_PARTICLES, "mixed", dev)
    tree, trav, tcls = build_all(src, tgt, ADJOINT_MAX_PARTICLES)
    tree_t, trav_t, tcls_t = transpose_traversal(tree, trav, tcls)
    wf = _wrangler(cfg, tree, trav, tcls, False, gradient=False)
    wb = _wrangler(cfg, tree_t, trav_t, tcls_t, False, gradient=True)
    qd = torch.as_tensor(q, device=dev)

    def fwd():
        return drive_fmm(None, wf, [qd])[0]

    phi = fwd()
    gd = (phi - phi_ref).contiguous()

    def bwd():
        out = drive_fmm(None, wb, [gd])
        return out[0], qd * torch.stack(out[1:4])

    def tm(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    t_f, t_b = tm(fwd), tm(bwd)
    gq, gsrc = bwd()
    gdn = gd.cpu().numpy()
    psi = P2P(knl, gradient=True)(None, src, tgt, (gdn,), device=dev)
    gq_ref = psi[0]
    gsrc_ref = qd * torch.stack(psi[1:4])
    rel = lambda a, b: float((a - b).norm() / b.norm())
    return {"forward_ms": t_f, "backward_ms": t_b, "ratio": t_b / t_f,
            "grad_strength_relL2_vs_direct": rel(gq, gq_ref),
            "grad_source_pos_relL2_vs_direct": rel(gsrc, gsrc_ref),
            "workload": f"sphere(perturbed) {ns} sources -> shell {nt} targets, p={order}, mixed"}


def batch_problems(nproblems=512):
    """The batched workload: problem i draws from seed 1000 + i its size
    N_i = floor(exp(U(ln 1000, ln 65536))), N_i points U[0,1]^3 (sources =
    targets) and N_i strengths N(0, 1)."""
    srcs, qs = [], []
    for i in range(nproblems):
        rng = np.random.default_rng(1000 + i)
        n = int(np.floor(np.exp(rng.uniform(np.log(1000), np.log(65536)))))
        srcs.append(rng.random((3, n)))
        qs.append(rng.standard_normal(n))
    return srcs, qs


def batched_bench(dev, steps=5, warmup=3, nproblems=512, order=8, nseq=16):
    """512 independent problems (p = 8, mixed, max 32 per box, exclude_self)
    as one forest: CUDA-graph replay and eager launches of the whole batch,
    against the same problems evaluated one drive_fmm at a time (the first
    ``nseq`` problems, rate extrapolated by points). Accuracy: relative L2
    error on 4 problems (512 sampled targets each) against the FP64 direct
    sum. L2 flushed between timed batches."""
    import torch
    from sumpy_b200 import (P2P, LaplaceKernel, SumpyExpansionWrangler,
                            SumpyTreeIndependentDataForWrangler, drive_fmm)
    from sumpy_b200 import _capi
    from sumpy_b200.batch import BatchedLaplaceFMM
    from sumpy_b200.expansion import (
        LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
        LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp)
    from sumpy_b200.tree import build_all
    box = [[0.0, 1.0]] * 3
    srcs, qs = batch_problems(nproblems)
    ntot = sum(q.size for q in qs)
    t0 = time.perf_counter()
    b = BatchedLaplaceFMM(srcs, order=order, max_particles_in_box=BATCH_MAX_PARTICLES,
                          precision="mixed", bbox=box, device=dev, use_graph=True,
                          autotune=True)
    t_build = time.perf_counter() - t0
    w_dev = torch.as_tensor(np.concatenate(qs), device=dev)
    t0 = time.perf_counter()
    b.capture()
    t_capture = time.perf_counter() - t0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def timed(fn):
        for _ in range(warmup):
            fn()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        torch.cuda.synchronize()
        for i in range(steps):
            flush.fill_(float(i))
            evs[i][0].record()
            fn()
            evs[i][1].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in evs) / steps

    ms_graph = timed(lambda: b.evaluate(w_dev))
    b.use_graph = False
    _capi.launch_counter.reset()
    b.evaluate(w_dev)
    launches = _capi.launch_counter.value
    ms_eager = timed(lambda: b.evaluate(w_dev))
    b.use_graph = True
    b.check_status()

    # one problem at a time (what a loop over sumpy FMMs does), first nseq problems
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)
    seq = []
    for i in range(nseq):
        _, trav, tcls = build_all(srcs[i], None, BATCH_MAX_PARTICLES, bbox=box)
        wr = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: order,
                                    translation_classes_data=tcls, precision="mixed",
                                    device=dev)
        seq.append((wr, torch.as_tensor(qs[i], device=dev)))
    nseq_pts = sum(q.numel() for _, q in seq)

    def run_seq():
        for wr, q in seq:
            drive_fmm(None, wr, [q])

    ms_seq = timed(run_seq)
    seq_rate = nseq_pts / (ms_seq * 1e-3) / 1e6

    # accuracy on 4 problems
    pots = b(w_dev)
    errs = []
    rng = np.random.default_rng(5)
    for i in (0, 1, nproblems // 2, nproblems - 1):
        n = qs[i].size
        smp = rng.choice(n, size=min(512, n), replace=False)
        (ref,) = P2P([knl], exclude_self=True)(None, srcs[i][:, smp], srcs[i], (qs[i],),
                                               target_to_source=smp, device=dev)
        ref = ref.cpu().numpy()
        got = pots[i].cpu().numpy()[smp]
        errs.append(float(np.linalg.norm(got - ref) / np.linalg.norm(ref)))
    return {
        "workload": f"{nproblems} problems U[0,1]^3, N_i=floor(exp(U(ln 1000, ln 65536))) "
                    f"(seed 1000+i), p={order}, mixed, exclude_self",
        "total_points": int(ntot), "nboxes": int(b.tree.nboxes),
        "graph": {"ms_per_batch": ms_graph, "Mpts_s": ntot / (ms_graph * 1e-3) / 1e6,
                  "problems_s": nproblems / (ms_graph * 1e-3)},
        "eager": {"ms_per_batch": ms_eager, "Mpts_s": ntot / (ms_eager * 1e-3) / 1e6,
                  "launches_per_batch": launches},
        "one_problem_at_a_time": {
            "Mpts_s": seq_rate, "problems_timed": nseq, "points_timed": int(nseq_pts),
            "ms_for_timed": ms_seq,
            "note": "drive_fmm per problem, warm, same kernels; whole-batch time "
                    "extrapolated by points"},
        "batch_over_one_at_a_time": (ntot / (ms_graph * 1e-3) / 1e6) / seq_rate,
        "m2l_item_groups": b.wrangler.m2l_item_groups,
        "relL2_vs_direct": errs,
        "forest_build_s": round(t_build, 2), "capture_s": round(t_capture, 2),
    }


def matrix_bench(dev, steps=5, warmup=3, n=20_000, nsub=20_000_000):
    """Interaction matrices (P2PMatrixGenerator / P2PMatrixSubsetGenerator):
    the dense n x n Laplace matrix of n = 20k points U[0,1]^3 (3.2 GB of
    FP64 written; HBM-write bound: bytes = 8 per entry), the n/2 x n/2
    Helmholtz matrix (k = 10, 16 bytes per entry), and 20M random index
    pairs. CUDA-event time per call, inputs resident; roofline against the
    measured HBM copy bandwidth."""
    import torch
    from sumpy_b200 import (HelmholtzKernel, LaplaceKernel, P2PMatrixGenerator,
                            P2PMatrixSubsetGenerator)
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = peaks.get("hbm_gbs", 6650.0)
    rng = np.random.default_rng(15)
    pts = torch.as_tensor(rng.random((3, n)), device=dev)

    def tm(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    out = {}
    lap = P2PMatrixGenerator([LaplaceKernel(3)])
    ms = tm(lambda: lap(None, pts, pts, device=dev))
    gbs = 8.0 * n * n / (ms * 1e-3) / 1e9
    out["laplace_dense"] = {"shape": [n, n], "ms": ms, "GB_s": gbs, "frac_hbm": gbs / hbm}
    nh = n // 2
    hel = P2PMatrixGenerator([HelmholtzKernel(3)])
    ms = tm(lambda: hel(None, pts[:, :nh], pts[:, :nh], device=dev, k=10.0))
    gbs = 16.0 * nh * nh / (ms * 1e-3) / 1e9
    out["helmholtz_dense"] = {"shape": [nh, nh], "k": 10.0, "ms": ms, "GB_s": gbs,
                              "frac_hbm": gbs / hbm}
    it = torch.as_tensor(rng.integers(0, n, nsub), device=dev, dtype=torch.int32)
    js = torch.as_tensor(rng.integers(0, n, nsub), device=dev, dtype=torch.int32)
    sub = P2PMatrixSubsetGenerator([LaplaceKernel(3)])
    ms = tm(lambda: sub(None, pts, pts, tgtindices=it, srcindices=js, device=dev))
    out["laplace_subset"] = {"pairs": nsub, "ms": ms, "Gentries_s": nsub / (ms * 1e-3) / 1e9,
                             "GB_s_indices_and_result": 16.0 * nsub / (ms * 1e-3) / 1e9}
    out["peak_hbm_gbs"] = hbm
    return out


def uniform_bench(dev, steps=5, warmup=3, n=20_000, order=6, cpu=True):
    """The reference's own CPU-runnable case: 20k sources and 20k separate
    targets U[0,1]^3 (seeds 15, 18; strengths seed 44), p = 6, max 30 per box,
    FP64 end to end. GPU time (CUDA events), accuracy against the FP64 GPU
    direct sum, and as its CPU baseline the oracle (C + OpenMP, all host
    threads) on the same tree."""
    import torch
    from sumpy_b200 import (P2P, LaplaceKernel, SumpyExpansionWrangler,
                            SumpyTreeIndependentDataForWrangler, drive_fmm)
    from sumpy_b200.expansion import (
        LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
        LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp)
    from sumpy_b200.tree import build_all
    src = np.random.default_rng(15).random((3, n))
    tgt = np.random.default_rng(18).random((3, n))
    q = np.random.default_rng(44).standard_normal(n)
    tree, trav, tcls = build_all(src, tgt, 30)
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl])
    # replayed from a CUDA graph like the headline: at 20k points the eager
    # launch sequence is host-bound, and its timing drifts with the state the
    # earlier workloads leave in the process
    w = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: order,
                               translation_classes_data=tcls, device=dev, cuda_graph=True)
    qd = torch.as_tensor(q, device=dev)
    for _ in range(warmup):
        drive_fmm(None, w, [qd])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        (pot,) = drive_fmm(None, w, [qd])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    (ref,) = P2P([knl])(None, tgt, src, (q,), device=dev)
    out = {"workload": f"uniform {n} sources + {n} targets, p={order}, FP64", "launch": "CUDA graph replay",
           "ms_per_step": ms, "Mpts_s": n / (ms * 1e-3) / 1e6,
           "relL2_vs_direct": float((pot - ref).norm() / ref.norm())}
    if cpu:
        from oracle import oracle as O
        t0 = time.perf_counter()
        O.run_fmm(tree, trav, tcls, order, q)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"ms_per_step": 1e3 * dt, "cores": os.cpu_count(), "kind": "port",
                               "sample": "the same 20k + 20k evaluation, FP64 C/OpenMP oracle"}
        out["gpu_over_cpu"] = 1e3 * dt / ms
    return out


def helmholtz_bench(dev, steps=3, warmup=2, npoints=500_000, order=14, k=10.0,
                    precisions=("mixed", "fp64")):
    """3D Helmholtz (G = e^{ikr}/r, k = 10): 500k points on the unit sphere
    (sources = targets, exclude_self), strengths N(0,1) + i N(0,1), p = 14,
    max 32 per box. Mixed (complex64 near field on FP64 offsets, split-TF32
    M2L on the real embedding) and FP64 forms timed with CUDA events (L2
    flushed between steps); accuracy on 2,048 sampled targets against the
    complex128 GPU direct sum; per-stage times of the mixed form."""
    import torch
    from sumpy_b200 import (P2P, HelmholtzKernel, SumpyExpansionWrangler,
                            SumpyTreeIndependentDataForWrangler, drive_fmm)
    from sumpy_b200.expansion import (
        LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
        LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp)
    from sumpy_b200.tree import build_all
    rng = np.random.default_rng(2025)
    g = rng.standard_normal((3, npoints))
    pts = g / np.linalg.norm(g, axis=0)
    q = rng.standard_normal(npoints) + 1j * rng.standard_normal(npoints)
    t0 = time.perf_counter()
    tree, trav, tcls = build_all(pts, None, HELMHOLTZ_MAX_PARTICLES)
    t_tree = time.perf_counter() - t0
    knl = HelmholtzKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)
    qd = torch.as_tensor(q, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def timed(fn):
        for _ in range(warmup):
            fn()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        torch.cuda.synchronize()
        for i in range(steps):
            flush.fill_(float(i))
            evs[i][0].record()
            fn()
            evs[i][1].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in evs) / steps

    smp = rng.choice(npoints, size=2048, replace=False)
    (ref,) = P2P([knl], exclude_self=True)(None, pts[:, smp], pts, (q,),
                                           target_to_source=smp, device=dev, k=k)
    ref = ref.cpu().numpy()
    out = {"workload": f"unit sphere n={npoints}, k={k}, p={order}, complex strengths, "
                       f"exclude_self, max {HELMHOLTZ_MAX_PARTICLES} per box",
           "tree_build_s": round(t_tree, 3), "m2l_entries": int(len(trav.from_sep_siblings_lists))}
    for precision in precisions:
        t0 = time.perf_counter()
        w = SumpyExpansionWrangler(ti, trav, np.complex128, lambda *a: order,
                                   kernel_extra_kwargs={"k": k}, translation_classes_data=tcls,
                                   precision=precision, device=dev)
        (pot,) = drive_fmm(None, w, [qd])
        torch.cuda.synchronize()
        setup = time.perf_counter() - t0
        if precision == "mixed":
            from sumpy_b200.autotune import tune_m2l_item_groups
            tune_m2l_item_groups(w, lambda: drive_fmm(None, w, [qd]))
        ms = timed(lambda: drive_fmm(None, w, [qd]))
        w.check_status()
        got = pot.cpu().numpy()[smp]
        out[precision] = {"Mpts_s": npoints / (ms * 1e-3) / 1e6, "ms_per_step": ms,
                          "m2l_item_groups": w.m2l_item_groups,
                          "relL2_vs_direct": float(np.linalg.norm(got - ref) /
                                                   np.linalg.norm(ref)),
                          "setup_s": round(setup, 2)}
        if precision == "mixed":
            out["stage_ms_mixed"] = stage_breakdown(w, trav, qd, dev, roofline=False)[0]
            # adjoint with respect to the strengths: the FMM on the transposed
            # traversal (sumpy_b200.autograd.HelmholtzFMM's backward)
            from sumpy_b200.adjoint import transpose_traversal
            import gc
            # the eager launch sequence allocates per call: start from a
            # collected caching allocator, as the forward timing did
            gc.collect()
            torch.cuda.empty_cache()
            tree_t, trav_t, tcls_t = transpose_traversal(tree, trav, tcls)
            wa = SumpyExpansionWrangler(ti, trav_t, np.complex128, lambda *a: order,
                                        kernel_extra_kwargs={"k": k},
                                        translation_classes_data=tcls_t,
                                        precision=precision, device=dev)
            gd = pot.conj().contiguous()
            drive_fmm(None, wa, [gd])
            ms_adj = timed(lambda: drive_fmm(None, wa, [gd]))
            out["adjoint_forward_ratio_mixed"] = ms_adj / ms
            del wa
        del w
        torch.cuda.empty_cache()
    if "fp64" in out and "mixed" in out:
        out["mixed_over_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    return out


def stage_breakdown(w, trav, q_dev, dev, roofline=True, pipe_peaks=None):
    """Per-stage device times of one FMM (CUDA events between the wrangler
    calls on the launching stream) and the roofline of the dominant stage."""
    import torch
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    def one_pass():
        ev = []

        def mark(name):
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            ev.append((name, e))

        torch.cuda.synchronize()
        mark("start")
        qd = w.reorder_sources(q_dev)
        mark("reorder")
        mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qd])
        mark("p2m")
        mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                  trav.source_parent_boxes, mp)
        mark("m2m")
        w.eval_direct(None, trav.target_boxes, trav.neighbor_source_boxes_starts,
                      trav.neighbor_source_boxes_lists, [qd])
        mark("p2p")
        loc = w.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                                   trav.target_or_target_parent_boxes,
                                   trav.from_sep_siblings_starts, trav.from_sep_siblings_lists,
                                   mp)
        mark("m2l")
        w.eval_multipoles(None, trav.target_boxes_sep_smaller_by_source_level,
                          trav.from_sep_smaller_by_level, mp)
        mark("m2p")
        pl = w.form_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                           trav.target_or_target_parent_boxes, trav.from_sep_bigger_starts,
                           trav.from_sep_bigger_lists, [qd])
        mark("p2l")
        loc = w.refine_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                              trav.target_or_target_parent_boxes, loc + pl)
        mark("l2l")
        w.eval_locals(None, trav.level_start_target_box_nrs, trav.target_boxes, loc)
        mark("l2p")
        torch.cuda.synchronize()
        return {n1: e0.elapsed_time(e1) for (n0, e0), (n1, e1) in zip(ev, ev[1:])}

    # warm (clocks up after the host-side phases), then the per-stage median of 3 passes
    one_pass()
    passes = [one_pass() for _ in range(3)]
    stage = {k: float(np.median([ps[k] for ps in passes])) for k in passes[0]}
    if not roofline:
        return stage, None, None

    # algorithmic work per stage (the units the stage processes)
    tree = w.tree
    n = (w.level_orders[0] + 1) ** 2
    tb = trav.target_boxes
    ns = trav.neighbor_source_boxes_starts
    nl = trav.neighbor_source_boxes_lists
    cnt_t = tree.box_target_counts_nonchild[tb].astype(np.int64)
    src_per_list = np.add.reduceat(
        tree.box_source_counts_nonchild[nl].astype(np.int64), ns[:-1]) if len(nl) else 0
    empty = np.diff(ns) == 0
    src_per_list = np.where(empty, 0, src_per_list)
    pairs = int((cnt_t * src_per_list).sum()) - (tree.ntargets if tree.sources_are_targets else 0)
    m2l_entries = len(trav.from_sep_siblings_lists)
    m2p_pairs = 0
    for tbs, csr in zip(trav.target_boxes_sep_smaller_by_source_level,
                        trav.from_sep_smaller_by_level):
        if len(tbs):
            m2p_pairs += int((tree.box_target_counts_nonchild[np.asarray(tbs)].astype(np.int64)
                              * np.diff(np.asarray(csr.starts))).sum())
    mixed = w.precision == "mixed"
    kernels = {
        "m2l": "m2l_tf32x3_kernel" if mixed else "m2l_f64_kernel<128>",
        "m2p": "m2p_mixed_kernel<P>" if mixed else "m2p_reg_kernel<P>",
        "p2p": "p2p_csr_kernel<mixed>" if mixed else "p2p_csr_kernel<f64>",
        "p2l": "p2l_mixed_kernel<P>" if mixed else "p2l_reg_kernel<P>",
    }
    peak_bf16 = peaks.get("bf16_tflops", 1590.0)
    peak_hbm = peaks.get("hbm_gbs", 6650.0)
    src = "MEASURED_PEAKS.json (of measured)" if peaks else "fallback"

    def m2l_roof():
        ach = 2 * n * n * m2l_entries / (stage["m2l"] * 1e-3) / 1e12
        r = {"kernel": kernels["m2l"], "bound": "tensor", "achieved": ach, "peak": peak_bf16,
             "unit": "TFLOP/s", "frac": ach / peak_bf16, "traffic": None,
             "peak_source": "bf16_tflops " + src,
             "work": {"flops": 2 * n * n * m2l_entries, "entries": m2l_entries,
                      "per_unit": "2 n^2 flops per List-2 entry"}}
        if mixed:
            r["note"] = ("tcgen05 split-TF32 GEMM; algorithmic flops = 2 n^2 per List-2 entry "
                         "(not the x3 split products, empty slots or padding); the stage time "
                         "includes the TF32 split pre-pass")
        # dram__bytes_read.sum + dram__bytes_write.sum of this launch on the 1M-point
        # workload, one ncu capture per leaf size (profiles/m2l_tf32x3_sphere_plummer_1M_p10.md)
        captured = {32: 1.227e9 + 0.195e9, 96: 256.6e6 + 38.4e6}
        if mixed and tree.nsources == NPOINTS and n == (ORDER + 1) ** 2 and \
                MAX_PARTICLES in captured and \
                int(tree.box_source_counts_nonchild.max()) <= MAX_PARTICLES:
            r["traffic"] = captured[MAX_PARTICLES]
            r["traffic_unit"] = "bytes per launch (ncu capture)"
        return r

    # the dominant stage, with the stage's own roofline: M2L the tensor cores,
    # P2P the FP32 (mixed) / FP64 pipe, M2P and P2L HBM with 40 B per
    # evaluation (one target's or source's coordinates and value) -- they are
    # compute-bound at this order, so their FLOP/s against the measured
    # FP32/FP64 GEMM rate as well
    dom = max(("m2l", "m2p", "p2p", "p2l"), key=lambda k: stage[k])
    fp = pipe_peaks or {}
    if dom == "m2l":
        roof = m2l_roof()
    elif dom == "p2p":
        pk = fp.get("fp32_tflops" if mixed else "fp64_tflops")
        ach = 11 * pairs / (stage["p2p"] * 1e-3) / 1e12
        roof = {"kernel": kernels["p2p"], "bound": "fp32" if mixed else "fp64",
                "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": (ach / pk) if pk else None, "traffic": None,
                "peak_source": "torch.matmul FP32/FP64 GEMM measured in this run",
                "work": {"flops": 11 * pairs, "pairs": pairs, "per_unit": "11 flops per pair"}}
    else:
        units = m2p_pairs if dom == "m2p" else int(
            tree.box_source_counts_nonchild[np.asarray(trav.from_sep_bigger_lists)].sum())
        nbytes = 40 * units
        flops = units * 10 * n
        ach = nbytes / (stage[dom] * 1e-3) / 1e9
        pk = fp.get("fp32_tflops" if mixed else "fp64_tflops")
        ftf = flops / (stage[dom] * 1e-3) / 1e12
        roof = {"kernel": kernels[dom], "bound": "hbm", "achieved": ach, "peak": peak_hbm,
                "unit": "GB/s", "frac": ach / peak_hbm, "traffic": None,
                "peak_source": "hbm_gbs " + src,
                "work": {"bytes": nbytes, "evaluations": units,
                         "per_unit": "40 B per (target, List-3 box) / (List-4 source, box)"},
                "flops": {"achieved_tflops": ftf, "peak_tflops": pk,
                          "per_unit": "~10 n flops per evaluation",
                          "frac": (ftf / pk) if pk else None}}
    roof["dominant_stage"] = dom
    return stage, roof, m2l_roof()


def pipe_peaks_measured(dev):
    """FP32 and FP64 CUDA-core rates measured here: torch.matmul GEMMs with
    TF32 disabled (cuBLAS SGEMM / DGEMM), best of 5, CUDA events."""
    import torch
    out = {}
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for name, dt, m in (("fp32_tflops", torch.float32, 8192),
                            ("fp64_tflops", torch.float64, 4096)):
            a = torch.randn(m, m, device=dev, dtype=dt)
            b = torch.randn(m, m, device=dev, dtype=dt)
            torch.matmul(a, b)
            best = None
            for _ in range(5):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                torch.matmul(a, b)
                e1.record()
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1)
                best = t if best is None else min(best, t)
            out[name] = 2.0 * m ** 3 / (best * 1e-3) / 1e12
            del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return out


if __name__ == "__main__":
    main()
