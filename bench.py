"""Benchmark of the B200 SAL-gradient treecode.

One step = one solve of the SAL gradient (both components at every cell) of
the field batch on a device-resident grid: the code.f90 path (dual tree
traversal) on the 2,313,486-cell MPAS-like synthetic grid, d = 8, theta = 0.7,
leaves < 200 points.  Inputs are seeded synthetic stand-ins of the reference's
MPAS CSVs (not distributed with it).

  python bench.py [--gpus N --steps K --warmup W] [--form ref|accurate] [--impl reference]

Multi-GPU runs are independent replicas (one grid per GPU, no collective in
the solve): value = cells * fields * steps * world / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sal-fort_b200"))
sys.path.insert(0, ROOT)

METRIC = "SAL-grad evals/s @2.3M cells, rel-L2 err vs FP64 direct; p50/p99 solve latency"
FLOPS_PER_PAIR = 31.0      # one kernel evaluation incl. 2 accumulates ('/' and sqrt count 1)
FLOPS_PER_MAC = 2.0


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="ref", choices=["ref", "accurate"])
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--degree", type=int, default=8)
    ap.add_argument("--thresh", type=int, default=200)
    ap.add_argument("--theta", type=float, default=0.7)
    ap.add_argument("--targets", type=int, default=10000)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_problem(args, device):
    from salgpu import synth
    t0 = time.perf_counter()
    g = synth.config_grid(args.config, device=device)
    h = synth.config_ssh(args.config, g, nfields=1, device=device)
    return g, h, time.perf_counter() - t0


def cpu_baseline(args, g, h, sample_seconds):
    """The oracle (a line-faithful C restatement of the reference) on a random
    seeded sample of the interaction list with all host threads; the full
    solve time is extrapolated by the sampled fraction of the list."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    ot = O.tree_traverse(g.xs, g.ys, g.zs, args.thresh)
    L = O.dual_tree_traversal(ot, args.theta, args.thresh)
    setup = time.perf_counter() - t0
    pairs_all, macs_all = O.dtt_work(ot, L, args.degree)
    rng = np.random.default_rng(1234)
    # pick the sample size from a short calibration run
    frac = 0.002
    while True:
        sel = np.sort(rng.choice(len(L), max(1, int(frac * len(L))), replace=False))
        t1 = time.perf_counter()
        O.fast_sum(ot, L[sel], g.xs, g.ys, g.zs, g.areas, h, args.degree, nranks=cores)
        dt = time.perf_counter() - t1
        if dt > 0.25 * sample_seconds or frac >= 1.0:
            break
        frac = min(1.0, frac * max(2.0, 0.5 * sample_seconds / max(dt, 1e-3)))
    pairs_s, macs_s = O.dtt_work(ot, L[sel], args.degree)
    f_work = (pairs_s.sum() + macs_s) / (pairs_all.sum() + macs_all)
    f_list = len(sel) / len(L)
    t_full = dt / f_list
    return {"value": g.n / t_full, "unit": "evals/s", "cores": cores, "kind": "port",
            "sample": f"{len(sel)} of {len(L)} DTT interactions ({100 * f_list:.2f}%, seeded uniform; "
                      f"{100 * f_work:.2f}% of pair+MAC work), {dt:.1f} s on {cores} threads, "
                      f"full solve extrapolated to {t_full:.1f} s; host setup {setup:.1f} s",
            "extrapolated_solve_s": t_full}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    g, h, _ = make_problem(args, "cuda" if _cuda() else "cpu")
    cb = cpu_baseline(args, g, h[0], args.cpu_seconds)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "evals/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * cb["extrapolated_solve_s"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded Fibonacci ocean grid + spherical-harmonic SSH",
            "config": {"workload": f"{args.config}: {g.n} cells, dual tree traversal (code.f90 fast_sum), "
                                   f"d={args.degree}, theta={args.theta}, leaf<{args.thresh}, 1 field",
                       "cells": g.n, "fields": 1},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def main():
    args = _args()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    import salgpu as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    dev = torch.device("cuda", local)
    form = {"ref": S.FORM_REF, "accurate": S.FORM_ACCURATE}[args.form]

    g, h, t_gen = make_problem(args, dev)
    t0 = time.perf_counter()
    tree = S.tree_traverse(g.xs, g.ys, g.zs, g.n, args.thresh)
    inter = S.dual_tree_traversal(tree, args.theta, args.thresh)
    t_lists = time.perf_counter() - t0
    grid = S.Grid(tree, g.xs, g.ys, g.zs, g.areas, args.degree, S.MODE_DTT, inter, device=local)
    st = grid.stats()
    ssh = torch.tensor(h[0], device=dev)
    ox = torch.empty_like(ssh)
    oy = torch.empty_like(ssh)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    for _ in range(args.warmup):
        grid.solve(ssh, form=form, out=(ox, oy))
    torch.cuda.synchronize()
    grid.sync()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clk = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    for k in range(args.steps):
        flush.fill_(float(k))                 # evicts L2 between timed solves
        starts[k].record(stream)
        grid.solve(ssh, form=form, out=(ox, oy))
        ends[k].record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    if world > 1:
        dist.barrier()
    grid.sync()
    per = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    total_ms = float(per.sum())
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())

    # ---- per-pass device times (separate instrumented pass)
    grid.timing(1)
    for k in range(max(3, args.steps // 2)):
        flush.fill_(float(k))
        grid.solve(ssh, form=form, out=(ox, oy))
    phase, nsol = grid.timing(0)
    leaf_ms = phase[2] / nsol
    proxy_ms = phase[1] / nsol
    up_ms = phase[0] / nsol

    # ---- accuracy vs the FP64 direct sum on sampled targets
    tg = np.sort(np.random.default_rng(99).choice(g.n, min(args.targets, g.n), replace=False)).astype(np.int32)
    T = lambda a: torch.tensor(a, device=dev)
    dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * h[0]), T(tg))
    tgt = torch.tensor(tg, device=dev, dtype=torch.long)
    ex, ey = ox[tgt] - dx, oy[tgt] - dy
    rel = float(torch.sqrt((ex * ex + ey * ey).sum() / (dx * dx + dy * dy).sum()))
    mx = float(torch.sqrt(ex * ex + ey * ey).max() / torch.sqrt(dx * dx + dy * dy).max())

    # ---- end to end through the host-buffer C-ABI entry point (fast_sum)
    h_ssh = torch.tensor(h[0]).pin_memory().numpy()
    h_x = torch.zeros(g.n, dtype=torch.float64).pin_memory().numpy()
    h_y = torch.zeros(g.n, dtype=torch.float64).pin_memory().numpy()
    for _ in range(2):
        grid.fast_sum_host(h_ssh, h_x, h_y, form)
    e2e_t = []
    for _ in range(max(3, args.steps // 2)):
        t1 = time.perf_counter()
        grid.fast_sum_host(h_ssh, h_x, h_y, form)
        e2e_t.append(time.perf_counter() - t1)
    e2e_val = g.n / float(np.mean(e2e_t))

    peak64 = S.fma_peak(64)
    leaf_flops = FLOPS_PER_PAIR * (st["pairs_pp"] + st["pairs_pc"]) + 2 * FLOPS_PER_MAC * st["macs_down"]
    achieved = leaf_flops / (leaf_ms * 1e-3) / 1e12
    total_flops = (FLOPS_PER_PAIR * (st["pairs_pp"] + st["pairs_pc"] + st["pairs_cp"] + st["pairs_cc"])
                   + FLOPS_PER_MAC * (st["macs_up"] + 2 * st["macs_down"]))

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline(args, g, h[0], args.cpu_seconds)

    if rank == 0:
        value = g.n * args.steps * world / (total_ms * 1e-3)
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded Fibonacci ocean grid + spherical-harmonic SSH (stand-in for the MPAS CSVs)",
            "config": {"workload": f"{args.config}: {g.n} cells, dual tree traversal (code.f90 fast_sum), "
                                   f"d={args.degree}, theta={args.theta}, leaf<{args.thresh}, 1 field, "
                                   f"{args.form} FP64 form", "cells": g.n, "fields": 1, "form": args.form,
                       "parallelism": f"replicas x{world}", "l2": "flushed (256 MB write) between timed solves"},
            "latency_ms": {"p50": float(np.percentile(per, 50)), "p99": float(np.percentile(per, 99))},
            "accuracy": {"rel_l2_vs_fp64_direct": rel, "max_err_over_max_ref": mx, "targets": len(tg)},
            "roofline": {"bound": "fp64", "kernel": "eval_kernel<leaf> (PP+PC pairs + DOWN interpolation)",
                         "achieved": achieved, "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                         "peak_source": "sal_fma_peak(64) on this GPU (FP64 FMA pipe; MEASURED_PEAKS.json has no FP64 figure)",
                         "traffic": None, "leaf_ms": leaf_ms, "proxy_ms": proxy_ms, "prep_upward_ms": up_ms,
                         "algorithmic_tflop_per_solve": total_flops / 1e12},
            "work": {k: st[k] for k in ("pairs_pp", "pairs_pc", "pairs_cp", "pairs_cc", "macs_up", "macs_down")},
            "setup_s": {"grid_generation": t_gen, "tree_and_lists": t_lists, "plan_and_upload": st["setup_seconds"]},
            "e2e": {"value": e2e_val, "unit": "evals/s", "h2d_bytes_per_step": 8 * g.n,
                    "d2h_bytes_per_step": 16 * g.n, "api": "sal_fast_sum_host (host buffers)"},
            "clocks": clocks,
            "gpu_launches": 6 * args.steps,
        }
        if cb:
            line["cpu_baseline"] = cb
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
