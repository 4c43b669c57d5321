"""Benchmark of the B200 SAL-gradient treecode.

One step = one solve of the SAL gradient (both components at every cell) for
the step's batch of SSH fields on a device-resident grid: the code.f90 path
(dual tree traversal) on the 2,313,486-cell MPAS-like synthetic grid, d = 8,
theta = 0.7, leaves < 200 points.  Inputs are seeded synthetic stand-ins for
the reference's MPAS CSVs (not distributed with it).

  python bench.py [--gpus N --steps K --warmup W] [--form mixed|ref|accurate] [--fields F]
  python bench.py --impl reference          # the CPU oracle port, same metric

Default: the batched mixed-precision form, 64 fields per step (cfg3); the plain
FP64 form of the same grid is timed in the same run and reported beside it.
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
    ap.add_argument("--form", default="mixed", choices=["ref", "accurate", "mixed"])
    ap.add_argument("--fields", type=int, default=None)
    ap.add_argument("--config", default=None)
    ap.add_argument("--degree", type=int, default=8)
    ap.add_argument("--thresh", type=int, default=200)
    ap.add_argument("--theta", type=float, default=0.7)
    ap.add_argument("--targets", type=int, default=10000)
    ap.add_argument("--check-fields", type=int, default=64, help="fields checked against the FP64 direct sum")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=8.0)
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-host", action="store_true", help="serving requests carry host arrays")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-tune", default=None,
                    help="batched-form settings of the served grids as name=value,... (default: the server's)")
    ap.add_argument("--no-autotune", action="store_true", help="time the batched form's default settings")
    ap.add_argument("--tune", default=None,
                    help="batched form's settings as name=value,... (sal_tune fields); replaces the autotuner")
    ap.add_argument("--tile-store", default="auto", choices=("auto", "0"),
                    help="also time the FP16 leaf pass replaying its kernel tiles from device memory "
                         "(sal_tune.tile_store) beside the headline; auto: when the device has room for them")
    ap.add_argument("--no-stt", action="store_true", help="skip the mom6_code.f90 path measurement")
    ap.add_argument("--cpu-table", action="store_true", help="time the oracle on cfg0/cfg1/cfg2 and exit")
    a = ap.parse_args()
    if a.fields is None:
        a.fields = 64 if a.form == "mixed" else 1
    if a.config is None:
        a.config = "cfg3" if a.fields > 1 else "cfg2"
    return a


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
    h = synth.config_ssh(args.config, g, nfields=args.fields, device=device)
    return g, h, time.perf_counter() - t0


RANK_SPLIT = 8      # the reference's MPI split of the DTT list, MOD(i, P) == rank (fast_sum_module.f90:304)


def cpu_shares(args, g):
    """The oracle's tree and DTT list of the grid, split into the RANK_SPLIT
    shares MOD(i, P) == r of fast_sum_module.f90:304, each with its fraction of
    the solve's pair + MAC work."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    ot = O.tree_traverse(g.xs, g.ys, g.zs, args.thresh)
    L = O.dual_tree_traversal(ot, args.theta, args.thresh)
    setup = time.perf_counter() - t0
    pairs_all, macs_all = O.dtt_work(ot, L, args.degree)
    i = np.arange(1, len(L) + 1)
    shares, frac = [], []
    for r in range(RANK_SPLIT):
        sh = L[(i % RANK_SPLIT) == r]
        p, m = O.dtt_work(ot, sh, args.degree)
        shares.append(sh)
        frac.append((p.sum() + m) / (pairs_all.sum() + macs_all))
    return ot, L, shares, frac, setup


def solve_share(args, g, h, ot, share, cores):
    """One rank's share of a one-field solve: the oracle's fast_sum (a
    line-faithful C restatement of fast_sum_module.f90) over the share with all
    host threads."""
    from oracle import oracle as O
    t1 = time.perf_counter()
    O.fast_sum(ot, share, g.xs, g.ys, g.zs, g.areas, h, args.degree, nranks=cores)
    return time.perf_counter() - t1


def cpu_baseline(args, g, h, sample_seconds):
    """The oracle on the host's cores, measured (not extrapolated): rank
    shares of one field's solve are timed one after another until
    sample_seconds have passed or all RANK_SPLIT shares (a complete solve) are
    done.  evals/s = cells x (work fraction of the timed shares) / time.  The
    reference solves one field per call, so its evals/s is the same for any
    number of fields."""
    cores = os.cpu_count() or 1
    ot, L, shares, frac, setup = cpu_shares(args, g)
    t, f, done = 0.0, 0.0, 0
    for r in range(RANK_SPLIT):
        t += solve_share(args, g, h, ot, shares[r], cores)
        f += frac[r]
        done += 1
        if t >= sample_seconds:
            break
    whole = done == RANK_SPLIT
    return {"value": g.n * f / t, "unit": "evals/s", "cores": cores, "kind": "port",
            "sample": (f"one field, {done} of the {RANK_SPLIT} rank shares MOD(i,{RANK_SPLIT})==r of the "
                       f"{len(L)}-interaction DTT list ({100 * f:.1f}% of the pair+MAC work"
                       f"{', a complete solve' if whole else ''}), {t:.1f} s measured on {cores} threads; "
                       f"host tree + list setup {setup:.1f} s"),
            "solve_s": t / f, "measured_s": t, "complete_solve": whole}


def workload_name(args, n):
    form = {"ref": "plain FP64 (reference operation order)", "accurate": "FP64 accurate form",
            "mixed": "batched mixed precision: FP32 kernel tiles, TF32 or (autotuner's choice) scaled FP16 hi/lo "
                     "tensor-core contractions (tcgen05), FP64 self pairs"}[args.form]
    return (f"{args.config}: {n} cells x {args.fields} SSH fields, dual tree traversal (code.f90 fast_sum), "
            f"d={args.degree}, theta={args.theta}, leaf<{args.thresh}; {form}")


def run_reference(args):
    """The reference's CPU algorithm (the oracle port; no Fortran compiler
    exists on these machines) on the host's cores.  One step is one rank's
    share MOD(i, 8) == r of a one-field solve of the same grid (the reference's
    own MPI decomposition of the list, fast_sum_module.f90:304), r cycling
    through the eight shares, solved with every host thread; every step is
    timed whole.  value = cells x (work fraction of the timed shares) / time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    args.fields = 1
    cores = os.cpu_count() or 1
    g, h, _ = make_problem(args, "cuda" if _cuda() else "cpu")
    ot, L, shares, frac, setup = cpu_shares(args, g)
    for k in range(args.warmup):
        solve_share(args, g, h[0], ot, shares[k % RANK_SPLIT], cores)
    times, f = [], 0.0
    for k in range(args.steps):
        r = k % RANK_SPLIT
        times.append(solve_share(args, g, h[0], ot, shares[r], cores))
        f += frac[r]
    total = float(np.sum(times))
    value = g.n * f / total
    cb = {"value": value, "unit": "evals/s", "cores": cores, "kind": "port",
          "sample": (f"each step one of the {RANK_SPLIT} rank shares MOD(i,{RANK_SPLIT})==r of the "
                     f"{len(L)}-interaction DTT list of one field (steps cover {f:.2f} complete solves), "
                     f"oracle fast_sum on {cores} threads; host tree + list setup {setup:.1f} s")}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded Fibonacci ocean grid + spherical-harmonic SSH",
            "config": {"workload": workload_name(args, g.n) + " (reference algorithm, one field per call)",
                       "cells": g.n, "fields": 1, "step": f"one rank share (1/{RANK_SPLIT} of the list)"},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_table(args):
    """BASELINE.md's CPU table: the reference's algorithms (the oracle port)
    on the host's cores, setup and solve timed apart, each with its error
    against the FP64 direct sum (GPU direct sum when a GPU is present, else
    the oracle's).  Prints one JSON line."""
    from oracle import oracle as O
    from salgpu import synth
    cores = os.cpu_count() or 1
    rows = []

    def err_vs_direct(g, h, x, y, tg):
        if _cuda():
            import torch
            import salgpu as S
            T = lambda a: torch.tensor(a, device="cuda")
            dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * h), T(tg.astype(np.int32)))
            dx, dy = dx.cpu().numpy(), dy.cpu().numpy()
        else:
            dx, dy = O.direct_sum(g.xs, g.ys, g.zs, g.areas, h, tg, cores)
        ex, ey = x[tg] - dx, y[tg] - dy
        return (float(np.sqrt(np.sum(ex * ex + ey * ey) / np.sum(dx * dx + dy * dy))),
                float(np.max(np.hypot(ex, ey)) / np.max(np.hypot(dx, dy))))

    def sample(g, k, seed=99):
        return np.sort(np.random.default_rng(seed).choice(g.n, min(k, g.n), replace=False))

    # cfg0: DTT (code.f90), 1 thread and all threads
    g = synth.config_grid("cfg0")
    h = synth.config_ssh("cfg0", g)[0]
    t0 = time.perf_counter()
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 100)
    L = O.dual_tree_traversal(ot, 0.7, 100)
    setup = time.perf_counter() - t0
    for th in (1, cores):
        t0 = time.perf_counter()
        x, y = O.fast_sum(ot, L, g.xs, g.ys, g.zs, g.areas, h, 8, nranks=th)
        dt = time.perf_counter() - t0
        e, m = err_vs_direct(g, h, x, y, np.arange(g.n))
        rows.append({"config": "cfg0", "path": "DTT fast_sum", "cells": g.n, "threads": th, "setup_s": setup,
                     "solve_s": dt, "evals_per_s": g.n / dt, "rel_l2_vs_direct": e, "max_over_max": m,
                     "targets": g.n})
    # cfg1: STT (mom6_code.f90), both proxy-weight orientations, all threads
    g = synth.config_grid("cfg1")
    h = synth.config_ssh("cfg1", g, seed=13)[0]
    t0 = time.perf_counter()
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 200)
    ppan = O.assign_points_to_panels(ot, g.xs, g.ys, g.zs)
    pc, pp = O.single_tree_traversal(ot, 0.7, 200, g.xs, g.ys, g.zs)
    setup = time.perf_counter() - t0
    for tr in (True, False):
        t0 = time.perf_counter()
        w = O.proxy_source_compute(ot, ppan, g.xs, g.ys, g.zs, h, g.areas, 8, tr, nthreads=cores)
        t1 = time.perf_counter()
        x, y = O.pc_compute(ot, pc, g.xs, g.ys, g.zs, 8, w, nthreads=cores)
        t2 = time.perf_counter()
        O.pp_compute(ot, pp, g.xs, g.ys, g.zs, g.areas, h, out=(x, y), nthreads=cores)
        t3 = time.perf_counter()
        e, m = err_vs_direct(g, h, x, y, sample(g, 10000))
        rows.append({"config": "cfg1", "path": "STT mom6 " + ("ref_compat (transposed weights)" if tr else "correct"),
                     "cells": g.n, "threads": cores, "setup_s": setup, "solve_s": t3 - t0,
                     "phases_s": {"proxy_source_compute": t1 - t0, "pc_compute": t2 - t1, "pp_compute": t3 - t2},
                     "evals_per_s": g.n / (t3 - t0), "rel_l2_vs_direct": e, "max_over_max": m, "targets": 10000,
                     "pc_entries": len(pc), "pp_entries": len(pp)})
    # cfg2: DTT, all threads, a complete solve
    g = synth.config_grid("cfg2")
    h = synth.config_ssh("cfg2", g, seed=17)[0]
    t0 = time.perf_counter()
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 200)
    L = O.dual_tree_traversal(ot, 0.7, 200)
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    x, y = O.fast_sum(ot, L, g.xs, g.ys, g.zs, g.areas, h, 8, nranks=cores)
    dt = time.perf_counter() - t0
    e, m = err_vs_direct(g, h, x, y, sample(g, 10000))
    rows.append({"config": "cfg2", "path": "DTT fast_sum", "cells": g.n, "threads": cores, "setup_s": setup,
                 "solve_s": dt, "evals_per_s": g.n / dt, "rel_l2_vs_direct": e, "max_over_max": m,
                 "targets": 10000})
    print(json.dumps({"cpu_table": rows, "kind": "port", "cores": cores}), flush=True)


def stt_run(args, S, torch, dev):
    """The mom6_code.f90 path (single tree traversal) on the 0.25 degree
    1440 x 720 lon-lat ocean grid (cfg1), plain FP64 in the reference's
    operation order (ref_compat weights): device time of one solve
    (proxy_source_compute + pc_compute + pp_compute as one sal_solve on the
    grid), and end to end through the reference-signature entry points with
    host arrays, as mom6_code.f90:272-312 calls them (the first call builds
    and caches the device grids; the timed calls reuse them).  The oracle's
    time on the host's cores for the same three calls comes from a bounded
    sample of targets."""
    from salgpu import synth
    g = synth.config_grid("cfg1", device=dev)
    h = synth.config_ssh("cfg1", g, nfields=1, seed=13, device=dev)[0]
    t0 = time.perf_counter()
    tree = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 200)
    ppan = S.assign_points_to_panels(tree, g.xs, g.ys, g.zs)
    pc, pp = S.single_tree_traversal(tree, 0.7, 200, g.xs, g.ys, g.zs)
    t_lists = time.perf_counter() - t0
    grid = S.mom6_grid(tree, pc, pp, g.xs, g.ys, g.zs, g.areas, 8, ref_compat=True, device=dev.index or 0)
    ssh = torch.tensor(h, device=dev)
    out = (torch.empty_like(ssh), torch.empty_like(ssh))
    for _ in range(2):
        grid.solve(ssh, out=out)
    stream = torch.cuda.current_stream(dev)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e[0].record(stream)
    for _ in range(5):
        grid.solve(ssh, out=out)
    e[1].record(stream)
    torch.cuda.synchronize()
    dev_ms = e[0].elapsed_time(e[1]) / 5
    grid.timing(1)
    for _ in range(3):
        grid.solve(ssh, out=out)
    phase, nsol = grid.timing(0)
    st = grid.stats()
    del grid
    # end to end: the three reference-signature calls on host arrays
    P = (8 + 1) ** 2
    npn = tree.npanels
    w = np.zeros(P * npn)
    sx, sy = np.zeros(g.n), np.zeros(g.n)
    S.dropin_config(S.FORM_REF, S.MODE_STT_REF_COMPAT)
    t0 = time.perf_counter()
    S.proxy_source_compute(w, tree, ppan, g.xs, g.ys, g.zs, h, g.areas, 8, g.n)
    S.pc_compute(sx, sy, pc, tree, g.xs, g.ys, g.zs, 8, w)
    S.pp_compute(sx, sy, pp, tree, g.xs, g.ys, g.zs, g.areas, h)
    first = time.perf_counter() - t0
    reps = []
    for _ in range(3):
        w[:] = 0.0
        sx[:] = 0.0
        sy[:] = 0.0
        t0 = time.perf_counter()
        S.proxy_source_compute(w, tree, ppan, g.xs, g.ys, g.zs, h, g.areas, 8, g.n)
        S.pc_compute(sx, sy, pc, tree, g.xs, g.ys, g.zs, 8, w)
        S.pp_compute(sx, sy, pp, tree, g.xs, g.ys, g.zs, g.areas, h)
        reps.append(time.perf_counter() - t0)
    S.dropin_release()
    e2e_s = float(np.median(reps))
    pairs = st["pairs_pp"] + st["pairs_pc"]
    out = {"workload": f"cfg1: {g.n} lon-lat ocean cells (1440 x 720 before the mask), single tree traversal "
                       "(mom6_code.f90), d=8, theta=0.7, leaf<200, plain FP64, ref_compat weights",
           "cells": g.n, "pc_entries": len(pc), "pp_entries": len(pp), "kernel_pairs": pairs,
           "device_ms": dev_ms, "evals_per_s": g.n / (dev_ms * 1e-3),
           "passes_ms": {"prep_upward": phase[0] / nsol, "leaf_pc_pp": phase[2] / nsol},
           "fp64_tflops_leaf": FLOPS_PER_PAIR * pairs / (phase[2] / nsol * 1e-3) / 1e12,
           "e2e": {"value": g.n / e2e_s, "unit": "evals/s", "seconds": e2e_s, "first_call_s": first,
                   "api": "sal_mom6_proxy_source_compute + sal_mom6_pc_compute + sal_mom6_pp_compute, host arrays"},
           "setup_s": {"tree_and_lists": t_lists, "plan_and_upload": st["setup_seconds"]}}
    if not args.no_cpu:
        # the oracle's three calls on every list entry of a seeded target
        # sample, all host threads; the solve time scales by the sampled share
        # of the entries
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        ot = O.tree_traverse(g.xs, g.ys, g.zs, 200)
        opan = O.assign_points_to_panels(ot, g.xs, g.ys, g.zs)
        t0 = time.perf_counter()
        wr = O.proxy_source_compute(ot, opan, g.xs, g.ys, g.zs, h, g.areas, 8, True, nthreads=cores)
        t_up = time.perf_counter() - t0
        tg = np.sort(np.random.default_rng(21).choice(g.n, 60000, replace=False))
        sel = np.zeros(g.n + 1, bool)
        sel[tg + 1] = True
        spc, spp = pc[sel[pc[:, 0]]], pp[sel[pp[:, 0]]]
        t0 = time.perf_counter()
        O.pc_compute(ot, spc, g.xs, g.ys, g.zs, 8, wr, nthreads=cores)
        O.pp_compute(ot, spp, g.xs, g.ys, g.zs, g.areas, h, nthreads=cores)
        t_s = time.perf_counter() - t0
        frac = (len(spc) * P + len(spp)) / (len(pc) * P + len(pp))
        cpu_s = t_up + t_s / frac
        out["cpu_baseline"] = {"value": g.n / cpu_s, "unit": "evals/s", "cores": cores, "kind": "port",
                               "sample": f"proxy_source_compute whole ({t_up:.1f} s); pc/pp_compute on the "
                                         f"entries of 60,000 seeded targets ({100 * frac:.1f}% of the work, "
                                         f"{t_s:.1f} s), scaled to the whole list"}
    return out


def serving_run(args, S, torch, dev):
    """The serving mix: four Fibonacci ocean grids (40,962 / 163,842 / 655,362
    / 2,313,486 cells) resident under an HBM budget, Poisson arrivals at
    args.serve_rate per second, each request 1-16 fields drawn from a pool of
    seeded degree 1-128 fields of its grid (grid weights 0.4/0.3/0.2/0.1),
    batched per grid as they arrive.  Returns latency percentiles, throughput
    and the accuracy of sampled served results vs the FP64 direct sum."""
    from salgpu import serve, synth
    sizes = {"serve_40962": 40962, "serve_163842": 163842, "serve_655362": 655362, "serve_2313486": 2313486}
    weights = {"serve_40962": 0.4, "serve_163842": 0.3, "serve_655362": 0.2, "serve_2313486": 0.1}
    tune = None if not args.serve_tune else {k: int(v) for k, v in (kv.split("=") for kv in args.serve_tune.split(","))}
    srv = serve.Server(60 << 30, max_batch=64, device=dev.index or 0, tune=tune)
    pools, grids = {}, {}
    for name in sizes:
        g = synth.config_grid(name, device=dev)
        pool = synth.config_ssh("cfg3", g, nfields=16, seed=31, device=dev)
        # device-resident requests (fields produced on the GPU) unless --serve-host
        pools[name] = pool if args.serve_host else torch.tensor(pool, device=dev)
        grids[name] = g
        srv.register_grid(serve.GridSpec(name, g.xs, g.ys, g.zs, g.areas, args.degree, args.thresh, args.theta))
    # admit every grid and warm its kernels before the clock starts
    for name in sizes:
        srv.submit(serve.Request(name, pools[name][:2]))
    srv.run_until_idle()
    # warm every request shape (1-16 fields) on every grid, so that the
    # device allocator has cached blocks for the results before the clock starts
    for k in range(1, 17):
        for name in sizes:
            srv.submit(serve.Request(name, pools[name][:k]))
        srv.run_until_idle()
    srv.run_until_idle()
    # requests in flight at once hold fields and results of up to a few GB:
    # the allocator's cache holds that much before the clock starts
    srv.reserve(12 << 30)
    srv.slowest.clear()
    t0 = time.perf_counter()
    reqs = serve.run_workload(srv, pools, weights, args.serve_rate, args.serve_seconds, seed=7, keep=2)
    wall = time.perf_counter() - t0
    out = serve.summarize(reqs, sizes, wall, srv.batches)
    out["slowest_host_calls_ms"] = {k: round(v * 1e3, 2) for k, v in sorted(srv.slowest.items(), key=lambda kv: -kv[1])[:6]}
    out.update({"rate_req_per_s": args.serve_rate, "seconds": args.serve_seconds, "max_batch_fields": 64,
                "evictions": srv.evictions, "requests_on": "host" if args.serve_host else "device"})
    # accuracy of served results: first field of a few requests of each grid
    T = lambda a: torch.tensor(a, device=dev)
    errs = []
    for name in sizes:
        done = [q for q in reqs if q.grid == name and q.status == "done" and q.out_x is not None][:2]
        g = grids[name]
        tg = np.sort(np.random.default_rng(5).choice(g.n, min(2000, g.n), replace=False)).astype(np.int32)
        for q in done:
            host = lambda a: a.cpu().numpy() if isinstance(a, torch.Tensor) else a
            w = g.areas * host(q.ssh[0])
            dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(w), T(tg))
            dx, dy = dx.cpu().numpy(), dy.cpu().numpy()
            ex, ey = host(q.out_x[0])[tg] - dx, host(q.out_y[0])[tg] - dy
            errs.append(float(np.sqrt(np.sum(ex * ex + ey * ey) / np.sum(dx * dx + dy * dy))))
    out["rel_l2_vs_fp64_direct_max"] = max(errs) if errs else None
    srv.close()
    return out


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def time_solves(torch, grid, ssh, form, out, steps, flush, stream):
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for k in range(steps):
        flush.fill_(float(k))                 # evicts L2 between timed solves
        starts[k].record(stream)
        grid.solve(ssh, form=form, out=out)
        ends[k].record(stream)
    torch.cuda.synchronize()
    return np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])


def main():
    args = _args()
    if args.cpu_table:
        return cpu_table(args)
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
    form = {"ref": S.FORM_REF, "accurate": S.FORM_ACCURATE, "mixed": S.FORM_MIXED}[args.form]
    F = args.fields

    g, h, t_gen = make_problem(args, dev)
    t0 = time.perf_counter()
    tree = S.tree_traverse(g.xs, g.ys, g.zs, g.n, args.thresh)
    inter = S.dual_tree_traversal(tree, args.theta, args.thresh)
    t_lists = time.perf_counter() - t0
    # the same tree and list built on the device (fast admission); the host
    # build above stays the one solved
    # (the first device build at this size loads its kernels: time the second)
    S.dual_tree_traversal(S.tree_traverse(g.xs, g.ys, g.zs, g.n, args.thresh, device=local),
                          args.theta, args.thresh, device=local)
    t0 = time.perf_counter()
    dtree = S.tree_traverse(g.xs, g.ys, g.zs, g.n, args.thresh, device=local)
    dinter = S.dual_tree_traversal(dtree, args.theta, args.thresh, device=local)
    t_lists_dev = time.perf_counter() - t0
    dev_build_same = bool(np.array_equal(dinter, inter))
    del dtree, dinter
    grid = S.Grid(tree, g.xs, g.ys, g.zs, g.areas, args.degree, S.MODE_DTT, inter, device=local, max_fields=F)
    st = grid.stats()
    ssh = torch.tensor(h, device=dev)                      # (F, N), resident before timing
    ox = torch.empty_like(ssh)
    oy = torch.empty_like(ssh)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    tuned = None
    if form == S.FORM_MIXED and args.tune:
        tuned = {"set": grid.tune(**{k: int(v) for k, v in (kv.split("=") for kv in args.tune.split(","))})}
    elif form == S.FORM_MIXED and not args.no_autotune:
        # the batched form's autotuner on this grid and these fields: coordinate
        # descent over its choices, each timed with the L2 flushed and checked
        # against the FP64 direct sum (first field, 2,000 targets, 5e-6 bar)
        default = grid.tune()
        t0 = time.perf_counter()
        best, ms_best, ms_default = grid.autotune(ssh[:64], ntargets=2000, max_rel_err=5e-6)
        tuned = {"default": default, "chosen": best, "ms_default": ms_default, "ms_chosen": ms_best,
                 "search_s": time.perf_counter() - t0}
    # the leaf pass's operand precision (the autotuner's choice for 64-field blocks)
    leaf_f16 = form == S.FORM_MIXED and F == 64 and grid.tune().get("f16", 0) == 1
    st_after = grid.stats()
    for _ in range(args.warmup):
        grid.solve(ssh, form=form, out=(ox, oy))
    torch.cuda.synchronize()
    grid.sync()

    clk = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    per = time_solves(torch, grid, ssh, form, (ox, oy), args.steps, flush, stream)
    clocks = clk.stop()
    if world > 1:
        dist.barrier()
    grid.sync()
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
    up_ms, proxy_ms, leaf_ms = (phase[i] / nsol for i in range(3))
    st = grid.stats()
    if form == S.FORM_MIXED:                     # one timing record per field block
        nblk = (F + 63) // 64 if F > 32 else 1
        up_ms, proxy_ms, leaf_ms = up_ms * nblk, proxy_ms * nblk, leaf_ms * nblk

    # ---- accuracy vs the FP64 direct sum on sampled targets
    tg = np.sort(np.random.default_rng(99).choice(g.n, min(args.targets, g.n), replace=False)).astype(np.int32)
    T = lambda a: torch.tensor(a, device=dev)
    tgt = torch.tensor(tg, device=dev, dtype=torch.long)
    rels, mxs = [], []
    xd, yd, zd, tgd = T(g.xs), T(g.ys), T(g.zs), T(tg)
    for f in range(min(args.check_fields, F)):
        dx, dy = S.direct_sum(xd, yd, zd, T(g.areas * h[f]), tgd)
        ex, ey = ox[f][tgt] - dx, oy[f][tgt] - dy
        rels.append(float(torch.sqrt((ex * ex + ey * ey).sum() / (dx * dx + dy * dy).sum())))
        mxs.append(float(torch.sqrt(ex * ex + ey * ey).max() / torch.sqrt(dx * dx + dy * dy).max()))

    # ---- the kernel-tile store, timed beside the headline (which computes its
    # tiles): the FP16 leaf pass's kernel tiles depend on the grid alone; kept
    # in device memory, the first solve records them and later solves read
    # them instead of computing them, with the same results bit for bit
    tile = None
    if leaf_f16 and args.tile_store != "0":
        need = grid.stats()["tile_store_bytes"]
        free, _ = torch.cuda.mem_get_info(dev)
        if free > need + (24 << 30):
            tx, ty = torch.empty_like(ssh), torch.empty_like(ssh)
            grid.tune(tile_store=1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            grid.solve(ssh, form=form, out=(tx, ty))          # allocates the store, records the tiles
            torch.cuda.synchronize()
            t_first = time.perf_counter() - t0
            grid.solve(ssh, form=form, out=(tx, ty))
            pr = time_solves(torch, grid, ssh, form, (tx, ty), 3, flush, stream)
            grid.timing(1)
            for k in range(3):
                flush.fill_(float(k))
                grid.solve(ssh, form=form, out=(tx, ty))
            tph, tn = grid.timing(0)
            same = bool(torch.equal(tx, ox) and torch.equal(ty, oy))
            grid.tune(tile_store=0)                           # frees the store
            del tx, ty
            ms = float(np.median(pr))
            tile = {"bytes": need, "first_solve_ms": 1e3 * t_first, "ms_per_solve": ms,
                    "evals_per_s": g.n * F / (ms * 1e-3), "leaf_ms": tph[2] / tn,
                    "leaf_hbm_gbs": (need + 16.0 * F * g.n) / (tph[2] / tn * 1e-3) / 1e9,
                    "results_equal_computed_tiles": same,
                    "note": "sal_tune.tile_store = 1; not the headline, which computes its kernel tiles every solve"}

    # ---- plain FP64 form of the same grid, for the batched-vs-plain ratio
    plain = plain_e2e = None
    if form == S.FORM_MIXED and not args.no_fp64:
        s1 = ssh[:1].contiguous()
        o1 = (torch.empty_like(s1), torch.empty_like(s1))
        for _ in range(2):
            grid.solve(s1, form=S.FORM_REF, out=o1)
        pp = time_solves(torch, grid, s1, S.FORM_REF, o1, 3, flush, stream)
        plain = g.n / (float(pp.mean()) * 1e-3)
        # the plain form end to end: one field from pinned host memory through
        # sal_solve_host (copy in, solve, copy both components out, wait)
        h1 = torch.tensor(h[:1]).pin_memory()
        r1 = (torch.empty_like(h1).pin_memory(), torch.empty_like(h1).pin_memory())
        grid.solve_host(h1.numpy(), r1[0].numpy(), r1[1].numpy(), S.FORM_REF)
        t1 = time.perf_counter()
        for _ in range(3):
            grid.solve_host(h1.numpy(), r1[0].numpy(), r1[1].numpy(), S.FORM_REF)
        plain_e2e = g.n * 3 / (time.perf_counter() - t1)

    # ---- end to end through the host-buffer C ABI (pinned buffers).  Each step
    # copies its fields in, solves and copies both components out.  The
    # pipelined entry point overlaps one step's copies with its neighbours'
    # solves (two staging slots, results alternate between two host sets);
    # the synchronous one is timed too.
    h_ssh = torch.tensor(h).pin_memory()
    hs = h_ssh.numpy()
    h_out = [(torch.empty_like(h_ssh).pin_memory(), torch.empty_like(h_ssh).pin_memory()) for _ in range(2)]
    ho = [(x.numpy(), y.numpy()) for x, y in h_out]
    grid.solve_host(hs, ho[0][0], ho[0][1], form)
    e2e_steps = max(3, args.steps // 3)
    e2e_t = []
    for _ in range(e2e_steps):
        t1 = time.perf_counter()
        grid.solve_host(hs, ho[0][0], ho[0][1], form)
        e2e_t.append(time.perf_counter() - t1)
    e2e_sync = g.n * F / float(np.mean(e2e_t))
    for k in range(2):
        grid.solve_host_async(hs, ho[k][0], ho[k][1], form)
    grid.solve_host_wait()
    e2e_steps = max(6, args.steps)
    t1 = time.perf_counter()
    for k in range(e2e_steps):
        grid.solve_host_async(hs, ho[k % 2][0], ho[k % 2][1], form)
    grid.solve_host_wait()
    e2e_val = g.n * F * e2e_steps / (time.perf_counter() - t1)

    # ---- roofline of the dominant kernel (the leaf pass)
    if form == S.FORM_MIXED:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        bf16 = peaks.get("bf16_tflops", 1590.0)
        f16 = leaf_f16
        # the leaf pass's MMAs: kind::f16 (dense FP16 = the bf16 rate) or kind::tf32 (half of it)
        peak = bf16 if f16 else bf16 / 2.0
        leaf_flops = 4.0 * F * (st["pairs_pp"] + st["pairs_pc"] + 3.0 * st["macs_down_batched"])
        achieved = leaf_flops / (leaf_ms * 1e-3) / 1e12
        prec = "FP16" if f16 else "TF32"
        src = "bf16_tflops of measured" if "bf16_tflops" in peaks else "1.59 PFLOP/s bf16 fallback"
        roof = {"bound": "tensor", "kernel": f"tc_leaf_kernel<0> (tcgen05 {prec} hi/lo, M=128 field parts x N=256 "
                          "target components; PP+PC kernel tiles, DOWN interpolation) + its weight store",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": (f"FP16 dense = {src}" if f16 else f"TF32 dense = {src} / 2"),
                "flops_counted": "algorithmic 4*F per pair (2 components x FMA x F fields); the hi/lo split "
                                 "executes 4x these on the tensor cores (W_hi,W_lo x T_hi,T_lo), plus padding",
                # ncu dram__bytes_read.sum + dram__bytes_write.sum of one tc_leaf_kernel launch on the
                # 655,362-cell, 64-field case (FP16: 4.01 + 2.76 GB; TF32: 3.95 + 2.65 GB), scaled by the
                # cell count
                "traffic": (6.767e9 if f16 else 6.600e9) * g.n / 655362 if F == 64 else None,
                "traffic_source": "ncu capture on 655,362 cells x 64 fields, scaled by cells",
                "leaf_ms": leaf_ms, "proxy_ms": proxy_ms, "prep_upward_ms": up_ms}
        if tile:
            # the replaying leaf pass streams its tiles from HBM: its HBM fraction
            hbm = peaks.get("hbm_gbs", 6650.0)
            tile["leaf_hbm_frac"] = tile["leaf_hbm_gbs"] / hbm
            tile["hbm_peak_source"] = "hbm_gbs of measured" if "hbm_gbs" in peaks else "6.65 TB/s fallback"
    else:
        peak64 = S.fma_peak(64)
        leaf_flops = FLOPS_PER_PAIR * (st["pairs_pp"] + st["pairs_pc"]) + 2 * FLOPS_PER_MAC * st["macs_down"]
        achieved = leaf_flops / (leaf_ms * 1e-3) / 1e12
        roof = {"bound": "fp64", "kernel": "eval_kernel<leaf> (PP+PC pairs + DOWN interpolation)",
                "achieved": achieved, "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                "peak_source": "sal_fma_peak(64) on this GPU (FP64 FMA pipe; MEASURED_PEAKS.json has no FP64 figure)",
                "traffic": None, "leaf_ms": leaf_ms, "proxy_ms": proxy_ms, "prep_upward_ms": up_ms}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline(args, g, h[0], args.cpu_seconds)
    stt = None
    if rank == 0 and world == 1 and form == S.FORM_MIXED and not args.no_stt:
        stt = stt_run(args, S, torch, dev)
    served = None
    if rank == 0 and world == 1 and form == S.FORM_MIXED and not args.no_serve:
        del grid
        torch.cuda.empty_cache()
        served = serving_run(args, S, torch, dev)

    if rank == 0:
        value = g.n * F * args.steps * world / (total_ms * 1e-3)
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": (("f32/f16 hi-lo" if leaf_f16 else "f32/tf32 hi-lo") + " (fp64 self pairs)"
                      if form == S.FORM_MIXED and F == 64 else "f32/tf32 (fp64 self pairs)" if form == S.FORM_MIXED
                      else "f64"),
            "data": "synthetic: seeded Fibonacci ocean grid + spherical-harmonic SSH (stand-in for the MPAS CSVs)",
            "config": {"workload": workload_name(args, g.n), "cells": g.n, "fields": F, "form": args.form,
                       "parallelism": f"replicas x{world}", "l2": "flushed (256 MB write) between timed solves"},
            "latency_ms": {"p50": float(np.percentile(per, 50)), "p99": float(np.percentile(per, 99))},
            "accuracy": {"rel_l2_vs_fp64_direct_max": max(rels), "rel_l2_vs_fp64_direct_mean": float(np.mean(rels)),
                         "max_err_over_max_ref": max(mxs), "fields_checked": len(rels), "targets": len(tg)},
            "plain_fp64": None if plain is None else {
                "value": plain, "unit": "evals/s", "batched_over_plain": value / world / plain,
                "e2e": {"value": plain_e2e, "unit": "evals/s", "api": "sal_solve_host, SAL_FORM_REF, one field",
                        "h2d_bytes_per_step": 8 * g.n, "d2h_bytes_per_step": 16 * g.n}},
            "roofline": roof,
            "work": {k: st[k] for k in ("pairs_pp", "pairs_pc", "pairs_cp", "pairs_cc", "macs_up", "macs_down",
                                        "macs_up_batched", "macs_down_batched")},
            "autotune": tuned,
            "tile_store": tile,
            "setup_s": {"grid_generation": t_gen, "tree_and_lists": t_lists, "plan_and_upload": st["setup_seconds"],
                        "tree_and_lists_on_device": t_lists_dev, "device_build_list_equal": dev_build_same},
            "e2e": {"value": e2e_val, "unit": "evals/s", "h2d_bytes_per_step": 8 * g.n * F,
                    "d2h_bytes_per_step": 16 * g.n * F, "steps": e2e_steps,
                    "api": "sal_solve_host_async + sal_solve_host_wait (pinned host buffers, two staging slots)",
                    "sync_value": e2e_sync, "sync_api": "sal_solve_host"},
            "clocks": clocks,
            # batched form: the library's count per block (prep, stores, upward, transfers, proxy,
            # finalize, leaf); FP64 forms: prep, upward, finalize, proxy, finalize, leaf
            "gpu_launches": (st_after["launches_batched"] * args.steps * (((F + 63) // 64) if F > 32 else 1)
                             if form == S.FORM_MIXED else 6 * args.steps),
        }
        if cb:
            line["cpu_baseline"] = cb
        if stt:
            line["stt_mom6"] = stt
        if served:
            line["serving"] = served
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
