"""Continuous-batching request loop for SAL-gradient solves on resident grids.

The reference solves one field per program run, rebuilding its tree each
time (code.f90).  Here each registered grid keeps its tree, interaction lists,
proxies and work plan resident in device memory; SSH fields arrive as
requests (1..64 fields each), are batched per grid as they arrive, and each
batch is one batched mixed-precision solve (SAL_FORM_MIXED) on the grid's own
CUDA stream, so batches of different grids overlap on the device.  Smaller
grids get higher stream priorities: their short batches are scheduled onto
SMs ahead of a large grid's long one as its CTAs retire.
With `graphs=True` each (grid, batch width) is captured into a CUDA graph on
its first batch and replayed afterwards (the staging buffers are the grid's
own, so the call shape is fixed).  It is off by default: in one measured run
the smallest grid's batches took 3.4 ms instead of 2.2 ms with graphs on, as
if the replayed kernels lost the stream priority that keeps them ahead of a
large grid's.

A request's fields are either a host array (copied through the grid's pinned
staging buffers; results come back as host arrays) or a CUDA tensor on the
server's device (copied device to device; results stay on the device).

Scheduling rules:
  * a grid has at most one batch in flight (its batch buffers are its own);
  * whenever a grid is idle and has pending requests, its oldest requests are
    packed (whole requests, at most `max_batch` fields) into the next batch --
    at once if they fill a batch, otherwise once the oldest has waited
    `patience` times the grid's recent batch time (a running average): a
    batch costs about the same for 1 or 64 fields, so a grid whose batches
    are expensive gathers more fields per batch and leaves the device to the
    others (patience 0: launch as soon as the grid is idle);
  * grids are admitted to the device by an HBM budget: a grid whose resident
    bytes (plan + batched buffers + batch staging) do not fit evicts idle
    grids, least recently used first; a grid that alone exceeds the budget is
    refused and its requests fail with `SalError(SAL_ENOMEM)`;
  * requests can be cancelled until their batch is launched.

Latency of a request = completion of its batch (including the copy of its
results into its own arrays) minus its arrival time.  Each field's result does not depend on which other fields
share its batch (tensor-core columns never mix), which
tests/test_serve.py checks.
"""
from __future__ import annotations

import gc
import itertools
import time
from collections import OrderedDict, deque
from dataclasses import dataclass, field

import numpy as np

from . import FORM_MIXED, MODE_DTT, SAL_EINVAL, SAL_ENOMEM, Grid, SalError, dual_tree_traversal, tree_traverse


@dataclass
class Request:
    grid: str
    ssh: object                # (F, N) float64: numpy array (host) or CUDA tensor (device)
    arrival: float = 0.0
    ready: object = None       # device requests: CUDA event after which ssh holds the fields
                               # (None: all work queued so far on the current stream)
    rid: int = -1
    status: str = "pending"    # pending | running | done | failed | cancelled
    out_x: object = None         # same kind as ssh
    out_y: object = None
    error: Exception | None = None
    done_time: float = 0.0

    nf: int = 0                # fields (kept after ssh is released)

    def __post_init__(self):
        if self.ssh is not None:
            self.nf = self.ssh.shape[0]

    @property
    def nfields(self) -> int:
        return self.nf

    @property
    def latency(self) -> float:
        return self.done_time - self.arrival


@dataclass
class GridSpec:
    name: str
    xs: np.ndarray
    ys: np.ndarray
    zs: np.ndarray
    areas: np.ndarray
    degree: int = 8
    thresh: int = 200
    theta: float = 0.7


@dataclass
class _Resident:
    spec: GridSpec
    tree: object
    inter: np.ndarray
    grid: Grid | None = None
    bytes: int = 0
    stream: object = None
    ssh_dev: object = None
    ox_dev: object = None
    oy_dev: object = None
    h_in: object = None
    h_ox: object = None
    h_oy: object = None
    pending: deque = field(default_factory=deque)
    inflight: list | None = None
    event: object = None
    last_used: float = 0.0
    launched: float = 0.0
    batch_error: Exception | None = None
    pending_fields: int = 0
    batch_time: float = 0.0            # running average of launch-to-done seconds


class Server:
    """Resident grids + per-grid continuous batching on CUDA streams."""

    def __init__(self, hbm_budget_bytes: int, max_batch: int = 64, device: int = 0, clock=time.perf_counter,
                 grid_factory=Grid, priorities: bool = True, patience: float = 2.0, graphs: bool = False,
                 device_setup: bool = True, tune: dict | None = None):
        try:
            import torch
        except ImportError:           # the CPU test double needs no torch
            torch = None
        self.torch = torch
        self.budget = int(hbm_budget_bytes)
        self.max_batch = int(max_batch)
        self.device = device
        self.clock = clock
        self.grid_factory = grid_factory
        self.grids: "OrderedDict[str, _Resident]" = OrderedDict()
        self.used = 0
        self._ids = itertools.count()
        self.completed: list[Request] = []
        self.evictions = 0
        self.priorities = priorities
        self.patience = float(patience)
        self.graphs = graphs                 # one CUDA graph per (grid, batch width)
        self.device_setup = device_setup     # tree and list built on the device when one is present
        # batched-form choices set on every admitted grid (sal_grid_tune_set): FP16 leaf operands and
        # 64-unit chains, the autotuner's pick on the 2.3M-cell grid; one group per CTA keeps the
        # CTAs short, so higher-priority grids' kernels get SMs quickly
        self.tune = dict(f16=1, chain_ksteps=64) if tune is None else dict(tune)
        self.batches: list[tuple] = []     # (grid, fields, launch time, done time) of finished batches
        self.slowest: dict = {}            # the longest host-side launch / poll / results call per grid, seconds

    # ------------------------------------------------------------------ grids
    def register_grid(self, spec: GridSpec) -> None:
        """Builds the tree and lists of a grid (tree_module.f90) once, on the
        device when there is one and device_setup is set; the device plan is
        created on admission."""
        on_dev = self.device_setup and self.torch is not None and self.torch.cuda.is_available()
        dev = self.device if on_dev else None
        tree = tree_traverse(spec.xs, spec.ys, spec.zs, len(spec.xs), spec.thresh, device=dev)
        inter = dual_tree_traversal(tree, spec.theta, spec.thresh, device=dev)
        self.grids[spec.name] = _Resident(spec, tree, inter)

    def _bytes_needed(self, r: _Resident, g: Grid) -> int:
        st = g.stats()
        n = len(r.spec.xs)
        staging = 3 * self.max_batch * n * 8          # device ssh + two outputs
        return int(st["device_bytes"] + st["mixed_bytes"] + staging)

    def _evict(self, need: int, keep: str) -> bool:
        for name, r in list(self.grids.items()):
            if self.used + need <= self.budget:
                return True
            if name == keep or r.grid is None or r.inflight is not None:
                continue
            self._release(r)
            self.evictions += 1
        return self.used + need <= self.budget

    def _release(self, r: _Resident) -> None:
        r.grid = None
        r.ssh_dev = r.ox_dev = r.oy_dev = None
        self.used -= r.bytes
        r.bytes = 0

    def _admit(self, r: _Resident) -> None:
        s = r.spec
        g = self.grid_factory(r.tree, s.xs, s.ys, s.zs, s.areas, s.degree, MODE_DTT, r.inter, device=self.device,
                              max_fields=self.max_batch)
        if self.tune and hasattr(g, "tune"):
            g.tune(**self.tune)
        need = self._bytes_needed(r, g)
        if need > self.budget:
            del g
            raise SalError(SAL_ENOMEM, f"grid {s.name} needs {need} bytes, above the HBM budget {self.budget}")
        if not self._evict(need, s.name):
            del g
            raise SalError(SAL_ENOMEM, f"no room for grid {s.name}: busy grids hold the budget")
        r.grid = g
        r.bytes = need
        self.used += need
        if self.graphs and hasattr(g, "set_graphs"):
            g.set_graphs(True)
        self._alloc_staging(r)

    def reserve(self, nbytes: int) -> None:
        """Grows torch's caching allocator on the serving device by nbytes
        (one block, freed at once and kept in the cache): requests' fields and
        results are then carved from it instead of cudaMalloc calls in the
        middle of the request stream."""
        if self.torch is None or nbytes <= 0:
            return
        blk = self.torch.empty(int(nbytes), dtype=self.torch.uint8, device=self.torch.device("cuda", self.device))
        del blk

    # ------------------------------------------------------------------ device hooks
    # (a test double overrides these four to exercise the scheduling on the CPU)
    def _stream_priority(self, r: _Resident) -> int:
        # rank of the grid by size among the registered grids: the smallest
        # gets the highest priority (most negative); torch clamps to the range
        if not self.priorities:
            return 0
        sizes = sorted({len(g.spec.xs) for g in self.grids.values()})
        return -(len(sizes) - 1 - sizes.index(len(r.spec.xs)))

    def _alloc_staging(self, r: _Resident) -> None:
        torch = self.torch
        n = len(r.spec.xs)
        dev = torch.device("cuda", self.device)
        if r.stream is None:
            r.stream = torch.cuda.Stream(device=dev, priority=self._stream_priority(r))
            r.h_in = torch.empty((self.max_batch, n), dtype=torch.float64).pin_memory()
            r.h_ox = torch.empty((self.max_batch, n), dtype=torch.float64).pin_memory()
            r.h_oy = torch.empty((self.max_batch, n), dtype=torch.float64).pin_memory()
        r.ssh_dev = torch.empty((self.max_batch, n), dtype=torch.float64, device=dev)
        r.ox_dev = torch.empty_like(r.ssh_dev)
        r.oy_dev = torch.empty_like(r.ssh_dev)

    def _launch_device(self, r: _Resident, batch: list, nf: int) -> None:
        torch = self.torch
        on_dev = [isinstance(q.ssh, torch.Tensor) for q in batch]
        f = 0
        for q, d in zip(batch, on_dev):
            if not d:
                r.h_in[f:f + q.nfields].numpy()[:] = q.ssh
            f += q.nfields
        # device requests: wait for their fields only (a request without a
        # ready event waits for the submitting stream); waiting on a whole
        # low-priority stream would hand its priority to this batch
        cur = None
        for q, d in zip(batch, on_dev):
            if not d:
                continue
            if q.ready is not None:
                r.stream.wait_event(q.ready)
            elif cur is None:
                cur = torch.cuda.current_stream(r.ssh_dev.device)
                r.stream.wait_stream(cur)
        with torch.cuda.stream(r.stream):
            f = 0
            for q, d in zip(batch, on_dev):
                src = q.ssh if d else r.h_in[f:f + q.nfields]
                r.ssh_dev[f:f + q.nfields].copy_(src, non_blocking=True)
                f += q.nfields
            r.grid.solve(r.ssh_dev[:nf], form=FORM_MIXED, out=(r.ox_dev[:nf], r.oy_dev[:nf]),
                         stream=r.stream.cuda_stream)
            f = 0
            for q, d in zip(batch, on_dev):
                k = q.nfields
                if d:
                    q.out_x = r.ox_dev[f:f + k].clone()
                    q.out_y = r.oy_dev[f:f + k].clone()
                else:
                    r.h_ox[f:f + k].copy_(r.ox_dev[f:f + k], non_blocking=True)
                    r.h_oy[f:f + k].copy_(r.oy_dev[f:f + k], non_blocking=True)
                f += k
            r.event = torch.cuda.Event()
            r.event.record(r.stream)

    def _batch_done(self, r: _Resident) -> bool:
        if not r.event.query():
            return False
        try:
            r.grid.sync(r.stream.cuda_stream)   # the stream is idle: only reads the grid's time-out flag
        except SalError as e:
            r.batch_error = e
        return True

    def _results(self, r: _Resident, q: Request, f: int):
        if isinstance(q.ssh, self.torch.Tensor):
            return q.out_x, q.out_y                   # written on the grid's stream before its event
        return r.h_ox[f:f + q.nfields].numpy().copy(), r.h_oy[f:f + q.nfields].numpy().copy()

    # ------------------------------------------------------------------ requests
    def submit(self, req: Request) -> Request:
        if req.grid not in self.grids:
            raise SalError(SAL_EINVAL, f"unknown grid {req.grid}")
        r = self.grids[req.grid]
        n = len(r.spec.xs)
        if req.ssh.ndim != 2 or req.ssh.shape[1] != n or not (1 <= req.nfields <= self.max_batch):
            raise SalError(SAL_EINVAL, f"request for grid {req.grid} must be (F, {n}) with 1 <= F <= {self.max_batch}")
        req.rid = next(self._ids)
        if not req.arrival:
            req.arrival = self.clock()
        r.pending.append(req)
        r.pending_fields += req.nfields
        return req

    def cancel(self, req: Request) -> bool:
        r = self.grids[req.grid]
        if req.status == "pending" and req in r.pending:
            r.pending.remove(req)
            r.pending_fields -= req.nfields
            req.status = "cancelled"
            return True
        return False

    # ------------------------------------------------------------------ loop
    def _launch(self, r: _Resident) -> None:
        batch, nf = [], 0
        while r.pending and nf + r.pending[0].nfields <= self.max_batch:
            q = r.pending.popleft()
            r.pending_fields -= q.nfields
            batch.append(q)
            nf += q.nfields
        if not batch:
            return
        if r.grid is None:
            try:
                self._admit(r)
            except (SalError, MemoryError) as e:
                for q in batch:
                    q.status, q.error, q.done_time = "failed", e, self.clock()
                    self.completed.append(q)
                return
        for q in batch:
            q.status = "running"
        t0 = self.clock()
        self._launch_device(r, batch, nf)
        self._note_slow("launch " + r.spec.name, self.clock() - t0)
        r.inflight = batch
        r.last_used = r.launched = self.clock()
        self.grids.move_to_end(r.spec.name)

    def _note_slow(self, what: str, dt: float) -> None:
        # the slowest host-side step of each kind: where a stalled loop spends its time
        if dt > self.slowest.get(what, 0.0):
            self.slowest[what] = dt

    def _reap(self, r: _Resident) -> None:
        t0 = self.clock()
        done = r.inflight is not None and self._batch_done(r)
        self._note_slow("poll " + r.spec.name, self.clock() - t0)
        if not done:
            return
        now = self.clock()
        f = 0
        err, r.batch_error = r.batch_error, None
        for q in r.inflight:
            try:
                if err is not None:
                    raise err
                q.out_x, q.out_y = self._results(r, q, f)
                q.status = "done"
            except SalError as e:
                q.status, q.error = "failed", e
            q.done_time = now
            f += q.nfields
            self.completed.append(q)
        self._note_slow("results " + r.spec.name, self.clock() - now)
        self.batches.append((r.spec.name, f, r.launched, now))
        dt = now - r.launched
        r.batch_time = dt if r.batch_time == 0.0 else 0.8 * r.batch_time + 0.2 * dt
        r.inflight = None

    def step(self) -> int:
        """Reaps finished batches and launches new ones; returns the number of
        batches in flight."""
        for r in self.grids.values():
            self._reap(r)
        now = self.clock()
        order = sorted((r for r in self.grids.values() if r.pending and r.inflight is None and self._ready(r, now)),
                       key=lambda r: r.pending[0].arrival)
        for r in order:
            self._launch(r)
        return sum(r.inflight is not None for r in self.grids.values())

    def _ready(self, r: _Resident, now: float) -> bool:
        return (self.patience <= 0.0 or r.pending_fields >= self.max_batch
                or now - r.pending[0].arrival >= self.patience * r.batch_time)

    def busy(self) -> bool:
        return any(r.pending or r.inflight is not None for r in self.grids.values())

    def run_until_idle(self, poll_s: float = 0.0002) -> None:
        while self.busy():
            if self.step() and poll_s:
                time.sleep(poll_s)

    def close(self) -> None:
        for r in self.grids.values():
            while r.inflight is not None:
                self._reap(r)
            if r.grid is not None:
                self._release(r)


def poisson_arrivals(rng: np.random.Generator, rate: float, duration: float) -> np.ndarray:
    """Arrival times of a Poisson process of `rate` per second on [0, duration)."""
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return np.array(out)
        out.append(t)


def run_workload(server: Server, pools: dict, weights: dict, rate: float, duration: float, seed: int = 0,
                 max_rhs: int = 16, keep: int | None = None) -> list:
    """Replays Poisson arrivals in real time: each request picks a grid by
    `weights`, 1..max_rhs fields (uniform) drawn from that grid's field pool
    (a numpy array: host requests; a CUDA tensor: device requests), and is
    submitted at its arrival time while the loop keeps batching.  With `keep`,
    only the first `keep` finished requests of each grid hold on to their
    fields and results; the others drop them as a client that consumed its
    result would (holding every result of a long run would fill the device)."""
    rng = np.random.default_rng(seed)
    times = poisson_arrivals(rng, rate, duration)
    gen = None                     # device requests are gathered on their own high-priority stream
    for pool in pools.values():
        if not isinstance(pool, np.ndarray):
            import torch
            gen = torch.cuda.Stream(device=pool.device, priority=-8)
            break
    names = list(weights)
    p = np.array([weights[k] for k in names], dtype=float)
    p /= p.sum()
    plan = []
    for t in times:
        name = names[rng.choice(len(names), p=p)]
        F = int(rng.integers(1, max_rhs + 1))
        pool = pools[name]
        idx = rng.integers(0, pool.shape[0], size=F)
        if not isinstance(pool, np.ndarray):
            import torch
            idx = torch.as_tensor(idx, device=pool.device)
        plan.append((t, name, idx))
    reqs = []
    # the loop is single-threaded: a cyclic-garbage pass in the middle of it
    # would stall every grid's batching at once
    gc_was = gc.isenabled()
    gc.disable()
    try:
        _replay(server, plan, pools, gen, keep, reqs)
    finally:
        if gc_was:
            gc.enable()
    return reqs


def _replay(server: Server, plan: list, pools: dict, gen, keep, reqs: list) -> None:
    t0 = server.clock()
    i = 0
    seen, kept = len(server.completed), {}
    while i < len(plan) or server.busy():
        if keep is not None and len(server.completed) > seen:
            for q in server.completed[seen:]:
                kept[q.grid] = kept.get(q.grid, 0) + 1
                if kept[q.grid] > keep:
                    q.ssh = q.out_x = q.out_y = None
            seen = len(server.completed)
        now = server.clock() - t0
        while i < len(plan) and plan[i][0] <= now:
            t, name, idx = plan[i]
            if gen is None:
                reqs.append(server.submit(Request(name, pools[name][idx], arrival=t0 + t)))
            else:
                import torch
                with torch.cuda.stream(gen):
                    x = pools[name][idx]
                    ev = torch.cuda.Event()
                    ev.record(gen)
                reqs.append(server.submit(Request(name, x, arrival=t0 + t, ready=ev)))
            i += 1
        server.step()


def summarize(reqs: list, cells: dict, wall: float, batches: list | None = None) -> dict:
    done = [q for q in reqs if q.status == "done"]
    lat = np.array([q.latency for q in done]) * 1e3
    evals = sum(cells[q.grid] * q.nfields for q in done)
    single = np.array([q.latency for q in done if q.nfields == 1]) * 1e3
    out = {"requests": len(reqs), "done": len(done), "failed": sum(q.status == "failed" for q in reqs),
           "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
           "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
           "single_field_p50_ms": float(np.percentile(single, 50)) if len(single) else None,
           "evals_per_s": evals / wall if wall > 0 else None}
    per = {}
    t0 = min((q.arrival for q in reqs), default=0.0)
    for name in cells:
        lg = np.array([q.latency for q in done if q.grid == name]) * 1e3
        if not len(lg):
            continue
        d = {"requests": int(len(lg)), "p50_ms": float(np.percentile(lg, 50)), "p99_ms": float(np.percentile(lg, 99))}
        if batches:
            bs = [b for b in batches if b[0] == name and b[2] >= t0]
            if bs:
                d["batches"] = len(bs)
                d["mean_fields_per_batch"] = float(np.mean([b[1] for b in bs]))
                d["mean_batch_ms"] = float(np.mean([(b[3] - b[2]) * 1e3 for b in bs]))
                d["max_batch_ms"] = float(max((b[3] - b[2]) * 1e3 for b in bs))
        per[name] = d
    out["per_grid"] = per
    if batches:
        # where the tail comes from: the longest stretch with no batch launched
        # (a stalled host loop) against the longest batch (a slow device)
        ls = sorted(b[2] for b in batches if b[2] >= t0)
        if len(ls) > 1:
            gaps = np.diff(ls)
            k = int(np.argmax(gaps))
            out["max_launch_gap_ms"] = float(gaps[k] * 1e3)
            out["max_launch_gap_at_s"] = float(ls[k] - t0)
    return out
