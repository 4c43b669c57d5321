"""Serving loop tests.

CPU: the scheduling (batching, admission by HBM budget, LRU eviction,
cancellation, refusal and allocation failure) runs against a test double that
replaces only the device hooks; every failure is made on the host.
GPU: each request's result is the same alone and inside a mixed batch, and
served results meet the 1e-5 rel-L2 bar against the FP64 direct sum.
"""
import numpy as np
import pytest

from conftest import grid_and_ssh, rel_l2


# ------------------------------------------------------------------ CPU test double
class FakeGrid:
    """Stands in for salgpu.Grid: fixed sizes, no device."""
    fail_next = False

    def __init__(self, tree, xs, ys, zs, areas, degree, mode, inter, device=0, max_fields=64):
        import salgpu as S
        if FakeGrid.fail_next:
            FakeGrid.fail_next = False
            raise S.SalError(S.SAL_ENOMEM, "simulated cudaMalloc failure")
        self.n = len(xs)

    def stats(self):
        return {"device_bytes": 100 * self.n, "mixed_bytes": 50 * self.n}

    def sync(self):
        pass


def _fake_server(budget, max_batch=8, patience=0.0):
    from salgpu import serve

    class FakeServer(serve.Server):
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            self.launched = []
            self.t = 0.0

        def _alloc_staging(self, r):
            pass

        def _launch_device(self, r, batch, nf):
            self.launched.append((r.spec.name, [q.rid for q in batch], nf))
            r.event = 2                        # completes after two polls

        def _batch_done(self, r):
            r.event -= 1
            return r.event <= 0

        def _results(self, r, q, f):
            return np.zeros((q.nfields, len(r.spec.xs))), np.zeros((q.nfields, len(r.spec.xs)))

    clock = iter(np.arange(0.0, 1e6, 1e-3))
    return FakeServer(budget, max_batch=max_batch, clock=lambda: next(clock), grid_factory=FakeGrid, patience=patience)


def _spec(name, n, seed=0):
    from salgpu import serve
    from salgpu import synth
    g = synth.fibonacci_grid(n, seed=seed, device="cpu")
    return serve.GridSpec(name, g.xs, g.ys, g.zs, g.areas, thresh=40)


def _bytes(n, max_batch=8):
    return 150 * n + 3 * max_batch * n * 8


def test_batching_packs_whole_requests_fifo():
    from salgpu import serve
    srv = _fake_server(10 ** 9, max_batch=8)
    srv.register_grid(_spec("a", 500))
    n = 500
    reqs = [srv.submit(serve.Request("a", np.zeros((k, n)))) for k in (3, 4, 2, 5)]
    srv.run_until_idle(poll_s=0)
    assert [b[1] for b in srv.launched] == [[reqs[0].rid, reqs[1].rid], [reqs[2].rid, reqs[3].rid]]
    assert [b[2] for b in srv.launched] == [7, 7]
    assert all(q.status == "done" for q in reqs)


def test_summary_reports_launch_gaps_and_slowest_host_calls():
    """The serving summary's diagnostics: per grid the longest batch, the
    longest stretch with no batch launched, and the loop's slowest host calls
    (launch, poll, results) per grid."""
    from salgpu import serve
    srv = _fake_server(10 ** 9, max_batch=8)
    srv.register_grid(_spec("a", 300))
    reqs = [srv.submit(serve.Request("a", np.zeros((5, 300)))) for _ in range(3)]
    srv.run_until_idle(poll_s=0)
    assert len(srv.batches) == 3                      # 5 + 5 fields do not fit a batch of 8
    out = serve.summarize(reqs, {"a": 300}, 1.0, srv.batches)
    launches = sorted(b[2] for b in srv.batches)
    assert out["max_launch_gap_ms"] == pytest.approx(1e3 * float(np.max(np.diff(launches))))
    assert out["per_grid"]["a"]["max_batch_ms"] == pytest.approx(1e3 * max(b[3] - b[2] for b in srv.batches))
    assert {"launch a", "poll a", "results a"} <= set(srv.slowest)
    assert all(v > 0 for v in srv.slowest.values())


def test_admission_evicts_least_recently_used_idle_grid():
    from salgpu import serve
    budget = _bytes(400) + _bytes(500) + 10          # two of the three grids fit
    srv = _fake_server(budget)
    for name, n in (("a", 400), ("b", 500), ("c", 300)):
        srv.register_grid(_spec(name, n))
    for name, n in (("a", 400), ("b", 500)):
        srv.submit(serve.Request(name, np.zeros((1, n))))
    srv.run_until_idle(poll_s=0)
    assert srv.evictions == 0 and srv.grids["a"].grid is not None and srv.grids["b"].grid is not None
    srv.submit(serve.Request("c", np.zeros((1, 300))))
    srv.run_until_idle(poll_s=0)
    assert srv.evictions == 1 and srv.grids["a"].grid is None       # a was the least recently used
    assert srv.grids["c"].grid is not None and srv.used <= budget


def test_grid_above_budget_is_refused_and_loop_continues():
    from salgpu import serve
    import salgpu as S
    srv = _fake_server(_bytes(300) + 10)
    srv.register_grid(_spec("big", 2000))
    srv.register_grid(_spec("small", 300))
    big = srv.submit(serve.Request("big", np.zeros((2, 2000))))
    small = srv.submit(serve.Request("small", np.zeros((1, 300))))
    srv.run_until_idle(poll_s=0)
    assert big.status == "failed" and big.error.code == S.SAL_ENOMEM
    assert small.status == "done"


def test_allocation_failure_fails_the_batch_only():
    from salgpu import serve
    srv = _fake_server(10 ** 9)
    srv.register_grid(_spec("a", 300))
    FakeGrid.fail_next = True
    r1 = srv.submit(serve.Request("a", np.zeros((1, 300))))
    srv.run_until_idle(poll_s=0)
    r2 = srv.submit(serve.Request("a", np.zeros((1, 300))))
    srv.run_until_idle(poll_s=0)
    assert r1.status == "failed" and "simulated" in str(r1.error)
    assert r2.status == "done"


def test_cancel_and_malformed_requests():
    from salgpu import serve
    import salgpu as S
    srv = _fake_server(10 ** 9, max_batch=4)
    srv.register_grid(_spec("a", 300))
    with pytest.raises(S.SalError):
        srv.submit(serve.Request("a", np.zeros((1, 299))))          # wrong point count
    with pytest.raises(S.SalError):
        srv.submit(serve.Request("a", np.zeros((5, 300))))          # more fields than a batch holds
    with pytest.raises(S.SalError):
        srv.submit(serve.Request("nope", np.zeros((1, 300))))
    r1 = srv.submit(serve.Request("a", np.zeros((4, 300))))
    r2 = srv.submit(serve.Request("a", np.zeros((2, 300))))
    srv.step()                                                       # r1 launched, r2 waits
    assert srv.cancel(r2) and r2.status == "cancelled"
    assert not srv.cancel(r1)
    srv.run_until_idle(poll_s=0)
    assert r1.status == "done" and [b[1] for b in srv.launched] == [[r1.rid]]


def test_patience_gathers_fields_until_the_batch_fills_or_the_wait_runs_out():
    from salgpu import serve
    srv = _fake_server(10 ** 9, max_batch=8, patience=2.0)
    srv.register_grid(_spec("a", 300))
    r0 = srv.submit(serve.Request("a", np.zeros((1, 300))))
    srv.run_until_idle(poll_s=0)                       # no batch time known yet: launches at once
    assert [b[1] for b in srv.launched] == [[r0.rid]]
    bt = srv.grids["a"].batch_time
    assert bt > 0
    r1 = srv.submit(serve.Request("a", np.zeros((2, 300))))
    srv.step()
    assert len(srv.launched) == 1                      # waits: 2 fields, no time has passed
    r2 = srv.submit(serve.Request("a", np.zeros((6, 300))))
    srv.step()                                         # 8 fields fill the batch
    assert [b[1] for b in srv.launched][-1] == [r1.rid, r2.rid]
    srv.run_until_idle(poll_s=0)
    r3 = srv.submit(serve.Request("a", np.zeros((1, 300))))
    srv.run_until_idle(poll_s=0)                       # launched once it has waited 2 batch times
    assert r3.status == "done" and r3.done_time - r3.arrival >= 2 * bt * 0.8


def test_poisson_arrivals_rate():
    from salgpu import serve
    t = serve.poisson_arrivals(np.random.default_rng(0), 200.0, 50.0)
    assert abs(len(t) / 50.0 - 200.0) < 10 and np.all(np.diff(t) > 0)


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_served_results_equal_alone_and_in_the_mix_and_meet_accuracy():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import salgpu as S
    from salgpu import serve
    grids = {}
    srv = serve.Server(8 << 30, max_batch=64)
    for name, thr in (("small_3000", 40), ("cfg0", 100)):
        g, hs = grid_and_ssh(name, nfields=12, seed=21)
        grids[name] = (g, hs)
        srv.register_grid(serve.GridSpec(name, g.xs, g.ys, g.zs, g.areas, thresh=thr))
    rng = np.random.default_rng(4)
    mix = []
    for k in range(12):
        name = ("small_3000", "cfg0")[k % 2]
        idx = rng.choice(12, int(rng.integers(1, 5)), replace=False)
        mix.append((srv.submit(serve.Request(name, grids[name][1][idx])), idx))
    srv.run_until_idle()
    assert all(q.status == "done" for q, _ in mix)
    for q, idx in mix[:4]:                                            # each one again, alone
        alone = srv.submit(serve.Request(q.grid, grids[q.grid][1][idx]))
        srv.run_until_idle()
        assert np.array_equal(alone.out_x, q.out_x) and np.array_equal(alone.out_y, q.out_y)
    q, idx = mix[1]                                                   # a cfg0 request vs the direct sum
    g, hs = grids[q.grid]
    T = lambda a: torch.tensor(a, device="cuda")
    tg = np.arange(g.n, dtype=np.int32)
    for j, f in enumerate(idx):
        dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * hs[f]), T(tg))
        torch.cuda.synchronize()
        assert rel_l2(q.out_x[j], q.out_y[j], dx.cpu().numpy(), dy.cpu().numpy()) <= 1e-5
    # device-resident requests: same results as the host path
    dreq = [(srv.submit(serve.Request(q.grid, T(grids[q.grid][1][idx]))), q) for q, idx in mix[:6]]
    srv.run_until_idle()
    torch.cuda.synchronize()
    for d, q in dreq:
        assert d.status == "done" and isinstance(d.out_x, torch.Tensor)
        assert np.array_equal(d.out_x.cpu().numpy(), q.out_x) and np.array_equal(d.out_y.cpu().numpy(), q.out_y)
    srv.close()
