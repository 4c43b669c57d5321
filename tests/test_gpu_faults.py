"""GPU tests of the failure paths: device-side staging waits that run out, and
the host staging of the *_host entry points.

* sal_grid_inject_timeout makes the next FP64 solve's leaf pass leave each
  group's last staging copy unissued, with a short poll limit, so every group's
  last wait runs out with no copy in flight (no trap, no fault, no endless
  loop).  The host must see SAL_ETIMEOUT, the flag must clear, and the next
  solve on the same grid must match the oracle again.
* sal_solve_host and sal_solve_host_async keep device staging sized for the
  widest batch seen; when a wider batch comes the old staging is released, so
  the grid's device bytes track the current size only.
"""
import numpy as np
import pytest

from conftest import grid_and_ssh, rel_l2

pytestmark = pytest.mark.gpu

TOL_PARITY = 1e-12
POLLS = 1 << 12


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _small():
    import salgpu as S
    from oracle import oracle as O
    g, hh = grid_and_ssh("small_3000", nfields=3, seed=5)
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 20)
    L = S.dual_tree_traversal(pt, 0.7, 20)
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 20)
    ox, oy = O.fast_sum(ot, O.dual_tree_traversal(ot, 0.7, 20), g.xs, g.ys, g.zs, g.areas, hh[0], 8)
    return S, g, hh, pt, L, (ox, oy)


def test_injected_staging_timeout_is_reported_and_the_grid_recovers():
    torch = _torch()
    S, g, hh, pt, L, (ox, oy) = _small()
    grid = S.Grid(pt, g.xs, g.ys, g.zs, g.areas, 8, S.MODE_DTT, L)
    # host entry point: the time-out surfaces as SAL_ETIMEOUT from the call
    grid.inject_timeout(POLLS)
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    with pytest.raises(S.SalError) as e:
        grid.fast_sum_host(hh[0], gx, gy)
    assert e.value.code == S.SAL_ETIMEOUT
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    grid.fast_sum_host(hh[0], gx, gy)
    assert rel_l2(gx, gy, ox, oy) <= TOL_PARITY
    # device entry point: the time-out surfaces at the next sal_grid_sync
    ssh = torch.tensor(hh[0], device="cuda")
    grid.inject_timeout(POLLS)
    grid.solve(ssh)
    torch.cuda.synchronize()
    with pytest.raises(S.SalError) as e:
        grid.sync()
    assert e.value.code == S.SAL_ETIMEOUT
    grid.sync()                        # the flag was cleared
    dx, dy = grid.solve(ssh)
    torch.cuda.synchronize()
    grid.sync()
    assert rel_l2(dx.cpu().numpy(), dy.cpu().numpy(), ox, oy) <= TOL_PARITY
    # a cancelled injection does nothing
    grid.inject_timeout(POLLS)
    grid.inject_timeout(0)
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    grid.fast_sum_host(hh[0], gx, gy)
    assert rel_l2(gx, gy, ox, oy) <= TOL_PARITY


def test_host_staging_is_released_when_the_batch_grows():
    _torch()
    S, g, hh, pt, L, (ox, oy) = _small()
    grid = S.Grid(pt, g.xs, g.ys, g.zs, g.areas, 8, S.MODE_DTT, L, max_fields=3)
    base = grid.stats()["device_bytes"]
    n = g.n
    widest = 0
    for nf in (1, 2, 3, 2):
        h = np.ascontiguousarray(hh[:nf])
        x, y = np.zeros_like(h), np.zeros_like(h)
        grid.solve_host(h, x, y, S.FORM_REF)
        assert rel_l2(x[0], y[0], ox, oy) <= TOL_PARITY
        # in, out_x and out_y staging of the widest batch so far, nothing more
        widest = max(widest, nf)
        assert grid.stats()["device_bytes"] == base + 3 * 8 * n * widest
    base = grid.stats()["device_bytes"]
    # pipelined entry point: two slots, each grows on its own
    for nf in (1, 1, 2, 2, 3, 3):
        h = np.ascontiguousarray(hh[:nf])
        x, y = np.zeros_like(h), np.zeros_like(h)
        grid.solve_host_async(h, x, y, S.FORM_REF)
        grid.solve_host_wait()
        assert rel_l2(x[0], y[0], ox, oy) <= TOL_PARITY
    assert grid.stats()["device_bytes"] == base + 2 * 3 * 8 * n * 3
