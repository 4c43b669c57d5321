"""GPU parity of the FP64 treecode against the CPU oracle, through the C ABI.

Bars:
  * SAL_FORM_REF       vs oracle fast_sum / mom6 path:   rel-L2 <= 1e-12
  * SAL_FORM_ACCURATE  vs oracle fast_sum_cart:          rel-L2 <= 1e-12
  * GPU direct sum     vs oracle direct sum:             rel-L2 <= 1e-13
  * SAL_FORM_ACCURATE  vs FP64 direct sum (d = 8):       rel-L2 <= 1e-6
The tolerances are on rel-L2 over all reported targets of both components.
"""
import numpy as np
import pytest

from conftest import grid_and_ssh, rel_l2

pytestmark = pytest.mark.gpu

TOL_PARITY = 1e-12


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _setup(name, thresh, degree, theta=0.7):
    import salgpu as S
    from oracle import oracle as O
    g, h = grid_and_ssh(name)
    ot = O.tree_traverse(g.xs, g.ys, g.zs, thresh)
    L = O.dual_tree_traversal(ot, theta, thresh)
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, thresh)
    return S, O, g, h[0], ot, pt, L


@pytest.mark.parametrize("name,thresh,degree", [("small_3000", 20, 8), ("small_3000", 10, 2), ("cfg0", 100, 8)])
def test_fast_sum_ref_matches_oracle(name, thresh, degree):
    _torch()
    S, O, g, h, ot, pt, L = _setup(name, thresh, degree)
    ox, oy = O.fast_sum(ot, L, g.xs, g.ys, g.zs, g.areas, h, degree, nranks=8)
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    S.fast_sum(gx, gy, L, pt, g.xs, g.ys, g.zs, g.areas, h, g.n, degree)
    assert rel_l2(gx, gy, ox, oy) <= TOL_PARITY


def test_fast_sum_adds_into_outputs_and_rank_split():
    """intent(inout) semantics and the MOD(i, P) == rank split
    (fast_sum_module.f90:303-304) summed over ranks."""
    _torch()
    S, O, g, h, ot, pt, L = _setup("small_3000", 20, 8)
    ox, oy = O.fast_sum(ot, L, g.xs, g.ys, g.zs, g.areas, h, 8)
    gx, gy = np.ones(g.n), np.ones(g.n)
    for r in range(3):
        S.fast_sum(gx, gy, L, pt, g.xs, g.ys, g.zs, g.areas, h, g.n, 8, rank=r, process_count=3)
    assert rel_l2(gx - 1.0, gy - 1.0, ox, oy) <= TOL_PARITY


@pytest.mark.parametrize("name,thresh", [("small_3000", 20), ("cfg0", 100)])
def test_accurate_form_matches_oracle_cartesian(name, thresh):
    _torch()
    S, O, g, h, ot, pt, L = _setup(name, thresh, 8)
    ox, oy = O.fast_sum_cart(ot, L, g.xs, g.ys, g.zs, g.areas, h, 8, 8)
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    S.dropin_config(S.FORM_ACCURATE)
    try:
        S.fast_sum(gx, gy, L, pt, g.xs, g.ys, g.zs, g.areas, h, g.n, 8)
    finally:
        S.dropin_config(S.FORM_REF)
    assert rel_l2(gx, gy, ox, oy) <= TOL_PARITY


def test_device_solve_batched_equals_host_entry():
    torch = _torch()
    import salgpu as S
    g, hs = grid_and_ssh("small_3000", nfields=3, seed=5)
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 20)
    L = S.dual_tree_traversal(pt, 0.7, 20)
    grid = S.Grid(pt, g.xs, g.ys, g.zs, g.areas, 8, S.MODE_DTT, L, max_fields=3)
    ssh = torch.tensor(hs, device="cuda")
    for form in (S.FORM_REF, S.FORM_ACCURATE):
        ox, oy = grid.solve(ssh, form=form)
        torch.cuda.synchronize()
        grid.sync()
        for f in range(3):
            hx, hy = np.zeros(g.n), np.zeros(g.n)
            grid.fast_sum_host(hs[f], hx, hy, form)
            assert np.array_equal(ox[f].cpu().numpy(), hx) and np.array_equal(oy[f].cpu().numpy(), hy)


@pytest.mark.parametrize("ref_compat", [True, False])
def test_mom6_entry_points_match_oracle(ref_compat):
    _torch()
    import salgpu as S
    from oracle import oracle as O
    g, hh = grid_and_ssh("small_3000")
    h = hh[0]
    thresh, d = 20, 8
    ot = O.tree_traverse(g.xs, g.ys, g.zs, thresh)
    ppan = O.assign_points_to_panels(ot, g.xs, g.ys, g.zs)
    pc, pp = O.single_tree_traversal(ot, 0.7, thresh, g.xs, g.ys, g.zs)
    w_ref = O.proxy_source_compute(ot, ppan, g.xs, g.ys, g.zs, h, g.areas, d, transposed=ref_compat)
    ox, oy = O.pc_compute(ot, pc, g.xs, g.ys, g.zs, d, w_ref)
    px, py = O.pp_compute(ot, pp, g.xs, g.ys, g.zs, g.areas, h)

    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, thresh)
    grid = S.mom6_grid(pt, pc, pp, g.xs, g.ys, g.zs, g.areas, d, ref_compat=ref_compat)
    w = np.zeros_like(w_ref)
    grid.proxy_source_compute_host(h, w)
    assert np.linalg.norm(w - w_ref) <= TOL_PARITY * np.linalg.norm(w_ref)
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    grid.pc_compute_host(w_ref, gx, gy)
    assert rel_l2(gx, gy, ox, oy) <= TOL_PARITY
    qx, qy = np.zeros(g.n), np.zeros(g.n)
    grid.pp_compute_host(h, qx, qy)
    assert rel_l2(qx, qy, px, py) <= TOL_PARITY


def test_direct_sum_matches_oracle():
    torch = _torch()
    import salgpu as S
    from oracle import oracle as O
    g, hh = grid_and_ssh("cfg0")
    h = hh[0]
    tg = np.random.default_rng(3).choice(g.n, 2000, replace=False).astype(np.int32)
    dx, dy = O.direct_sum(g.xs, g.ys, g.zs, g.areas, h, tg)
    T = lambda a: torch.tensor(a, device="cuda")
    gx, gy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * h), torch.tensor(tg, device="cuda"))
    torch.cuda.synchronize()
    assert rel_l2(gx.cpu().numpy(), gy.cpu().numpy(), dx, dy) <= 1e-13


def test_accurate_form_converges_to_direct_sum():
    torch = _torch()
    import salgpu as S
    g, hh = grid_and_ssh("cfg0")
    h = hh[0]
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 100)
    L = S.dual_tree_traversal(pt, 0.7, 100)
    T = lambda a: torch.tensor(a, device="cuda")
    tg = np.arange(g.n, dtype=np.int32)
    dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * h), T(tg))
    errs = {}
    for d in (6, 8, 10):
        grid = S.Grid(pt, g.xs, g.ys, g.zs, g.areas, d, S.MODE_DTT, L)
        ox, oy = grid.solve(T(h), form=S.FORM_ACCURATE)
        torch.cuda.synchronize()
        errs[d] = rel_l2(ox.cpu().numpy(), oy.cpu().numpy(), dx.cpu().numpy(), dy.cpu().numpy())
    assert errs[8] <= 1e-6 and errs[10] < errs[8] < errs[6]
