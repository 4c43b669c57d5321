"""GPU tests on the shapes of the benchmark configurations.

* A MOM6-style logically rectangular lon-lat grid (the cfg1 shape at 1 degree,
  360 x 180 centres before the land mask, leaf 200): the three MOM6 entry
  points in ref_compat mode agree with the oracle to 1e-12, and correct mode
  agrees with the FP64 direct sum.  Spacing shrinks toward the poles here,
  which the Fibonacci grids of the other tests do not exercise.
* The 2,313,486-cell cfg2 grid (the size the metric is quoted on) at d=8 and
  d=10: the FP64 accurate form and the batched mixed-precision form against the
  FP64 direct sum on seeded sampled targets.  The batched bar is 1e-5 rel-L2.
"""
import numpy as np
import pytest

from conftest import rel_l2

TOL_PARITY = 1e-12   # GPU plain FP64 form vs the oracle (same operation order)

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_mom6_lonlat_grid_matches_oracle_and_direct_sum():
    torch = _torch()
    import salgpu as S
    from salgpu import synth
    from oracle import oracle as O
    g = synth.lonlat_grid(nlon=360, nlat=180, seed=3)
    h = synth.config_ssh("cfg1", g, nfields=1, seed=13)[0]
    thresh, d = 200, 8
    ot = O.tree_traverse(g.xs, g.ys, g.zs, thresh)
    ppan = O.assign_points_to_panels(ot, g.xs, g.ys, g.zs)
    pc, pp = O.single_tree_traversal(ot, 0.7, thresh, g.xs, g.ys, g.zs)
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, thresh)
    # ref_compat: the reference's transposed proxy weights, bit-for-bit operation order
    w_ref = O.proxy_source_compute(ot, ppan, g.xs, g.ys, g.zs, h, g.areas, d, transposed=True)
    ox, oy = O.pc_compute(ot, pc, g.xs, g.ys, g.zs, d, w_ref)
    px, py = O.pp_compute(ot, pp, g.xs, g.ys, g.zs, g.areas, h)
    grid = S.mom6_grid(pt, pc, pp, g.xs, g.ys, g.zs, g.areas, d, ref_compat=True)
    w = np.zeros_like(w_ref)
    grid.proxy_source_compute_host(h, w)
    assert np.linalg.norm(w - w_ref) <= TOL_PARITY * np.linalg.norm(w_ref)
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    grid.pc_compute_host(w_ref, gx, gy)
    assert rel_l2(gx, gy, ox, oy) <= TOL_PARITY
    qx, qy = np.zeros(g.n), np.zeros(g.n)
    grid.pp_compute_host(h, qx, qy)
    assert rel_l2(qx, qy, px, py) <= TOL_PARITY
    # correct mode (untransposed weights) converges to the direct sum
    grid_c = S.mom6_grid(pt, pc, pp, g.xs, g.ys, g.zs, g.areas, d, ref_compat=False)
    wc = np.zeros_like(w_ref)
    grid_c.proxy_source_compute_host(h, wc)
    cx, cy = np.zeros(g.n), np.zeros(g.n)
    grid_c.pc_compute_host(wc, cx, cy)
    grid_c.pp_compute_host(h, cx, cy)
    tg = np.sort(np.random.default_rng(8).choice(g.n, 3000, replace=False)).astype(np.int32)
    T = lambda a: torch.tensor(a, device="cuda")
    dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * h), T(tg))
    err = rel_l2(cx[tg], cy[tg], dx.cpu().numpy(), dy.cpu().numpy())
    print(f"lon-lat MOM6 correct mode vs direct sum: {err:.3e}")
    assert err <= 1e-4


@pytest.mark.parametrize("degree", [8, 10])
def test_cfg2_full_size_accurate_and_batched_forms_vs_direct_sum(degree):
    torch = _torch()
    import salgpu as S
    from salgpu import synth
    g = synth.config_grid("cfg2")
    hs = synth.config_ssh("cfg2", g, nfields=2, seed=17)
    t = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 200)
    L = S.dual_tree_traversal(t, 0.7, 200)
    grid = S.Grid(t, g.xs, g.ys, g.zs, g.areas, degree, S.MODE_DTT, L, max_fields=64)
    ssh = torch.tensor(hs, device="cuda")
    ax, ay = grid.solve(ssh, form=S.FORM_ACCURATE)
    mx, my = grid.solve(ssh, form=S.FORM_MIXED)
    torch.cuda.synchronize()
    tg = np.sort(np.random.default_rng(99).choice(g.n, 2000, replace=False)).astype(np.int32)
    T = lambda a: torch.tensor(a, device="cuda")
    idx = T(tg).long()
    for f in range(2):
        dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * hs[f]), T(tg))
        d = [dx.cpu().numpy(), dy.cpu().numpy()]
        ea = rel_l2(ax[f][idx].cpu().numpy(), ay[f][idx].cpu().numpy(), *d)
        em = rel_l2(mx[f][idx].cpu().numpy(), my[f][idx].cpu().numpy(), *d)
        print(f"cfg2 d={degree} field {f}: accurate {ea:.3e}  batched {em:.3e}")
        assert ea <= 1e-6
        assert em <= 1e-5
