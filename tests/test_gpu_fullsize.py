"""GPU parity at the benchmark configurations' full sizes.

Small-grid parity cannot see failures that only appear at scale (32-bit pool
offsets, item splits at the staging limit, unit budgets, plan sizes).  These
tests run the configurations' own grids:

* cfg2, 2,313,486 cells, d = 8, theta = 0.7, leaf 200, plain FP64 form
  (SAL_FORM_REF) against the oracle's fast_sum on the same share of the
  interaction list: the MPI split MOD(i, 8) == 0 of fast_sum_module.f90:304,
  which both sides evaluate (one of the eight ranks' work, so the oracle
  finishes in seconds on the host's cores).  Bar: rel-L2 <= 1e-12.
* cfg2, the whole list: the plain FP64 form, the accurate form and the batched
  form against the FP64 direct sum on 10,000 seeded targets.
* cfg1, the 0.25 degree 1440 x 720 lon-lat grid (leaf 200, d = 8) in
  ref_compat mode, through the reference-signature entry points:
  proxy_source_compute over every panel, and pc_compute / pp_compute at 4,000
  seeded targets (the oracle evaluates every list entry of
  those targets, so their sums are complete), against the oracle.  Bar:
  rel-L2 <= 1e-12.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_PARITY = 1e-12


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


_CFG2 = {}


def _cfg2():
    """The cfg2 grid, two SSH fields, the oracle's tree and DTT list (cached)."""
    if not _CFG2:
        from salgpu import synth
        from oracle import oracle as O
        g = synth.config_grid("cfg2")
        hs = synth.config_ssh("cfg2", g, nfields=2, seed=17)
        ot = O.tree_traverse(g.xs, g.ys, g.zs, 200)
        L = O.dual_tree_traversal(ot, 0.7, 200)
        _CFG2.update(g=g, hs=hs, ot=ot, L=L)
    return _CFG2


def test_cfg2_ref_form_matches_oracle_on_one_rank_share():
    _torch()
    import salgpu as S
    from oracle import oracle as O
    c = _cfg2()
    g, h, ot, L = c["g"], c["hs"][0], c["ot"], c["L"]
    P, rank = 8, 0
    i = np.arange(1, len(L) + 1)
    share = L[(i % P) == rank]
    ox, oy = O.fast_sum(ot, share, g.xs, g.ys, g.zs, g.areas, h, 8, nranks=os.cpu_count() or 1)
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 200)
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    S.fast_sum(gx, gy, L, pt, g.xs, g.ys, g.zs, g.areas, h, g.n, 8, rank=rank, process_count=P)
    S.dropin_release()
    err = rel_l2(gx, gy, ox, oy)
    mx = float(np.max(np.hypot(gx - ox, gy - oy)) / np.max(np.hypot(ox, oy)))
    print(f"cfg2 REF form, share {rank} of {P} ({len(share)} interactions): rel-L2 {err:.3e}, max/max {mx:.3e}")
    assert err <= TOL_PARITY


def test_cfg2_all_forms_vs_fp64_direct_sum_on_10000_targets():
    torch = _torch()
    import salgpu as S
    c = _cfg2()
    g, hs = c["g"], c["hs"]
    t = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 200)
    L = S.dual_tree_traversal(t, 0.7, 200)
    grid = S.Grid(t, g.xs, g.ys, g.zs, g.areas, 8, S.MODE_DTT, L, max_fields=64)
    ssh = torch.tensor(hs, device="cuda")
    out = {form: grid.solve(ssh, form=form) for form in (S.FORM_REF, S.FORM_ACCURATE, S.FORM_MIXED)}
    torch.cuda.synchronize()
    grid.sync()
    tg = np.sort(np.random.default_rng(99).choice(g.n, 10000, replace=False)).astype(np.int32)
    T = lambda a: torch.tensor(a, device="cuda")
    idx = T(tg).long()
    bars = {S.FORM_REF: 5e-3, S.FORM_ACCURATE: 1e-6, S.FORM_MIXED: 1e-5}
    names = {S.FORM_REF: "plain FP64", S.FORM_ACCURATE: "accurate FP64", S.FORM_MIXED: "batched mixed"}
    for f in range(2):
        dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * hs[f]), T(tg))
        d = [dx.cpu().numpy(), dy.cpu().numpy()]
        for form, (ox, oy) in out.items():
            x, y = ox[f][idx].cpu().numpy(), oy[f][idx].cpu().numpy()
            err = rel_l2(x, y, *d)
            mx = float(np.max(np.hypot(x - d[0], y - d[1])) / np.max(np.hypot(*d)))
            print(f"cfg2 d=8 field {f} {names[form]}: rel-L2 {err:.3e}, max/max {mx:.3e}")
            assert err <= bars[form]


def test_cfg1_quarter_degree_mom6_ref_compat_matches_oracle():
    _torch()
    import salgpu as S
    from salgpu import synth
    from oracle import oracle as O
    g = synth.config_grid("cfg1")
    h = synth.config_ssh("cfg1", g, nfields=1, seed=13)[0]
    thresh, d = 200, 8
    ot = O.tree_traverse(g.xs, g.ys, g.zs, thresh)
    ppan = O.assign_points_to_panels(ot, g.xs, g.ys, g.zs)
    pc, pp = O.single_tree_traversal(ot, 0.7, thresh, g.xs, g.ys, g.zs)
    w_ref = O.proxy_source_compute(ot, ppan, g.xs, g.ys, g.zs, h, g.areas, d, transposed=True)
    # the reference-signature entry points, with the oracle's own panels,
    # points_panels and lists as a Fortran caller would pass them
    panels = {k: getattr(ot, k) for k in ("level", "is_leaf", "id", "parent", "child", "face", "bounds",
                                          "pt_off", "pt_idx")}
    S.dropin_config(S.FORM_REF, S.MODE_STT_REF_COMPAT)
    w = np.zeros_like(w_ref)
    S.proxy_source_compute(w, panels, ppan, g.xs, g.ys, g.zs, h, g.areas, d, g.n)
    ew = float(np.linalg.norm(w - w_ref) / np.linalg.norm(w_ref))
    gx, gy = np.zeros(g.n), np.zeros(g.n)
    S.pc_compute(gx, gy, pc, panels, g.xs, g.ys, g.zs, d, w_ref)
    qx, qy = np.zeros(g.n), np.zeros(g.n)
    S.pp_compute(qx, qy, pp, panels, g.xs, g.ys, g.zs, g.areas, h)
    S.dropin_release()
    # the oracle on every list entry of 4,000 seeded targets
    tg = np.sort(np.random.default_rng(21).choice(g.n, 4000, replace=False))
    sel = np.zeros(g.n + 1, bool)
    sel[tg + 1] = True
    ox, oy = O.pc_compute(ot, pc[sel[pc[:, 0]]], g.xs, g.ys, g.zs, d, w_ref)
    px, py = O.pp_compute(ot, pp[sel[pp[:, 0]]], g.xs, g.ys, g.zs, g.areas, h)
    epc = rel_l2(gx[tg], gy[tg], ox[tg], oy[tg])
    epp = rel_l2(qx[tg], qy[tg], px[tg], py[tg])
    print(f"cfg1 {g.n} cells, {ot.npanels} panels, {len(pc)} PC + {len(pp)} PP entries: "
          f"weights {ew:.3e}, pc {epc:.3e}, pp {epp:.3e}")
    assert ew <= TOL_PARITY and epc <= TOL_PARITY and epp <= TOL_PARITY
