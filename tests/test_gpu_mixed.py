"""GPU tests of the batched mixed-precision form (SAL_FORM_MIXED).

Bars (rel-L2 over both components, per field):
  * vs the FP64 accurate form (same algorithm):  <= 5e-6
  * vs the FP64 direct sum (all cells):           <= 1e-5
  * a field alone vs the same field in a batch:   identical (the tensor-core
    columns of different fields never mix)
"""
import numpy as np
import pytest

from conftest import grid_and_ssh, rel_l2

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _grid(name, thresh, nfields, seed=11, degree=8, max_fields=None):
    """A grid and nfields seeded fields.  max_fields > 32 gives 64-field blocks
    (the tcgen05 passes) whatever nfields is; the default sizes the blocks for
    nfields (32-field mma.sync blocks below 33)."""
    import salgpu as S
    g, hs = grid_and_ssh(name, nfields=nfields, seed=seed)
    t = S.tree_traverse(g.xs, g.ys, g.zs, g.n, thresh)
    L = S.dual_tree_traversal(t, 0.7, thresh)
    mf = nfields if max_fields is None else max_fields
    return S, g, hs, S.Grid(t, g.xs, g.ys, g.zs, g.areas, degree, S.MODE_DTT, L, max_fields=mf)


@pytest.mark.parametrize("name,thresh", [("small_3000", 20), ("cfg0", 100)])
def test_mixed_matches_fp64_accurate_and_direct_sum(name, thresh):
    torch = _torch()
    S, g, hs, grid = _grid(name, thresh, 5)
    ssh = torch.tensor(hs, device="cuda")
    mx, my = grid.solve(ssh, form=S.FORM_MIXED)
    ax, ay = grid.solve(ssh, form=S.FORM_ACCURATE)
    T = lambda a: torch.tensor(a, device="cuda")
    tg = T(np.arange(g.n, dtype=np.int32))
    torch.cuda.synchronize()
    for f in range(5):
        dx, dy = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * hs[f]), tg)
        m = [v[f].cpu().numpy() for v in (mx, my, ax, ay)]
        d = [dx.cpu().numpy(), dy.cpu().numpy()]
        assert rel_l2(m[0], m[1], m[2], m[3]) <= 5e-6
        assert rel_l2(m[0], m[1], d[0], d[1]) <= 1e-5


def test_mixed_batch_invariance_and_field_blocks():
    torch = _torch()
    S, g, hs, grid = _grid("small_3000", 20, 70, seed=3)
    ssh = torch.tensor(hs, device="cuda")
    bx, by = grid.solve(ssh[:40], form=S.FORM_MIXED)          # one 64-field block
    cx, cy = grid.solve(ssh, form=S.FORM_MIXED)               # two blocks (64 + 6)
    torch.cuda.synchronize()
    for f in (0, 17, 39):
        ox, oy = grid.solve(ssh[f:f + 1], form=S.FORM_MIXED)  # the field alone
        torch.cuda.synchronize()
        assert torch.equal(ox[0], bx[f]) and torch.equal(oy[0], by[f])
        assert torch.equal(ox[0], cx[f]) and torch.equal(oy[0], cy[f])
    ax, ay = grid.solve(ssh[65:70], form=S.FORM_ACCURATE)
    torch.cuda.synchronize()
    for f in range(5):
        assert rel_l2(cx[65 + f].cpu().numpy(), cy[65 + f].cpu().numpy(), ax[f].cpu().numpy(),
                      ay[f].cpu().numpy()) <= 5e-6


def test_tcgen05_leaf_pass_matches_mma_sync_leaf_pass():
    """Grids sized for 64-field blocks run the leaf pass on tcgen05 (tensor
    memory accumulators); 32-field blocks run it with warp-level mma.sync.
    Both carry the same algorithm and TF32 split, so they agree to FP32
    rounding."""
    torch = _torch()
    import salgpu as S
    g, hs = grid_and_ssh("cfg0", nfields=6, seed=9)
    t = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 100)
    L = S.dual_tree_traversal(t, 0.7, 100)
    g32 = S.Grid(t, g.xs, g.ys, g.zs, g.areas, 8, S.MODE_DTT, L, max_fields=32)
    g64 = S.Grid(t, g.xs, g.ys, g.zs, g.areas, 8, S.MODE_DTT, L, max_fields=64)
    ssh = torch.tensor(hs, device="cuda")
    ax, ay = g32.solve(ssh, form=S.FORM_MIXED)
    bx, by = g64.solve(ssh, form=S.FORM_MIXED)
    torch.cuda.synchronize()
    g64.sync()
    for f in range(6):
        assert rel_l2(bx[f].cpu().numpy(), by[f].cpu().numpy(), ax[f].cpu().numpy(), ay[f].cpu().numpy()) <= 2e-6


@pytest.mark.parametrize("degree", [9, 12])
def test_tcgen05_passes_at_other_degrees(degree):
    """P = (d+1)^2 = 100 and 169 proxies: the upward pass's groups cover more
    than 85 and more than 128 proxy rows, the proxy pass's groups are cut in
    85-row chunks.  The batched form stays within 5e-6 of the FP64 accurate
    form (and has no NaN from tile rows left unwritten)."""
    torch = _torch()
    import salgpu as S
    g, hs = grid_and_ssh("small_3000", nfields=3, seed=6)
    t = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 20)
    L = S.dual_tree_traversal(t, 0.7, 20)
    grid = S.Grid(t, g.xs, g.ys, g.zs, g.areas, degree, S.MODE_DTT, L, max_fields=64)
    ssh = torch.tensor(hs, device="cuda")
    mx, my = grid.solve(ssh, form=S.FORM_MIXED)
    ax, ay = grid.solve(ssh, form=S.FORM_ACCURATE)
    torch.cuda.synchronize()
    assert not (torch.isnan(mx).any() or torch.isnan(my).any())
    for f in range(3):
        assert rel_l2(mx[f].cpu().numpy(), my[f].cpu().numpy(), ax[f].cpu().numpy(), ay[f].cpu().numpy()) <= 5e-6


def test_host_entry_points_and_pipelined_calls_match_device_solve():
    """sal_solve_host and three pipelined sal_solve_host_async calls (two
    staging slots, inputs alternating) give the device solve's results bit for
    bit; the second input has its fields reversed, so its results come back
    reversed."""
    torch = _torch()
    S, g, hs, grid = _grid("small_3000", 20, 64, seed=5)
    dx, dy = grid.solve(torch.tensor(hs, device="cuda"), form=S.FORM_MIXED)
    dx, dy = dx.cpu(), dy.cpu()
    h_in = [torch.tensor(hs).pin_memory(), torch.tensor(hs[::-1].copy()).pin_memory()]
    outs = [(torch.empty_like(h_in[0]).pin_memory(), torch.empty_like(h_in[0]).pin_memory()) for _ in range(3)]
    for k in range(3):
        grid.solve_host_async(h_in[k % 2].numpy(), outs[k][0].numpy(), outs[k][1].numpy(), S.FORM_MIXED)
    grid.solve_host_wait()
    sx, sy = torch.empty_like(h_in[0]).pin_memory(), torch.empty_like(h_in[0]).pin_memory()
    grid.solve_host(h_in[0].numpy(), sx.numpy(), sy.numpy(), S.FORM_MIXED)
    assert torch.equal(sx, dx) and torch.equal(sy, dy)
    for k in (0, 2):
        assert torch.equal(outs[k][0], dx) and torch.equal(outs[k][1], dy)
    assert torch.equal(outs[1][0], dx.flip(0)) and torch.equal(outs[1][1], dy.flip(0))


def test_graph_replay_matches_kernel_launches():
    """With graphs on, the first batched solve of a call shape runs and is
    captured; later solves of that shape replay the graph and give the same
    results bit for bit, on new field values, for two widths."""
    torch = _torch()
    S, g, hs, grid = _grid("small_3000", 20, 64, seed=7)
    ssh = torch.tensor(hs, device="cuda")
    ref = [grid.solve(ssh[:w], form=S.FORM_MIXED) for w in (64, 5)]
    ref2 = grid.solve(ssh.flip(0)[:5].contiguous(), form=S.FORM_MIXED)
    torch.cuda.synchronize()
    grid.set_graphs(True)
    st = torch.cuda.Stream()
    buf = torch.empty_like(ssh)
    ox, oy = torch.empty_like(ssh), torch.empty_like(ssh)
    with torch.cuda.stream(st):
        for it in range(3):
            for w, (rx, ry) in zip((64, 5), ref):
                buf[:w].copy_(ssh[:w])
                grid.solve(buf[:w], form=S.FORM_MIXED, out=(ox[:w], oy[:w]), stream=st.cuda_stream)
                st.synchronize()
                assert torch.equal(ox[:w], rx) and torch.equal(oy[:w], ry)
        buf[:5].copy_(ssh.flip(0)[:5])
        grid.solve(buf[:5], form=S.FORM_MIXED, out=(ox[:5], oy[:5]), stream=st.cuda_stream)
        st.synchronize()
        assert torch.equal(ox[:5], ref2[0]) and torch.equal(oy[:5], ref2[1])
    grid.set_graphs(False)


@pytest.mark.parametrize("degree", [8, 10])
def test_tree_passes_match_direct_passes(degree):
    """The batched form's tree passes (leaf-level upward pass plus
    child-to-parent transfers; parent-to-child transfers plus one DOWN item
    per leaf) reproduce its direct per-slot passes: the transfers are exact in
    exact arithmetic, so the two agree to FP32 rounding, and both stay within
    the bars against the FP64 accurate form and the direct sum.  The basis
    work they report falls."""
    torch = _torch()
    S, g, hs, grid = _grid("small_20000", 60, 4, seed=2, degree=degree, max_fields=64)
    ssh = torch.tensor(hs, device="cuda")
    assert grid.tune()["tree_passes"] == 1 and grid.tune()["field_block"] == 64
    tx, ty = grid.solve(ssh, form=S.FORM_MIXED)
    st_tree = grid.stats()
    grid.tune(tree_passes=0)
    dx_, dy_ = grid.solve(ssh, form=S.FORM_MIXED)
    st_direct = grid.stats()
    ax, ay = grid.solve(ssh, form=S.FORM_ACCURATE)
    torch.cuda.synchronize()
    grid.sync()
    assert st_tree["macs_up_batched"] < 0.5 * st_direct["macs_up_batched"]
    assert st_tree["macs_down_batched"] < 0.5 * st_direct["macs_down_batched"]
    assert st_direct["macs_up_batched"] == st_direct["macs_up"]
    T = lambda a: torch.tensor(a, device="cuda")
    tg = np.sort(np.random.default_rng(4).choice(g.n, 3000, replace=False)).astype(np.int32)
    for f in range(4):
        t = [v[f].cpu().numpy() for v in (tx, ty, dx_, dy_, ax, ay)]
        assert rel_l2(t[0], t[1], t[2], t[3]) <= 2e-6
        assert rel_l2(t[0], t[1], t[4], t[5]) <= 5e-6
        rx, ry = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * hs[f]), T(tg))
        assert rel_l2(t[0][tg], t[1][tg], rx.cpu().numpy(), ry.cpu().numpy()) <= 1e-5


def test_tune_settings_round_trip_and_keep_accuracy():
    """Every choice sal_grid_tune_set accepts re-cuts the plan (or the launch
    shape) and the batched form stays within its bar of the FP64 accurate
    form; bad settings are refused."""
    torch = _torch()
    S, g, hs, grid = _grid("small_20000", 60, 3, seed=8, max_fields=64)
    ssh = torch.tensor(hs, device="cuda")
    ax, ay = grid.solve(ssh, form=S.FORM_ACCURATE)
    settings = [dict(chain_ksteps=8), dict(chain_ksteps=64), dict(cta_groups=3), dict(proxy_unit_kpairs=100),
                dict(tree_passes=0, up_chunk=1000), dict(f16=1), dict(tree_passes=1), dict(f16=0),
                dict(field_block=32), dict(field_block=64, tree_passes=1)]
    for ch in settings:
        now = grid.tune(**ch)
        for k, v in ch.items():
            assert now[k] == v
        mx, my = grid.solve(ssh, form=S.FORM_MIXED)
        torch.cuda.synchronize()
        grid.sync()
        for f in range(3):
            assert rel_l2(mx[f].cpu().numpy(), my[f].cpu().numpy(), ax[f].cpu().numpy(),
                          ay[f].cpu().numpy()) <= 5e-6, ch
    with pytest.raises(S.SalError):
        grid.tune(chain_ksteps=0)
    with pytest.raises(S.SalError):
        grid.tune(field_block=48)


def test_autotune_picks_a_setting_within_the_bar():
    torch = _torch()
    S, g, hs, grid = _grid("small_20000", 60, 4, seed=12, max_fields=64)
    ssh = torch.tensor(hs, device="cuda")
    best, ms_best, ms_start = grid.autotune(ssh, ntargets=1000, max_rel_err=5e-6)
    assert grid.tune() == best
    assert 0 < ms_best <= ms_start * 1.05
    mx, my = grid.solve(ssh, form=S.FORM_MIXED)
    ax, ay = grid.solve(ssh, form=S.FORM_ACCURATE)
    torch.cuda.synchronize()
    grid.sync()
    for f in range(4):
        assert rel_l2(mx[f].cpu().numpy(), my[f].cpu().numpy(), ax[f].cpu().numpy(), ay[f].cpu().numpy()) <= 5e-6
    with pytest.raises(S.SalError):
        grid.autotune(ssh, ntargets=1000, max_rel_err=1e-12)
    assert grid.tune() == best        # a failed search leaves the setting as it was


def test_joint_solve_of_uneven_grids_equals_separate_solves():
    """sal_solve_joint runs the leaf passes of grids of different sizes in one
    launch.  Each target group's work is the same wherever it runs, so every
    result equals the grid's own sal_solve bit for bit."""
    torch = _torch()
    import salgpu as S
    cases = [("small_3000", 20, 3), ("small_20000", 60, 64), ("cfg0", 100, 7)]
    grids, sshs = [], []
    for name, thresh, nf in cases:
        S_, g, hs, grid = _grid(name, thresh, nf, seed=21)
        grid2 = S.Grid(S.tree_traverse(g.xs, g.ys, g.zs, g.n, thresh), g.xs, g.ys, g.zs, g.areas, 8, S.MODE_DTT,
                       S.dual_tree_traversal(S.tree_traverse(g.xs, g.ys, g.zs, g.n, thresh), 0.7, thresh),
                       max_fields=64)
        grids.append(grid2)
        sshs.append(torch.tensor(hs, device="cuda"))
    alone = [g.solve(s, form=S.FORM_MIXED) for g, s in zip(grids, sshs)]
    joint = S.solve_joint(grids, sshs)
    torch.cuda.synchronize()
    for g in grids:
        g.sync()
    for (ax, ay), (jx, jy) in zip(alone, joint):
        assert torch.equal(ax, jx) and torch.equal(ay, jy)
    with pytest.raises(S.SalError):
        S.solve_joint([grids[0], grids[0]], [sshs[0], sshs[0]])
    g9 = _grid("small_3000", 20, 3, seed=21, degree=9)[3]
    with pytest.raises(S.SalError):
        S.solve_joint([grids[0], g9], [sshs[0], sshs[0]])


@pytest.mark.parametrize("nfields", [64, 32])
def test_mixed_bytes_estimate_equals_the_allocation(nfields):
    """stats()["mixed_bytes"] before the first batched solve (what the serving
    loop budgets with) equals what that solve allocates, for 64-field
    (tcgen05) and 32-field (mma.sync) blocks."""
    torch = _torch()
    S, g, hs, grid = _grid("cfg0", 100, nfields)
    est = grid.stats()["mixed_bytes"]
    before = grid.stats()["device_bytes"]
    grid.solve(torch.tensor(hs, device="cuda"), form=S.FORM_MIXED)
    torch.cuda.synchronize()
    st = grid.stats()
    assert st["mixed_bytes"] == est
    assert st["device_bytes"] - before == est


@pytest.mark.parametrize("degree,tree", [(8, 1), (10, 1), (8, 0)])
def test_f16_leaf_pass_matches_tf32_and_direct_sum(degree, tree):
    """The FP16 leaf pass (sal_tune.f16 = 1: kind::f16 MMAs of 16 sources,
    FP16 hi + lo operands scaled by powers of two per target and per field)
    against the TF32 leaf pass and the FP64 accurate form (5e-6) and the FP64
    direct sum (1e-5), with the tree passes and with the direct passes (DOWN
    items between the kernel items), on fields of very different amplitude
    (the per-field scales must keep small fields as accurate as large ones)."""
    torch = _torch()
    S, g, hs, grid = _grid("small_20000", 60, 6, seed=5, degree=degree, max_fields=64)
    hs = hs * np.array([1.0, 1e-3, 1e3, 1e-6, 1.0, 5.0])[:, None]
    ssh = torch.tensor(hs, device="cuda")
    grid.tune(tree_passes=tree, f16=0)
    tx, ty = grid.solve(ssh, form=S.FORM_MIXED)
    grid.tune(f16=1)
    assert grid.tune()["f16"] == 1
    fx, fy = grid.solve(ssh, form=S.FORM_MIXED)
    ax, ay = grid.solve(ssh, form=S.FORM_ACCURATE)
    torch.cuda.synchronize()
    grid.sync()
    T = lambda a: torch.tensor(a, device="cuda")
    tg = np.sort(np.random.default_rng(6).choice(g.n, 3000, replace=False)).astype(np.int32)
    for f in range(6):
        t = [v[f].cpu().numpy() for v in (fx, fy, tx, ty, ax, ay)]
        assert np.all(np.isfinite(t[0])) and np.all(np.isfinite(t[1]))
        assert rel_l2(t[0], t[1], t[2], t[3]) <= 5e-6
        assert rel_l2(t[0], t[1], t[4], t[5]) <= 5e-6
        rx, ry = S.direct_sum(T(g.xs), T(g.ys), T(g.zs), T(g.areas * hs[f]), T(tg))
        assert rel_l2(t[0][tg], t[1][tg], rx.cpu().numpy(), ry.cpu().numpy()) <= 1e-5


def test_f16_joint_solve_equals_separate_solves_and_memory_estimate():
    """FP16 leaf passes of two grids in one launch equal their separate
    solves bit for bit; the batched-memory estimate counts the FP16 buffers."""
    torch = _torch()
    grids, sshs = [], []
    for name, thresh in (("small_3000", 20), ("cfg0", 100)):
        S, g, hs, grid = _grid(name, thresh, 5, seed=9, max_fields=64)
        grid.tune(f16=1)
        est = grid.stats()["mixed_bytes"]
        before = grid.stats()["device_bytes"]
        grids.append(grid)
        sshs.append(torch.tensor(hs, device="cuda"))
        sep = grid.solve(sshs[-1], form=S.FORM_MIXED)
        torch.cuda.synchronize()
        assert grid.stats()["device_bytes"] - before == est
        grid.sep = [v.clone() for v in sep]
    outs = S.solve_joint(grids, sshs)
    torch.cuda.synchronize()
    for grid, (ox, oy) in zip(grids, outs):
        assert torch.equal(ox, grid.sep[0]) and torch.equal(oy, grid.sep[1])


def test_f16_batch_invariance_and_zero_field():
    """FP16 leaf operands: every field's scale is its own, so a field's result
    is the same bit for bit alone and inside a batch of fields of any
    amplitude, and an all-zero field gives exact zeros (scale 1, no NaN)."""
    torch = _torch()
    S, g, hs, grid = _grid("small_3000", 20, 5, seed=17, max_fields=64)
    hs = hs * np.array([1.0, 1e4, 1e-5, 0.0, 3.0])[:, None]
    ssh = torch.tensor(hs, device="cuda")
    grid.tune(f16=1)
    bx, by = grid.solve(ssh, form=S.FORM_MIXED)
    torch.cuda.synchronize()
    assert torch.count_nonzero(bx[3]) == 0 and torch.count_nonzero(by[3]) == 0
    for f in (0, 2, 4):
        ox, oy = grid.solve(ssh[f:f + 1], form=S.FORM_MIXED)
        torch.cuda.synchronize()
        assert torch.equal(ox[0], bx[f]) and torch.equal(oy[0], by[f])


@pytest.mark.parametrize("degree,tree,every", [(8, 1, 1), (8, 0, 1), (10, 1, 1), (8, 1, 2), (8, 0, 3)])
def test_tile_store_records_and_replays_bitwise(degree, tree, every):
    """sal_tune.tile_store = 1: the first FP16 leaf pass records its kernel
    tiles (near-field, proxy and DOWN rows) in device memory and later solves
    replay them; tile_store = m > 1 keeps one item in m of each group, which
    later solves copy while the producers compute the others.  The recording solve, the replays (other fields, fewer fields,
    graphs on a stream) and the solve after switching the store off again all
    equal the computing leaf pass bit for bit; the memory estimate counts the
    store, whose size the stats report."""
    torch = _torch()
    S, g, hs, grid = _grid("small_20000", 60, 6, seed=23, degree=degree, max_fields=64)
    hs = hs * np.array([1.0, 1e-3, 1e3, 1e-6, 0.0, 5.0])[:, None]
    ssh = torch.tensor(hs, device="cuda")
    grid.tune(tree_passes=tree, f16=1, tile_store=0)
    ref = [v.clone() for v in grid.solve(ssh, form=S.FORM_MIXED)]
    ref3 = [v.clone() for v in grid.solve(ssh[2:5], form=S.FORM_MIXED)]
    torch.cuda.synchronize()
    full_bytes = grid.stats()["tile_store_bytes"]
    grid.tune(tile_store=every)
    assert grid.tune()["tile_store"] == every
    tile_bytes = grid.stats()["tile_store_bytes"]
    assert 0 < tile_bytes <= full_bytes and (every == 1) == (tile_bytes == full_bytes)
    est = grid.stats()["mixed_bytes"]
    before = grid.stats()["device_bytes"]
    for k in range(3):   # record, then replays
        ox, oy = grid.solve(ssh, form=S.FORM_MIXED)
        torch.cuda.synchronize()
        assert torch.equal(ox, ref[0]) and torch.equal(oy, ref[1]), k
    assert grid.stats()["device_bytes"] - before == est
    assert est > tile_bytes
    ox, oy = grid.solve(ssh[2:5], form=S.FORM_MIXED)
    torch.cuda.synchronize()
    assert torch.equal(ox, ref3[0]) and torch.equal(oy, ref3[1])
    # captured graphs replay the recorded tiles too
    # (a call shape is captured on its second solve and launched as a graph
    # from its third)
    grid.set_graphs(True)
    s = torch.cuda.Stream()
    ox, oy = torch.empty_like(ssh), torch.empty_like(ssh)
    for k in range(4):
        with torch.cuda.stream(s):
            ox.zero_()
            oy.zero_()
            grid.solve(ssh, form=S.FORM_MIXED, out=(ox, oy), stream=s.cuda_stream)
        s.synchronize()
        assert torch.equal(ox, ref[0]) and torch.equal(oy, ref[1]), k
    grid.set_graphs(False)
    grid.tune(tile_store=0)
    ox, oy = grid.solve(ssh, form=S.FORM_MIXED)
    torch.cuda.synchronize()
    assert torch.equal(ox, ref[0]) and torch.equal(oy, ref[1])
    grid.sync()
