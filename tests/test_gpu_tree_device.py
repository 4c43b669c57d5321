"""The device build of the tree and the dual-tree list against the host build.

tree_traverse (tree_module.f90:59-246) and dual_tree_traversal
(tree_module.f90:277-398) built on the device must give the host build's
panels (BFS order, ids, parents, children, faces, levels, bounds, radii), the
same points_inside of every panel and the same interaction list in the same
order, over the host tree and over the device tree; and a grid made from the
device build must solve bit for bit as the host-built one.  Cases: the cfg0,
cfg1 (0.25 degree lon-lat: whole columns of cells lie exactly on panel
midlines) and cfg2 (2,313,486 cells) grids, and edge cases (fewer points than
the threshold, one face only, clusters of identical points that refine to the
level cap, no points).
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _compare_trees(ht, dt):
    a, b = ht.export(), dt.export()
    for k in ("level", "is_leaf", "id", "parent", "child", "face", "pt_off", "pt_idx"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    assert np.array_equal(np.asarray(a["bounds"]), np.asarray(b["bounds"])), "panel bounds or radii differ"


def _check_grid(xs, ys, zs, thresh, theta=0.7, label=""):
    import salgpu as S
    n = len(xs)
    # the first device build at a size loads its kernels; time the second
    S.dual_tree_traversal(S.tree_traverse(xs, ys, zs, n, thresh, device=0), theta, thresh, device=0)
    t0 = time.perf_counter()
    ht = S.tree_traverse(xs, ys, zs, n, thresh)
    t1 = time.perf_counter()
    dt = S.tree_traverse(xs, ys, zs, n, thresh, device=0)
    t2 = time.perf_counter()
    hl = S.dual_tree_traversal(ht, theta, thresh)
    t3 = time.perf_counter()
    dl_host_tree = S.dual_tree_traversal(ht, theta, thresh, device=0)
    t4 = time.perf_counter()
    dl = S.dual_tree_traversal(dt, theta, thresh, device=0)
    _compare_trees(ht, dt)
    assert np.array_equal(hl, dl_host_tree), "device traversal of the host tree differs"
    assert np.array_equal(hl, dl), "device traversal of the device tree differs"
    print(f"{label} n={n} panels={ht.npanels} list={len(hl)}: tree host {t1 - t0:.3f} s device {t2 - t1:.3f} s; "
          f"list host {t3 - t2:.3f} s device {t4 - t3:.3f} s")
    return hl


@pytest.mark.parametrize("name,thresh", [("cfg0", 100), ("cfg1", 200), ("cfg2", 200)])
def test_device_build_matches_host_on_config_grids(name, thresh):
    _torch()
    from salgpu import synth
    g = synth.config_grid(name)
    _check_grid(g.xs, g.ys, g.zs, thresh, label=name)


def test_grid_from_device_build_solves_bitwise_as_host_build():
    """A grid admitted through the device build gives the host-built grid's
    results bit for bit, in the FP64 and the batched form."""
    torch = _torch()
    import salgpu as S
    from salgpu import synth
    g = synth.config_grid("cfg0")
    h = torch.tensor(synth.config_ssh("cfg0", g, nfields=4), device="cuda")
    out = []
    for dev in (None, 0):
        t = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 100, device=dev)
        L = S.dual_tree_traversal(t, 0.7, 100, device=dev)
        grid = S.Grid(t, g.xs, g.ys, g.zs, g.areas, 8, interaction_list=L, max_fields=64)
        ref = grid.solve(h[0], form=S.FORM_REF)
        mix = grid.solve(h, form=S.FORM_MIXED)
        torch.cuda.synchronize()
        out.append([a.cpu().numpy() for a in (*ref, *mix)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_device_build_edge_cases():
    _torch()
    from salgpu import synth
    pts = synth.fibonacci_points(5000)
    x, y, z = (np.ascontiguousarray(pts[:, i]) for i in range(3))
    # fewer points than the threshold: six root leaves
    _check_grid(x[:50], y[:50], z[:50], 200, label="below threshold")
    # one face only (x dominant and positive)
    on = (np.abs(x) >= np.abs(y)) & (np.abs(x) >= np.abs(z)) & (x > 0)
    _check_grid(x[on], y[on], z[on], 20, label="one face")
    # clusters of identical points refine to the level cap (tree_module.f90:80
    # has no cap; both builds stop at level 40)
    rep = np.repeat(np.arange(3), 40)
    cx, cy, cz = x[rep], y[rep], z[rep]
    xx, yy, zz = (np.ascontiguousarray(np.concatenate([a, b[:500]])) for a, b in ((cx, x), (cy, y), (cz, z)))
    hl = _check_grid(xx, yy, zz, 30, label="identical points")
    assert len(hl) > 0
    import salgpu as S
    e = S.tree_traverse(xx, yy, zz, len(xx), 30, device=0).export()
    assert int(np.max(e["level"])) == 40


def test_device_build_no_points():
    _torch()
    import salgpu as S
    z = np.zeros(0)
    ht = S.tree_traverse(z, z, z, 0, 200)
    dt = S.tree_traverse(z, z, z, 0, 200, device=0)
    _compare_trees(ht, dt)
    assert len(S.dual_tree_traversal(dt, 0.7, 200, device=0)) == 0
