"""CPU tests of the oracle (oracle/sal_oracle.c) against mathematical known answers.

The reference ships no tests or golden vectors and cannot be compiled here,
so the oracle is pinned by properties that any correct restatement must have:
geometry round trips, barycentric interpolation exactness, kernel identities,
completeness of the interaction lists, and agreement with an FP64 direct sum.
"""
import math

import numpy as np
import pytest

from conftest import grid_and_ssh, rel_l2
from oracle import oracle as O


def _numpy_gfunc(t, s):
    """Independent numpy statement of sal_grad_gfunc (fast_sum_module.f90:9-31),
    same operation order (numpy float64 operations are IEEE, no FMA)."""
    tx, ty, tz = t
    sx, sy, sz = s
    if not (abs(tz - 1.0) > 1e-15 and abs(tz + 1.0) > 1e-15):
        return 0.0, 0.0
    g = max(min(tx * sx + ty * sy + tz * sz, 1.0), -1.0)
    mp = 2.0 - 2.0 * g
    sqp = math.sqrt(mp)
    p1 = (1.0 - 6.21196) / (sqp * mp + 1e-16)
    p2 = (2.7 + 6.0) * (2.0 * g + sqp) / (2.0 * (g * g - 1.0) + 1e-16)
    val = (p1 + p2) * -2.343256857908601e-9
    x32 = tz * tz
    mp2 = math.sqrt(1.0 - x32)
    return (tx * sy - ty * sx) / mp2 * val, (sz * (1.0 - x32) - tz * (tx * sx + ty * sy)) / mp2 * val


def _unit(rng, n):
    p = rng.standard_normal((n, 3))
    return p / np.linalg.norm(p, axis=1, keepdims=True)


# ------------------------------------------------------------------ geometry
def test_face_from_xyz_ties_and_signs():
    assert O.face_from_xyz(1, 0, 0) == 1 and O.face_from_xyz(-1, 0, 0) == 3
    assert O.face_from_xyz(0, 1, 0) == 2 and O.face_from_xyz(0, -1, 0) == 4
    assert O.face_from_xyz(0, 0, 1) == 5 and O.face_from_xyz(0, 0, -1) == 6
    assert O.face_from_xyz(1, 1, 1) == 1          # ties go to x (cube_sphere_module.f90:13)
    assert O.face_from_xyz(0.2, 1, 1) == 2        # then to y


def test_xyz_xieta_round_trip():
    rng = np.random.default_rng(0)
    for p in _unit(rng, 2000):
        f = O.face_from_xyz(*p)
        xi, eta = O.xieta_from_xyz(*p, f)
        assert -math.pi / 4 - 1e-15 <= xi <= math.pi / 4 + 1e-15
        q = O.xyz_from_xieta(xi, eta, f)
        assert np.max(np.abs(np.array(q) - p)) < 4e-16


# ------------------------------------------------------------------ BLI
def test_chebyshev_nodes_descend_over_the_interval():
    nodes = O.bli_interp_points_shift(-0.3, 0.5, 8)
    assert nodes[0] == pytest.approx(0.5, abs=1e-16) and nodes[-1] == pytest.approx(-0.3, abs=1e-16)
    assert np.all(np.diff(nodes) < 0)


@pytest.mark.parametrize("degree", [2, 5, 8, 10])
def test_bli_reproduces_tensor_polynomials(degree):
    rng = np.random.default_rng(degree)
    a, b, c, e = -0.4, 0.1, 0.2, 0.7
    xn, en = O.bli_interp_points_shift(a, b, degree), O.bli_interp_points_shift(c, e, degree)
    coef = rng.standard_normal((degree + 1, degree + 1))
    poly = lambda x, y: sum(coef[i, j] * x ** i * y ** j for i in range(degree + 1) for j in range(degree + 1))
    vals = np.array([[poly(x, y) for y in en] for x in xn])
    for _ in range(20):
        x, y = rng.uniform(a, b), rng.uniform(c, e)
        B = O.interp_vals_bli(x, y, a, b, c, e, degree)
        assert np.sum(B) == pytest.approx(1.0, abs=1e-13)
        assert np.sum(B * vals) == pytest.approx(poly(x, y), abs=1e-11 * max(1.0, np.abs(vals).max()))


def test_bli_exact_node_branch():
    xn = O.bli_interp_points_shift(-0.4, 0.1, 8)
    en = O.bli_interp_points_shift(0.2, 0.7, 8)
    B = O.interp_vals_bli(xn[3], en[5], -0.4, 0.1, 0.2, 0.7, 8)
    expect = np.zeros((9, 9))
    expect[3, 5] = 1.0
    assert np.array_equal(B, expect)


# ------------------------------------------------------------------ kernel
def test_gfunc_matches_independent_numpy_statement_bitwise():
    rng = np.random.default_rng(1)
    P = _unit(rng, 300)
    pairs = [(P[i], P[j]) for i in range(0, 300, 3) for j in range(0, 300, 7)]
    pairs += [(p, p) for p in P[:50]]                                       # self pairs
    pairs += [(p, p + 1e-9 * rng.standard_normal(3)) for p in P[:50]]       # near duplicates
    pairs += [(p, -p) for p in P[:20]]                                      # antipodes
    for t, s in pairs:
        assert O.sal_grad_gfunc(*t, *s) == _numpy_gfunc(t, s)


def test_gfunc_self_pair_and_pole_guard():
    rng = np.random.default_rng(2)
    for p in _unit(rng, 100):
        gx, _ = O.sal_grad_gfunc(*p, *p)
        assert gx == 0.0                      # tx*ty - ty*tx
    assert O.sal_grad_gfunc(0.0, 0.0, 1.0, 0.6, 0.0, 0.8) == (0.0, 0.0)
    assert O.sal_grad_gfunc(0.0, 0.0, -1.0, 0.6, 0.0, 0.8) == (0.0, 0.0)


def test_gfunc_antipode_is_zero_not_its_limit():
    """At g = -1 the reference's p2 evaluates 0 / 1e-16 = 0 while its limit is
    -3*8.7/4; the oracle reproduces the reference (a documented defect that
    the CC interactions between opposite cube faces hit)."""
    t = np.array([1.0, 0.0, 0.0])
    gx, gy = O.sal_grad_gfunc(*t, *(-t))
    assert gx == 0.0 and gy == 0.0


# ------------------------------------------------------------------ tree and lists
@pytest.fixture(scope="module")
def small():
    g, h = grid_and_ssh("small_3000")
    t = O.tree_traverse(g.xs, g.ys, g.zs, 20)
    return g, h[0], t


def test_tree_invariants(small):
    g, _, t = small
    cnt = np.diff(t.pt_off)
    assert np.all(np.diff(t.level) >= 0)                          # BFS order
    assert cnt[:6].sum() == g.n                                   # root conservation (tree_module.f90:104-113)
    for k in range(t.npanels):
        if not t.is_leaf[k]:
            ch = t.child[k]
            assert list(ch) == list(range(ch[0], ch[0] + 4))       # children contiguous
            assert cnt[ch - 1].sum() == cnt[k]                    # refinement conservation (:209-216)
            assert sorted(np.concatenate([t.points_inside(c) for c in ch])) == sorted(t.points_inside(k + 1))
        else:
            assert cnt[k] < 20
    leaves = np.concatenate([t.points_inside(k + 1) for k in range(t.npanels) if t.is_leaf[k]])
    assert np.array_equal(np.sort(leaves), np.arange(1, g.n + 1))


def test_dtt_covers_every_pair_exactly_once(small):
    g, _, t = small
    L = O.dual_tree_traversal(t, 0.7, 20)
    assert set(np.unique(L[:, 2])) == {0, 1, 2, 3}
    cover = np.zeros((g.n, g.n), np.int8)
    for it, is_, _ in L:
        T = t.points_inside(it) - 1
        S = t.points_inside(is_) - 1
        cover[np.ix_(T, S)] += 1
    assert cover.min() == 1 and cover.max() == 1


def test_stt_covers_every_pair_exactly_once(small):
    g, _, t = small
    pc, pp = O.single_tree_traversal(t, 0.7, 20, g.xs, g.ys, g.zs)
    cover = np.zeros((g.n, g.n), np.int8)
    for ip, is_ in np.concatenate([pc, pp]):
        cover[ip - 1, t.points_inside(is_) - 1] += 1
    assert cover.min() == 1 and cover.max() == 1


def test_fast_sum_all_pp_equals_direct_sum(small):
    g, h, t = small
    L = O.dual_tree_traversal(t, 0.7, 20)
    L[:, 2] = 0
    ox, oy = O.fast_sum(t, L, g.xs, g.ys, g.zs, g.areas, h, 8, nranks=4)
    dx, dy = O.direct_sum(g.xs, g.ys, g.zs, g.areas, h, np.arange(g.n, dtype=np.int32))
    assert rel_l2(ox, oy, dx, dy) < 1e-13


def test_direct_sum_matches_python_loop():
    g, h = grid_and_ssh("small_3000")
    h = h[0]
    tg = np.array([0, 17, 999, 2999], np.int32)
    dx, dy = O.direct_sum(g.xs, g.ys, g.zs, g.areas, h, tg)
    for k, ti in enumerate(tg):
        ax = ay = 0.0
        t = (g.xs[ti], g.ys[ti], g.zs[ti])
        for s in range(0, g.n):
            gx, gy = _numpy_gfunc(t, (g.xs[s], g.ys[s], g.zs[s]))
            ax = ax + gx * g.areas[s] * h[s]
            ay = ay + gy * g.areas[s] * h[s]
        assert dx[k] == ax and dy[k] == ay


def test_rank_split_sums_to_serial(small):
    g, h, t = small
    L = O.dual_tree_traversal(t, 0.7, 20)
    a = O.fast_sum(t, L, g.xs, g.ys, g.zs, g.areas, h, 8, nranks=1)
    b = O.fast_sum(t, L, g.xs, g.ys, g.zs, g.areas, h, 8, nranks=5)
    assert rel_l2(b[0], b[1], a[0], a[1]) < 1e-14


def test_mom6_transposed_weights_are_inaccurate_and_correct_ones_are_not(small):
    g, h, t = small
    tg = np.arange(g.n, dtype=np.int32)
    dx, dy = O.direct_sum(g.xs, g.ys, g.zs, g.areas, h, tg)
    ref = O.mom6_solve(g.xs, g.ys, g.zs, g.areas, h, 0.7, 20, 8, transposed=True)
    cor = O.mom6_solve(g.xs, g.ys, g.zs, g.areas, h, 0.7, 20, 8, transposed=False)
    assert rel_l2(*cor, dx, dy) < 1e-4
    assert rel_l2(*ref, dx, dy) > 100 * rel_l2(*cor, dx, dy)


def test_cartesian_dtt_converges_spectrally(small):
    g, h, t = small
    L = O.dual_tree_traversal(t, 0.7, 20)
    tg = np.arange(g.n, dtype=np.int32)
    dx, dy = O.direct_sum(g.xs, g.ys, g.zs, g.areas, h, tg)
    e = [rel_l2(*O.fast_sum_cart(t, L, g.xs, g.ys, g.zs, g.areas, h, d, 4), dx, dy) for d in (4, 6, 8)]
    assert e[0] > e[1] > e[2] and e[2] < 1e-6
    e_ref = rel_l2(*O.fast_sum(t, L, g.xs, g.ys, g.zs, g.areas, h, 8, 4), dx, dy)
    assert e_ref > 10 * e[2]


def test_mom6_thread_split_is_bitwise_serial(small):
    """Threads that own disjoint panels (weights) or targets (pc/pp sums) keep
    every sum in the reference's order, so any thread count gives the serial
    result bit for bit."""
    g, h, t = small
    ppan = O.assign_points_to_panels(t, g.xs, g.ys, g.zs)
    pc, pp = O.single_tree_traversal(t, 0.7, 20, g.xs, g.ys, g.zs)
    w1 = O.proxy_source_compute(t, ppan, g.xs, g.ys, g.zs, h, g.areas, 8, True, nthreads=1)
    w5 = O.proxy_source_compute(t, ppan, g.xs, g.ys, g.zs, h, g.areas, 8, True, nthreads=5)
    assert np.array_equal(w1, w5)
    a = O.pc_compute(t, pc, g.xs, g.ys, g.zs, 8, w1, nthreads=1)
    b = O.pc_compute(t, pc, g.xs, g.ys, g.zs, 8, w1, nthreads=5)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    a = O.pp_compute(t, pp, g.xs, g.ys, g.zs, g.areas, h, nthreads=1)
    b = O.pp_compute(t, pp, g.xs, g.ys, g.zs, g.areas, h, nthreads=5)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
