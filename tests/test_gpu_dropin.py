"""GPU tests of the reference-signature entry points (sal_fast_sum,
sal_mom6_proxy_source_compute, sal_mom6_pc_compute, sal_mom6_pp_compute)
driven with reference-shaped arguments: the cube_panel array flattened from
the oracle's tree, the oracle's interaction lists and points_panels, and the
point arrays, in the call order of code.f90:92-100 and mom6_code.f90:272-312.

Checks: parity with the oracle (rel-L2 <= 1e-12), intent(inout) accumulation,
the MPI rank split, both ways of passing the panels (with and without
points_inside), and that a change of coordinates, areas, list or degree never
reuses a grid built for the old contents.
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


def _panels(ot):
    return {k: getattr(ot, k) for k in ("level", "is_leaf", "id", "parent", "child", "face", "bounds", "pt_off",
                                         "pt_idx")}


@pytest.mark.parametrize("with_points", [True, False])
def test_fast_sum_reference_shaped_calls(with_points):
    _torch()
    import salgpu as S
    from oracle import oracle as O
    S.dropin_release()
    g, hh = grid_and_ssh("small_3000")
    h = hh[0]
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 20)
    L = O.dual_tree_traversal(ot, 0.7, 20)
    panels = _panels(ot)
    ox, oy = O.fast_sum(ot, L, g.xs, g.ys, g.zs, g.areas, h, 8)
    # code.f90:92-96: outputs zeroed by the caller, fast_sum adds into them
    lon, lat = np.zeros(g.n), np.zeros(g.n)
    S.fast_sum(lon, lat, L, panels, g.xs, g.ys, g.zs, g.areas, h, g.n, 8, 0, 1, with_points_inside=with_points)
    assert rel_l2(lon, lat, ox, oy) <= TOL_PARITY
    # a second call on the cached grid adds again (intent(inout))
    S.fast_sum(lon, lat, L, panels, g.xs, g.ys, g.zs, g.areas, h, g.n, 8, 0, 1, with_points_inside=with_points)
    assert rel_l2(lon, lat, 2 * ox, 2 * oy) <= TOL_PARITY
    # three ranks' shares sum to the whole (Sum_Array, code.f90:99-100)
    lon, lat = np.zeros(g.n), np.zeros(g.n)
    for r in range(3):
        S.fast_sum(lon, lat, L, panels, g.xs, g.ys, g.zs, g.areas, h, g.n, 8, r, 3, with_points_inside=with_points)
    assert rel_l2(lon, lat, ox, oy) <= TOL_PARITY
    # same sizes, new contents: areas, degree and the list each force a new grid
    a2 = g.areas * 1.5
    lon, lat = np.zeros(g.n), np.zeros(g.n)
    S.fast_sum(lon, lat, L, panels, g.xs, g.ys, g.zs, a2, h, g.n, 8, 0, 1, with_points_inside=with_points)
    assert rel_l2(lon, lat, 1.5 * ox, 1.5 * oy) <= TOL_PARITY
    o6 = O.fast_sum(ot, L, g.xs, g.ys, g.zs, g.areas, h, 6)
    lon, lat = np.zeros(g.n), np.zeros(g.n)
    S.fast_sum(lon, lat, L, panels, g.xs, g.ys, g.zs, g.areas, h, g.n, 6, 0, 1, with_points_inside=with_points)
    assert rel_l2(lon, lat, *o6) <= TOL_PARITY
    L2 = L[::-1].copy()
    lon, lat = np.zeros(g.n), np.zeros(g.n)
    S.fast_sum(lon, lat, L2, panels, g.xs, g.ys, g.zs, g.areas, h, g.n, 8, 0, 1, with_points_inside=with_points)
    assert rel_l2(lon, lat, ox, oy) <= TOL_PARITY
    S.dropin_release()


def test_fast_sum_new_coordinates_of_the_same_size_get_a_new_grid():
    _torch()
    import salgpu as S
    from oracle import oracle as O
    S.dropin_release()
    g, hh = grid_and_ssh("small_3000")
    h = hh[0]
    # the same grid turned about the z axis: same sizes, other coordinates
    c, s = np.cos(0.3), np.sin(0.3)
    xs2, ys2 = c * g.xs - s * g.ys, s * g.xs + c * g.ys
    for xs, ys in ((g.xs, g.ys), (xs2, ys2)):
        ot = O.tree_traverse(xs, ys, g.zs, 20)
        L = O.dual_tree_traversal(ot, 0.7, 20)
        ox, oy = O.fast_sum(ot, L, xs, ys, g.zs, g.areas, h, 8)
        lon, lat = np.zeros(g.n), np.zeros(g.n)
        S.fast_sum(lon, lat, L, _panels(ot), xs, ys, g.zs, g.areas, h, g.n, 8)
        assert rel_l2(lon, lat, ox, oy) <= TOL_PARITY
    S.dropin_release()


@pytest.mark.parametrize("with_points", [True, False])
def test_mom6_sequence_reference_shaped(with_points):
    _torch()
    import salgpu as S
    from oracle import oracle as O
    S.dropin_release()
    g, hh = grid_and_ssh("small_3000")
    h = hh[0]
    thresh, d = 20, 8
    ot = O.tree_traverse(g.xs, g.ys, g.zs, thresh)
    ppan = O.assign_points_to_panels(ot, g.xs, g.ys, g.zs)
    pc, pp = O.single_tree_traversal(ot, 0.7, thresh, g.xs, g.ys, g.zs)
    panels = _panels(ot)
    P = (d + 1) ** 2
    for mode, transposed in ((S.MODE_STT_REF_COMPAT, True), (S.MODE_STT_CORRECT, False)):
        S.dropin_config(S.FORM_REF, mode)
        w_ref = O.proxy_source_compute(ot, ppan, g.xs, g.ys, g.zs, h, g.areas, d, transposed)
        ox, oy = O.pc_compute(ot, pc, g.xs, g.ys, g.zs, d, w_ref)
        O.pp_compute(ot, pp, g.xs, g.ys, g.zs, g.areas, h, out=(ox, oy))
        # mom6_code.f90:272-312
        w = np.zeros(P * ot.npanels)
        S.proxy_source_compute(w, panels, ppan, g.xs, g.ys, g.zs, h, g.areas, d, g.n, with_points_inside=with_points)
        assert np.linalg.norm(w - w_ref) <= TOL_PARITY * np.linalg.norm(w_ref)
        sx, sy = np.zeros(g.n), np.zeros(g.n)
        S.pc_compute(sx, sy, pc, panels, g.xs, g.ys, g.zs, d, w, with_points_inside=with_points)
        S.pp_compute(sx, sy, pp, panels, g.xs, g.ys, g.zs, g.areas, h, own_points=g.n,
                     with_points_inside=with_points)
        assert rel_l2(sx, sy, ox, oy) <= TOL_PARITY
    S.dropin_config(S.FORM_REF, S.MODE_STT_REF_COMPAT)
    S.dropin_release()


def test_mom6_entry_points_reject_what_they_cannot_reproduce():
    _torch()
    import salgpu as S
    from oracle import oracle as O
    g, hh = grid_and_ssh("small_3000")
    h = hh[0]
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 20)
    ppan = O.assign_points_to_panels(ot, g.xs, g.ys, g.zs)
    pc, pp = O.single_tree_traversal(ot, 0.7, 20, g.xs, g.ys, g.zs)
    panels = _panels(ot)
    w = np.zeros(81 * ot.npanels)
    bad = ppan.copy()
    bad[0, 0] = ppan[0, 0] % 6 + 1          # another face's root panel
    with pytest.raises(S.SalError) as e:
        S.proxy_source_compute(w, panels, bad, g.xs, g.ys, g.zs, h, g.areas, 8, g.n)
    assert e.value.code == S.SAL_EINVAL and "points_panels" in str(e.value)
    sx, sy = np.zeros(g.n), np.zeros(g.n)
    with pytest.raises(S.SalError) as e:
        S.pp_compute(sx, sy, pp, panels, g.xs, g.ys, g.zs, g.areas, h, e_xs=np.zeros(3), e_ys=np.zeros(3),
                     e_zs=np.zeros(3), e_areas=np.zeros(3), e_sshs=np.zeros(3))
    assert e.value.code == S.SAL_EINVAL and "halo" in str(e.value)
    assert not sx.any() and not sy.any()
    S.dropin_release()
