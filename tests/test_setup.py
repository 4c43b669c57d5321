"""CPU tests of the product's host side: the C ABI loads and exports every
declared symbol, and its tree / list builders equal the oracle's element for
element (tree_module.f90 decisions must not change)."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, grid_and_ssh
from oracle import oracle as O


def test_library_exports_every_header_symbol():
    import ctypes
    import salgpu as S
    hdr = open(os.path.join(ROOT, "include", "salgpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    declared = set(re.findall(r"\b(sal_[a-z0-9_]+)\s*\(", hdr))
    assert declared, "no declarations parsed"
    assert declared == set(S.EXPORTS), declared ^ set(S.EXPORTS)
    L = S.lib()
    for name in declared:
        assert isinstance(getattr(L, name), ctypes._CFuncPtr), name


def test_device_entry_points_fail_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import salgpu as S
    g, _ = grid_and_ssh("small_3000")
    t = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 20)
    L = S.dual_tree_traversal(t, 0.7, 20)
    with pytest.raises(S.SalError) as e:
        S.Grid(t, g.xs, g.ys, g.zs, g.areas, 8, S.MODE_DTT, L)
    assert e.value.code == S.SAL_ENODEV


@pytest.mark.parametrize("name,thresh", [("small_3000", 20), ("small_3000", 10), ("cfg0", 100), ("small_2000", 300)])
def test_tree_and_lists_equal_oracle(name, thresh):
    import salgpu as S
    g, _ = grid_and_ssh(name)
    ot = O.tree_traverse(g.xs, g.ys, g.zs, thresh)
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, thresh)
    e = pt.export()
    assert ot.npanels == pt.npanels
    for k in ("level", "is_leaf", "id", "parent", "child", "face"):
        assert np.array_equal(getattr(ot, k), e[k]), k
    assert np.array_equal(ot.bounds, e["bounds"])
    assert np.array_equal(ot.pt_off, e["pt_off"]) and np.array_equal(ot.pt_idx, e["pt_idx"])
    assert np.array_equal(O.dual_tree_traversal(ot, 0.7, thresh), S.dual_tree_traversal(pt, 0.7, thresh))
    a, b = O.single_tree_traversal(ot, 0.7, thresh, g.xs, g.ys, g.zs)
    c, d = S.single_tree_traversal(pt, 0.7, thresh, g.xs, g.ys, g.zs)
    assert np.array_equal(a, c) and np.array_equal(b, d)
    assert np.array_equal(O.assign_points_to_panels(ot, g.xs, g.ys, g.zs), S.assign_points_to_panels(pt, g.xs, g.ys, g.zs))


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.9])
def test_dtt_equal_oracle_across_theta(theta):
    import salgpu as S
    g, _ = grid_and_ssh("small_3000")
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 20)
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 20)
    assert np.array_equal(O.dual_tree_traversal(ot, theta, 20), S.dual_tree_traversal(pt, theta, 20))


def test_tree_import_round_trip_and_validation():
    import salgpu as S
    g, _ = grid_and_ssh("small_3000")
    pt = S.tree_traverse(g.xs, g.ys, g.zs, g.n, 20)
    e = pt.export()
    t2 = S.tree_import(e, g.xs, g.ys, g.zs)
    e2 = t2.export()
    for k in e:
        assert np.array_equal(e[k], e2[k]), k
    # a leaf that loses a point is rejected
    bad = {k: np.array(v, copy=True) for k, v in e.items()}
    leaf = int(np.nonzero((bad["is_leaf"] == 1) & (np.diff(bad["pt_off"]) > 1))[0][0])
    j = bad["pt_off"][leaf]
    bad["pt_idx"][j] = bad["pt_idx"][j + 1]
    with pytest.raises(S.SalError) as err:
        S.tree_import(bad, g.xs, g.ys, g.zs)
    assert err.value.code == S.SAL_EINVAL
    # an out-of-range child is rejected
    bad = {k: np.array(v, copy=True) for k, v in e.items()}
    k = int(np.nonzero(bad["is_leaf"] == 0)[0][0])
    bad["child"][k, 2] = 10 ** 6
    with pytest.raises(S.SalError):
        S.tree_import(bad, g.xs, g.ys, g.zs)


def test_oracle_tree_imports_into_product():
    """A tree built by another implementation (here the oracle, standing in for
    the Fortran caller's own tree_traverse) is accepted as is."""
    import salgpu as S
    g, _ = grid_and_ssh("small_3000")
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 20)
    panels = dict(level=ot.level, is_leaf=ot.is_leaf, id=ot.id, parent=ot.parent, child=ot.child, face=ot.face,
                  bounds=ot.bounds, pt_off=ot.pt_off, pt_idx=ot.pt_idx)
    t = S.tree_import(panels, g.xs, g.ys, g.zs)
    assert np.array_equal(S.dual_tree_traversal(t, 0.7, 20), O.dual_tree_traversal(ot, 0.7, 20))


def test_bad_arguments_are_rejected():
    import salgpu as S
    g, _ = grid_and_ssh("small_3000")
    with pytest.raises(S.SalError):
        S.tree_traverse(g.xs, g.ys, g.zs, g.n, 1)          # cluster_thresh < 2 would refine forever
    with pytest.raises(ValueError):
        S.tree_traverse(g.xs, g.ys, g.zs, g.n + 1, 20)


def test_empty_and_tiny_inputs():
    import salgpu as S
    t = S.tree_traverse(np.zeros(0), np.zeros(0), np.zeros(0), 0, 10)
    assert t.npanels == 6 and len(S.dual_tree_traversal(t, 0.7, 10)) == 0
    xs, ys, zs = np.array([1.0]), np.array([0.0]), np.array([0.0])
    t = S.tree_traverse(xs, ys, zs, 1, 10)
    L = S.dual_tree_traversal(t, 0.7, 10)
    assert L.tolist() == [[1, 1, 0]]


def test_identical_points_stop_refining():
    """Points that coincide would refine forever in the reference
    (tree_module.f90:127-130); refinement stops at level 40."""
    import salgpu as S
    xs = np.full(30, 0.6)
    ys = np.full(30, 0.0)
    zs = np.full(30, 0.8)
    t = S.tree_traverse(xs, ys, zs, 30, 10)
    assert t.info()[2] == 40


def test_reference_signature_entry_points_check_their_arguments_on_the_host():
    """The panels-without-points_inside path rebuilds the tree from the
    coordinates and compares it with the caller's panels before any device
    work: matching panels get as far as the device (SAL_ENODEV here, with no
    GPU), panels of other coordinates are refused with SAL_ETREE."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import salgpu as S
    g, hh = grid_and_ssh("small_3000")
    ot = O.tree_traverse(g.xs, g.ys, g.zs, 20)
    L = O.dual_tree_traversal(ot, 0.7, 20)
    panels = {k: getattr(ot, k) for k in ("level", "is_leaf", "id", "parent", "child", "face", "bounds", "pt_off",
                                           "pt_idx")}
    lon, lat = np.zeros(g.n), np.zeros(g.n)
    args = (lon, lat, L, panels, g.xs, g.ys, g.zs, g.areas, hh[0], g.n, 8)
    with pytest.raises(S.SalError) as e:
        S.fast_sum(*args, 3, 3)
    assert e.value.code == S.SAL_EINVAL
    for wp in (True, False):
        with pytest.raises(S.SalError) as e:
            S.fast_sum(*args, 0, 1, with_points_inside=wp)
        assert e.value.code == S.SAL_ENODEV
    xs2 = g.xs.copy()
    k = int(np.argmax(np.abs(g.xs)))
    xs2[k], ys2 = g.ys[k], g.ys.copy()
    ys2[k] = g.xs[k]                               # one point moved to another place on the sphere
    with pytest.raises(S.SalError) as e:
        S.fast_sum(lon, lat, L, panels, xs2, ys2, g.zs, g.areas, hh[0], g.n, 8, with_points_inside=False)
    assert e.value.code == S.SAL_ETREE
    assert not lon.any() and not lat.any()


def test_grid_ingestion_reads_list_directed_files_and_raw_float64(tmp_path):
    """sal_read_values parses one-value-per-line files as the reference's
    drivers read them (code.f90:36-56): Fortran list-directed forms with E, D
    or a bare-sign exponent, blank lines, trailing blanks; every value comes
    back bit for bit.  The raw .f64 form round-trips; short files and bad
    lines are refused."""
    import salgpu as S
    rng = np.random.default_rng(5)
    v = np.concatenate([rng.standard_normal(5000) * 10.0 ** rng.integers(-300, 300, 5000), [0.0, -0.0, 1.0, -2.5]])
    # %.17g round-trips every double; add Fortran-style renderings
    lines = [f"  {x:.17g}   " for x in v]
    lines[1] = lines[1].replace("e", "D")
    lines[2] = " " + repr(float(v[2])).upper() + "\r"
    lines.insert(7, "")
    p = tmp_path / "x.csv"
    p.write_text("\n".join(lines) + "\n")
    out = S.read_values(str(p), len(v))
    assert np.array_equal(out.view(np.uint64), v.view(np.uint64))
    assert np.array_equal(S.read_values(str(p), 10), v[:10])
    q = tmp_path / "y.csv"
    q.write_text("  0.125-002\n 1.5D+3\n -2.0E-1\n")
    assert np.array_equal(S.read_values(str(q), 3), [0.125e-2, 1.5e3, -0.2])
    b = tmp_path / "x.f64"
    S.write_values(str(b), v)
    assert np.array_equal(S.read_values(str(b), len(v)).view(np.uint64), v.view(np.uint64))
    with pytest.raises(S.SalError) as e:
        S.read_values(str(p), len(v) + 1)
    assert e.value.code == S.SAL_EINVAL and "fewer" in str(e.value)
    r = tmp_path / "bad.csv"
    r.write_text("1.0\nabc\n3.0\n")
    with pytest.raises(S.SalError) as e:
        S.read_values(str(r), 3)
    assert "value 2" in str(e.value)
    with pytest.raises(S.SalError):
        S.read_values(str(tmp_path / "missing.csv"), 1)
