"""ctypes front end of the CPU oracle (oracle/sal_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the product package.  The oracle is a
line-faithful C restatement of cygnari/sal-fort (fast_sum_module.f90,
mom6_fast_sum_module.f90, tree_module.f90, bli_module.f90,
cube_sphere_module.f90).  Parity unpinned: the reference ships no golden
vectors and cannot be compiled here; the oracle is pinned by mathematical
known-answer tests and by the FP64 direct sum.

All panel ids, point ids and list entries returned here are 1-based, as in the
Fortran.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsaloracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile (no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    d, i, vp = C.c_double, C.c_int, C.c_void_p
    L.or_face_from_xyz.argtypes = [d, d, d]
    L.or_face_from_xyz.restype = i
    L.or_xieta_from_xyz.argtypes = [d, d, d, C.POINTER(d), C.POINTER(d), i]
    L.or_xyz_from_xieta.argtypes = [C.POINTER(d), C.POINTER(d), C.POINTER(d), d, d, i]
    L.or_bli_interp_points_shift.argtypes = [_dp, d, d, i]
    L.or_interp_vals_bli.argtypes = [_dp, d, d, d, d, d, d, i]
    L.or_sal_grad_gfunc.argtypes = [d, d, d, d, d, d, C.POINTER(d), C.POINTER(d)]
    L.or_tree_traverse.argtypes = [i, _dp, _dp, _dp, i]
    L.or_tree_traverse.restype = vp
    L.or_tree_free.argtypes = [vp]
    L.or_tree_npanels.argtypes = [vp]
    L.or_tree_npanels.restype = i
    L.or_tree_total_points.argtypes = [vp]
    L.or_tree_total_points.restype = C.c_longlong
    L.or_tree_export.argtypes = [vp, _ip, _dp, _lp, _ip]
    L.or_dual_tree_traversal.argtypes = [vp, d, i, C.POINTER(C.POINTER(C.c_int))]
    L.or_dual_tree_traversal.restype = i
    L.or_single_tree_traversal.argtypes = [vp, d, i, _dp, _dp, _dp, i,
                                           C.POINTER(C.POINTER(C.c_int)), C.POINTER(i),
                                           C.POINTER(C.POINTER(C.c_int)), C.POINTER(i)]
    L.or_assign_points_to_panels.argtypes = [vp, _dp, _dp, _dp, i, _ip, i]
    L.or_assign_points_to_panels.restype = i
    L.or_free.argtypes = [vp]
    L.or_fast_sum.argtypes = [_dp, _dp, _ip, i, vp, _dp, _dp, _dp, _dp, _dp, i, i, i]
    L.or_fast_sum_cart.argtypes = [_dp, _dp, _ip, i, vp, _dp, _dp, _dp, _dp, _dp, i, i, i]
    L.or_proxy_source_compute.argtypes = [_dp, vp, _ip, i, _dp, _dp, _dp, _dp, _dp, i, i, i, i]
    L.or_pc_compute.argtypes = [_dp, _dp, _ip, i, vp, _dp, _dp, _dp, i, _dp, i, i]
    L.or_pp_compute.argtypes = [_dp, _dp, _ip, i, vp, _dp, _dp, _dp, _dp, _dp, i, i]
    L.or_direct_sum.argtypes = [_dp, _dp, _dp, _dp, _dp, i, _ip, i, _dp, _dp, i]
    L.or_dtt_work.argtypes = [vp, _ip, i, i, _dp, C.POINTER(d)]
    _lib = L
    return L


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------- geometry / BLI
def face_from_xyz(x, y, z) -> int:
    return lib().or_face_from_xyz(x, y, z)


def xieta_from_xyz(x, y, z, face):
    xi, eta = C.c_double(), C.c_double()
    lib().or_xieta_from_xyz(x, y, z, C.byref(xi), C.byref(eta), face)
    return xi.value, eta.value


def xyz_from_xieta(xi, eta, face):
    x, y, z = C.c_double(), C.c_double(), C.c_double()
    lib().or_xyz_from_xieta(C.byref(x), C.byref(y), C.byref(z), xi, eta, face)
    return x.value, y.value, z.value


def bli_interp_points_shift(min_x, max_x, degree):
    out = np.zeros(degree + 1)
    lib().or_bli_interp_points_shift(out, min_x, max_x, degree)
    return out


def interp_vals_bli(xi, eta, min_xi, max_xi, min_eta, max_eta, degree):
    """Returns vals with vals[i, j] = xi_basis[i] * eta_basis[j] (Fortran vals(i+1, j+1))."""
    n = degree + 1
    out = np.zeros(n * n)
    lib().or_interp_vals_bli(out, xi, eta, min_xi, max_xi, min_eta, max_eta, degree)
    return out.reshape(n, n, order="F")


def sal_grad_gfunc(tx, ty, tz, sx, sy, sz):
    a, b = C.c_double(), C.c_double()
    lib().or_sal_grad_gfunc(tx, ty, tz, sx, sy, sz, C.byref(a), C.byref(b))
    return a.value, b.value


# ---------------------------------------------------------------- tree
@dataclass
class Tree:
    handle: int
    n_points: int
    level: np.ndarray
    is_leaf: np.ndarray
    id: np.ndarray
    parent: np.ndarray
    child: np.ndarray      # (np, 4)
    face: np.ndarray
    bounds: np.ndarray     # (np, 7): min_xi, mid_xi, max_xi, min_eta, mid_eta, max_eta, radius
    pt_off: np.ndarray     # (np+1,)
    pt_idx: np.ndarray     # 1-based point ids

    @property
    def npanels(self) -> int:
        return len(self.level)

    def points_inside(self, k: int) -> np.ndarray:
        """points_inside of 1-based panel id k (1-based point ids)."""
        return self.pt_idx[self.pt_off[k - 1]:self.pt_off[k]]

    def __del__(self):
        if self.handle and _lib is not None:
            _lib.or_tree_free(self.handle)
            self.handle = 0


def tree_traverse(xs, ys, zs, cluster_thresh) -> Tree:
    """tree_module.f90:59-246."""
    xs, ys, zs = _f64(xs), _f64(ys), _f64(zs)
    L = lib()
    h = L.or_tree_traverse(len(xs), xs, ys, zs, int(cluster_thresh))
    npn = L.or_tree_npanels(h)
    tot = L.or_tree_total_points(h)
    ints = np.zeros(9 * npn, np.int32)
    dbl = np.zeros(7 * npn, np.float64)
    off = np.zeros(npn + 1, np.int64)
    idx = np.zeros(max(tot, 1), np.int32)
    L.or_tree_export(h, ints, dbl, off, idx)
    ints = ints.reshape(npn, 9)
    return Tree(h, len(xs), ints[:, 0].copy(), ints[:, 1].copy(), ints[:, 2].copy(), ints[:, 3].copy(),
                ints[:, 4:8].copy(), ints[:, 8].copy(), dbl.reshape(npn, 7).copy(), off, idx[:tot])


def dual_tree_traversal(tree: Tree, theta, thresh) -> np.ndarray:
    """tree_module.f90:277-398.  Returns (ninter, 3) int32: target, source, type."""
    L = lib()
    p = C.POINTER(C.c_int)()
    n = L.or_dual_tree_traversal(tree.handle, float(theta), int(thresh), C.byref(p))
    out = np.ctypeslib.as_array(p, shape=(3 * n,)).copy().reshape(n, 3) if n else np.zeros((0, 3), np.int32)
    L.or_free(p)
    return out


def single_tree_traversal(tree: Tree, theta, thresh, xs, ys, zs):
    """tree_module.f90:401-487.  Returns (pc, pp), each (n, 2) int32: target point, source panel."""
    L = lib()
    xs, ys, zs = _f64(xs), _f64(ys), _f64(zs)
    pc, pp = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    npc, npp = C.c_int(), C.c_int()
    L.or_single_tree_traversal(tree.handle, float(theta), int(thresh), xs, ys, zs, len(xs),
                               C.byref(pc), C.byref(npc), C.byref(pp), C.byref(npp))
    a = np.ctypeslib.as_array(pc, shape=(2 * npc.value,)).copy().reshape(-1, 2) if npc.value else np.zeros((0, 2), np.int32)
    b = np.ctypeslib.as_array(pp, shape=(2 * npp.value,)).copy().reshape(-1, 2) if npp.value else np.zeros((0, 2), np.int32)
    L.or_free(pc)
    L.or_free(pp)
    return a, b


def assign_points_to_panels(tree: Tree, xs, ys, zs) -> np.ndarray:
    """tree_module.f90:249-273.  Returns points_panels as (nlev, N) int32, -1 filled."""
    nlev = int(tree.level[-1]) + 1   # mom6_code.f90:188-189
    n = len(xs)
    pp = np.full(nlev * n, -1, np.int32)
    rc = lib().or_assign_points_to_panels(tree.handle, _f64(xs), _f64(ys), _f64(zs), n, pp, nlev)
    if rc != 0:
        raise ValueError(f"point {-rc} lies in no panel")
    return pp.reshape(nlev, n, order="F")


# ---------------------------------------------------------------- evaluators
def fast_sum(tree: Tree, inter: np.ndarray, xs, ys, zs, area, ssh, degree, nranks=1):
    """fast_sum_module.f90:291-332 (outputs start at zero, code.f90:92-93)."""
    n = len(xs)
    ox, oy = np.zeros(n), np.zeros(n)
    lst = _i32(inter.reshape(-1))
    lib().or_fast_sum(ox, oy, lst, len(inter), tree.handle, _f64(xs), _f64(ys), _f64(zs), _f64(area), _f64(ssh),
                      n, int(degree), int(nranks))
    return ox, oy


def fast_sum_cart(tree: Tree, inter: np.ndarray, xs, ys, zs, area, ssh, degree, nthreads=1):
    """fast_sum with CP/CC interpolating the Cartesian vector sum val*(s-x)*w at
    the target proxies and projecting onto the real target's east/north frame."""
    n = len(xs)
    ox, oy = np.zeros(n), np.zeros(n)
    lst = _i32(inter.reshape(-1))
    lib().or_fast_sum_cart(ox, oy, lst, len(inter), tree.handle, _f64(xs), _f64(ys), _f64(zs), _f64(area),
                           _f64(ssh), n, int(degree), int(nthreads))
    return ox, oy


def proxy_source_compute(tree: Tree, points_panels, xs, ys, zs, sshs, areas, degree, transposed=True,
                         nthreads=1):
    """mom6_fast_sum_module.f90:33-74; transposed=True is the reference's store.
    Threads own disjoint panel ranges; every weight sums its points in the
    reference's order for any thread count."""
    nlev = points_panels.shape[0]
    P = (degree + 1) ** 2
    w = np.zeros(P * tree.npanels)
    ppf = _i32(np.asfortranarray(points_panels).reshape(-1, order="F"))
    lib().or_proxy_source_compute(w, tree.handle, ppf, nlev, _f64(xs), _f64(ys), _f64(zs), _f64(sshs),
                                  _f64(areas), int(degree), len(xs), int(bool(transposed)), int(nthreads))
    return w


def pc_compute(tree: Tree, pc, xs, ys, zs, degree, weights, out=None, nthreads=1):
    """mom6_fast_sum_module.f90:153-174.  Threads own disjoint target ranges
    (as the reference's ranks own points); each target sums its entries in list
    order for any thread count."""
    n = len(xs)
    ox, oy = (np.zeros(n), np.zeros(n)) if out is None else out
    lib().or_pc_compute(ox, oy, _i32(pc.reshape(-1)), len(pc), tree.handle, _f64(xs), _f64(ys), _f64(zs),
                        int(degree), _f64(weights), n, int(nthreads))
    return ox, oy


def pp_compute(tree: Tree, pp, xs, ys, zs, areas, sshs, out=None, nthreads=1):
    """mom6_fast_sum_module.f90:177-192 at one rank (threads as in pc_compute)."""
    n = len(xs)
    ox, oy = (np.zeros(n), np.zeros(n)) if out is None else out
    lib().or_pp_compute(ox, oy, _i32(pp.reshape(-1)), len(pp), tree.handle, _f64(xs), _f64(ys), _f64(zs),
                        _f64(areas), _f64(sshs), n, int(nthreads))
    return ox, oy


def mom6_solve(xs, ys, zs, areas, sshs, theta, thresh, degree, transposed=True, nthreads=1):
    """The mom6_code.f90 solve sequence at one rank (:177-312)."""
    tree = tree_traverse(xs, ys, zs, thresh)
    ppan = assign_points_to_panels(tree, xs, ys, zs)
    pc, pp = single_tree_traversal(tree, theta, thresh, xs, ys, zs)
    w = proxy_source_compute(tree, ppan, xs, ys, zs, sshs, areas, degree, transposed, nthreads)
    ox, oy = pc_compute(tree, pc, xs, ys, zs, degree, w, nthreads=nthreads)
    pp_compute(tree, pp, xs, ys, zs, areas, sshs, out=(ox, oy), nthreads=nthreads)
    return ox, oy


def dtt_solve(xs, ys, zs, area, ssh, theta, thresh, degree, nranks=1):
    """The code.f90 solve sequence (:72-100)."""
    tree = tree_traverse(xs, ys, zs, thresh)
    inter = dual_tree_traversal(tree, theta, thresh)
    return fast_sum(tree, inter, xs, ys, zs, area, ssh, degree, nranks)


def direct_sum(xs, ys, zs, area, ssh, targets, nthreads=None):
    """FP64 direct O(N^2) sum at the given 0-based targets."""
    targets = _i32(targets)
    nt = len(targets)
    ox, oy = np.zeros(nt), np.zeros(nt)
    nthreads = nthreads or os.cpu_count() or 1
    lib().or_direct_sum(_f64(xs), _f64(ys), _f64(zs), _f64(area), _f64(ssh), len(xs), targets, nt, ox, oy,
                        int(nthreads))
    return ox, oy


def dtt_work(tree: Tree, inter: np.ndarray, degree):
    """Kernel pairs by interaction type (PP, PC, CP, CC) and proxy MACs of a DTT list."""
    pairs = np.zeros(4)
    macs = C.c_double()
    lib().or_dtt_work(tree.handle, _i32(inter.reshape(-1)), len(inter), int(degree), pairs, C.byref(macs))
    return pairs, macs.value
