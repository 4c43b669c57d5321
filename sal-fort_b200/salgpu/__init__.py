"""Python host layer of the B200 SAL-gradient treecode.

Mirrors cygnari/sal-fort's entry points over the C ABI of libsalgpu.so
(include/salgpu.h):

* setup, tree_module.f90: ``tree_traverse``, ``dual_tree_traversal``,
  ``single_tree_traversal``, ``assign_points_to_panels``;
* the code.f90 solve, fast_sum_module.f90: ``fast_sum``;
* the mom6_code.f90 solve, mom6_fast_sum_module.f90: ``proxy_source_compute``,
  ``pc_compute``, ``pp_compute``;
* device-resident use: ``Grid`` (one flattened grid, batched ``solve`` on torch
  CUDA tensors) and ``direct_sum`` (FP64 O(N^2) reference sum on the GPU).

Index conventions follow the reference: panel ids, point ids and interaction
lists are 1-based.  There is no CPU path: calls that compute need the CUDA
library and a GPU, and raise ``SalError`` otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsalgpu.so")

SAL_OK, SAL_EINVAL, SAL_ENOMEM, SAL_ECUDA, SAL_ETIMEOUT, SAL_ENODEV, SAL_ETREE = 0, -1, -2, -3, -4, -5, -6
MODE_DTT, MODE_STT_REF_COMPAT, MODE_STT_CORRECT = 0, 1, 2
FORM_REF, FORM_ACCURATE, FORM_MIXED = 0, 1, 2

# every symbol include/salgpu.h declares
EXPORTS = (
    "sal_last_error", "sal_free", "sal_tree_traverse", "sal_tree_import", "sal_tree_info", "sal_tree_export",
    "sal_tree_destroy", "sal_dual_tree_traversal", "sal_single_tree_traversal", "sal_assign_points_to_panels",
    "sal_grid_create", "sal_grid_stats_get", "sal_grid_sync", "sal_grid_destroy", "sal_solve", "sal_fast_sum_host",
    "sal_proxy_source_compute_host", "sal_pc_compute_host", "sal_pp_compute_host", "sal_direct_sum",
    "sal_grid_timing", "sal_fma_peak", "sal_direct_sum_noalloc", "sal_solve_host", "sal_solve_host_async",
    "sal_solve_host_wait", "sal_grid_set_graphs", "sal_grid_inject_timeout", "sal_fast_sum",
    "sal_mom6_proxy_source_compute", "sal_mom6_pc_compute", "sal_mom6_pp_compute", "sal_dropin_config",
    "sal_dropin_release", "sal_grid_tune_get", "sal_grid_tune_set", "sal_grid_autotune", "sal_read_values",
    "sal_write_values", "sal_solve_joint", "sal_tree_traverse_device", "sal_dual_tree_traversal_device",
)


class SalError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"salgpu error {code}: {msg}")
        self.code = code


class GridDesc(C.Structure):
    _fields_ = [
        ("point_count", C.c_int32),
        ("xs", C.c_void_p), ("ys", C.c_void_p), ("zs", C.c_void_p), ("areas", C.c_void_p),
        ("interp_degree", C.c_int32), ("mode", C.c_int32),
        ("list", C.c_void_p), ("list_count", C.c_int64),
        ("pc_list", C.c_void_p), ("pc_count", C.c_int64),
        ("pp_list", C.c_void_p), ("pp_count", C.c_int64),
        ("max_fields", C.c_int32), ("device", C.c_int32),
    ]


class GridStats(C.Structure):
    _fields_ = [
        ("point_count", C.c_int32), ("npanels", C.c_int32), ("nleaves", C.c_int32), ("degree", C.c_int32),
        ("mode", C.c_int32), ("list_count", C.c_int64),
        ("pairs_pp", C.c_double), ("pairs_pc", C.c_double), ("pairs_cp", C.c_double), ("pairs_cc", C.c_double),
        ("macs_up", C.c_double), ("macs_down", C.c_double),
        ("device_bytes", C.c_int64), ("setup_seconds", C.c_double), ("mixed_bytes", C.c_int64),
        ("macs_up_batched", C.c_double), ("macs_down_batched", C.c_double), ("launches_batched", C.c_int64),
        ("tile_store_bytes", C.c_int64),
    ]


class Tune(C.Structure):
    """sal_tune: runtime choices of the batched form's tcgen05 passes."""
    _fields_ = [
        ("chain_ksteps", C.c_int32), ("tree_passes", C.c_int32), ("up_chunk", C.c_int32),
        ("proxy_unit_kpairs", C.c_int32), ("cta_groups", C.c_int32), ("field_block", C.c_int32),
        ("f16", C.c_int32), ("tile_store", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_lock = threading.Lock()


def lib():
    """Loads libsalgpu.so; raises ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C sal-fort_b200` "
                              "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        pp_ = C.POINTER(C.c_void_p)
        L.sal_last_error.restype = C.c_char_p
        L.sal_free.argtypes = [vp]
        L.sal_tree_traverse.argtypes = [vp, vp, vp, i32, i32, pp_]
        L.sal_tree_import.argtypes = [i32, vp, vp, vp, vp, i32, vp, vp, vp, pp_]
        L.sal_tree_info.argtypes = [vp, C.POINTER(i32), C.POINTER(i64), C.POINTER(i32)]
        L.sal_tree_export.argtypes = [vp, vp, vp, vp, vp]
        L.sal_tree_destroy.argtypes = [vp]
        L.sal_dual_tree_traversal.argtypes = [vp, d, i32, C.POINTER(C.POINTER(i32)), C.POINTER(i64)]
        L.sal_tree_traverse_device.argtypes = [vp, vp, vp, i32, i32, i32, pp_]
        L.sal_dual_tree_traversal_device.argtypes = [vp, d, i32, i32, C.POINTER(C.POINTER(i32)), C.POINTER(i64)]
        L.sal_single_tree_traversal.argtypes = [vp, d, i32, vp, vp, vp, i32, C.POINTER(C.POINTER(i32)),
                                                C.POINTER(i64), C.POINTER(C.POINTER(i32)), C.POINTER(i64)]
        L.sal_assign_points_to_panels.argtypes = [vp, vp, vp, vp, i32, vp, i32]
        L.sal_grid_create.argtypes = [vp, C.POINTER(GridDesc), pp_]
        L.sal_grid_stats_get.argtypes = [vp, C.POINTER(GridStats)]
        L.sal_grid_sync.argtypes = [vp, vp]
        L.sal_grid_destroy.argtypes = [vp]
        L.sal_solve.argtypes = [vp, vp, i32, i64, vp, vp, i64, i32, vp]
        L.sal_fast_sum_host.argtypes = [vp, vp, vp, vp, i32]
        L.sal_solve_host.argtypes = [vp, vp, i32, i64, vp, vp, i64, i32]
        L.sal_solve_host_async.argtypes = [vp, vp, i32, i64, vp, vp, i64, i32]
        L.sal_solve_host_wait.argtypes = [vp]
        L.sal_grid_set_graphs.argtypes = [vp, i32]
        L.sal_grid_inject_timeout.argtypes = [vp, i32]
        L.sal_proxy_source_compute_host.argtypes = [vp, vp, vp]
        L.sal_pc_compute_host.argtypes = [vp, vp, vp, vp]
        L.sal_pp_compute_host.argtypes = [vp, vp, vp, vp]
        L.sal_direct_sum.argtypes = [vp, vp, vp, vp, i32, vp, i32, vp, vp, vp]
        L.sal_grid_timing.argtypes = [vp, i32, C.POINTER(d), C.POINTER(i64)]
        L.sal_fma_peak.argtypes = [i32, C.POINTER(d)]
        L.sal_direct_sum_noalloc.argtypes = [vp, vp, vp, vp, i32, vp, i32, vp, vp, vp]
        L.sal_fast_sum.argtypes = [vp, vp, vp, i64, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, i32, i32]
        L.sal_mom6_proxy_source_compute.argtypes = [vp, i32, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, i32, i32]
        L.sal_mom6_pc_compute.argtypes = [vp, vp, vp, i64, i32, vp, vp, vp, vp, vp, vp, vp, i32, i32, vp]
        L.sal_mom6_pp_compute.argtypes = [vp, vp, vp, i64, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                          vp, vp, i32, i32]
        L.sal_dropin_config.argtypes = [i32, i32]
        L.sal_read_values.argtypes = [C.c_char_p, i64, vp]
        L.sal_solve_joint.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp]
        L.sal_write_values.argtypes = [C.c_char_p, i64, vp]
        L.sal_grid_tune_get.argtypes = [vp, C.POINTER(Tune)]
        L.sal_grid_tune_set.argtypes = [vp, C.POINTER(Tune)]
        L.sal_grid_autotune.argtypes = [vp, vp, i32, i64, i32, d, C.POINTER(Tune), C.POINTER(d), C.POINTER(d)]
        _lib = L
        return L


def _check(rc):
    if rc != SAL_OK:
        raise SalError(rc, lib().sal_last_error().decode(errors="replace"))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


# ===================================================================== trees
class Tree:
    """Host cubed-sphere quadtree: the reference's cube_panel array
    (tree_module.f90:5-28), held by libsalgpu.  Panel ids are 1-based."""

    def __init__(self, handle, n):
        self.handle = C.c_void_p(handle)
        self.n_points = n
        self._exp = None

    def __del__(self):
        if getattr(self, "handle", None) and self.handle.value and _lib is not None:
            _lib.sal_tree_destroy(self.handle)
            self.handle = C.c_void_p(0)

    def info(self):
        np_, tot, ml = C.c_int32(), C.c_int64(), C.c_int32()
        _check(lib().sal_tree_info(self.handle, C.byref(np_), C.byref(tot), C.byref(ml)))
        return np_.value, tot.value, ml.value

    @property
    def npanels(self):
        return self.info()[0]

    def export(self):
        """Flattened panels: dict of level, is_leaf, id, parent, child (np,4),
        face, bounds (np,7), pt_off, pt_idx -- the sal_tree_import layout."""
        if self._exp is None:
            npn, tot, _ = self.info()
            ints = np.zeros(9 * npn, np.int32)
            dbl = np.zeros(7 * npn, np.float64)
            off = np.zeros(npn + 1, np.int64)
            idx = np.zeros(max(tot, 1), np.int32)
            _check(lib().sal_tree_export(self.handle, _ptr(ints), _ptr(dbl), _ptr(off), _ptr(idx)))
            I = ints.reshape(npn, 9)
            self._exp = dict(level=I[:, 0].copy(), is_leaf=I[:, 1].copy(), id=I[:, 2].copy(),
                             parent=I[:, 3].copy(), child=I[:, 4:8].copy(), face=I[:, 8].copy(),
                             bounds=dbl.reshape(npn, 7).copy(), pt_off=off, pt_idx=idx[:tot])
        return self._exp

    def points_inside(self, k):
        e = self.export()
        return e["pt_idx"][e["pt_off"][k - 1]:e["pt_off"][k]]


def tree_traverse(xs, ys, zs, point_count, cluster_thresh, device=None) -> Tree:
    """tree_module.f90:59-246.  device: None builds on the host; a CUDA
    ordinal refines on that device (the same tree, bit for bit)."""
    xs, ys, zs = _f64(xs), _f64(ys), _f64(zs)
    if len(xs) != point_count:
        raise ValueError("point_count differs from len(xs)")
    h = C.c_void_p()
    if device is None:
        _check(lib().sal_tree_traverse(_ptr(xs), _ptr(ys), _ptr(zs), int(point_count), int(cluster_thresh),
                                       C.byref(h)))
    else:
        _check(lib().sal_tree_traverse_device(_ptr(xs), _ptr(ys), _ptr(zs), int(point_count), int(cluster_thresh),
                                              int(device), C.byref(h)))
    return Tree(h.value, point_count)


def tree_import(panels: dict, xs, ys, zs) -> Tree:
    """A cube_panel array flattened by another builder (keys as Tree.export)."""
    xs, ys, zs = _f64(xs), _f64(ys), _f64(zs)
    npn = len(panels["level"])
    ints = _i32(np.column_stack([panels["level"], panels["is_leaf"], panels["id"], panels["parent"],
                                 panels["child"], panels["face"]]).reshape(-1))
    dbl = _f64(np.asarray(panels["bounds"]).reshape(-1))
    off = np.ascontiguousarray(panels["pt_off"], dtype=np.int64)
    idx = _i32(panels["pt_idx"])
    h = C.c_void_p()
    _check(lib().sal_tree_import(npn, _ptr(ints), _ptr(dbl), _ptr(off), _ptr(idx), len(xs), _ptr(xs), _ptr(ys),
                                 _ptr(zs), C.byref(h)))
    return Tree(h.value, len(xs))


def _take_list(p, count, width):
    n = count.value
    out = np.ctypeslib.as_array(p, shape=(width * n,)).copy().reshape(n, width) if n else np.zeros((0, width), np.int32)
    lib().sal_free(C.cast(p, C.c_void_p))
    return out


def dual_tree_traversal(tree: Tree, theta, cluster_thresh, device=None) -> np.ndarray:
    """tree_module.f90:277-398: (n, 3) int32 of (index_target, index_source, interact_type).
    device: None traverses on the host, else on that CUDA device (the same list)."""
    p, cnt = C.POINTER(C.c_int32)(), C.c_int64()
    if device is None:
        _check(lib().sal_dual_tree_traversal(tree.handle, float(theta), int(cluster_thresh), C.byref(p),
                                             C.byref(cnt)))
    else:
        _check(lib().sal_dual_tree_traversal_device(tree.handle, float(theta), int(cluster_thresh), int(device),
                                                    C.byref(p), C.byref(cnt)))
    return _take_list(p, cnt, 3)


def single_tree_traversal(tree: Tree, theta, cluster_thresh, xs, ys, zs, own_points=None):
    """tree_module.f90:401-487: (pc, pp) lists of (point id, panel id)."""
    xs, ys, zs = _f64(xs), _f64(ys), _f64(zs)
    own = len(xs) if own_points is None else own_points
    a, na = C.POINTER(C.c_int32)(), C.c_int64()
    b, nb = C.POINTER(C.c_int32)(), C.c_int64()
    _check(lib().sal_single_tree_traversal(tree.handle, float(theta), int(cluster_thresh), _ptr(xs), _ptr(ys),
                                           _ptr(zs), int(own), C.byref(a), C.byref(na), C.byref(b), C.byref(nb)))
    return _take_list(a, na, 2), _take_list(b, nb, 2)


def assign_points_to_panels(tree: Tree, xs, ys, zs, nlev=None) -> np.ndarray:
    """tree_module.f90:249-273: points_panels (nlev, N), -1 filled."""
    xs, ys, zs = _f64(xs), _f64(ys), _f64(zs)
    if nlev is None:
        nlev = int(tree.export()["level"][-1]) + 1   # mom6_code.f90:188-189
    out = np.zeros(nlev * len(xs), np.int32)
    _check(lib().sal_assign_points_to_panels(tree.handle, _ptr(xs), _ptr(ys), _ptr(zs), len(xs), _ptr(out), nlev))
    return out.reshape(nlev, len(xs), order="F")


# ===================================================================== device grids
class Grid:
    """A grid flattened into device-resident arrays (sal_grid_create)."""

    def __init__(self, tree: Tree, xs, ys, zs, areas, interp_degree, mode=MODE_DTT, interaction_list=None,
                 pc_list=None, pp_list=None, device=0, max_fields=1):
        self._keep = [_f64(xs), _f64(ys), _f64(zs), _f64(areas)]
        d = GridDesc()
        d.point_count = len(self._keep[0])
        d.xs, d.ys, d.zs, d.areas = (_ptr(a) for a in self._keep)
        d.interp_degree = int(interp_degree)
        d.mode = int(mode)
        if mode == MODE_DTT:
            L = _i32(np.asarray(interaction_list).reshape(-1))
            self._keep.append(L)
            d.list, d.list_count = _ptr(L), len(L) // 3
        else:
            a, b = _i32(np.asarray(pc_list).reshape(-1)), _i32(np.asarray(pp_list).reshape(-1))
            self._keep += [a, b]
            d.pc_list, d.pc_count = _ptr(a), len(a) // 2
            d.pp_list, d.pp_count = _ptr(b), len(b) // 2
        d.max_fields = int(max_fields)
        d.device = int(device)
        h = C.c_void_p()
        _check(lib().sal_grid_create(tree.handle, C.byref(d), C.byref(h)))
        self.handle = h
        self.n = d.point_count
        self.degree = int(interp_degree)
        self.mode = int(mode)
        self.device = int(device)
        self._keep = None

    def __del__(self):
        if getattr(self, "handle", None) and self.handle.value and _lib is not None:
            _lib.sal_grid_destroy(self.handle)
            self.handle = C.c_void_p(0)

    def stats(self) -> dict:
        s = GridStats()
        _check(lib().sal_grid_stats_get(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in GridStats._fields_}

    def solve(self, ssh, form=FORM_REF, out=None, stream=None):
        """SAL gradient of F fields on the device.  ssh: torch float64 CUDA
        tensor (F, N) or (N,); returns (out_x, out_y) of the same shape."""
        import torch
        if not (ssh.is_cuda and ssh.dtype == torch.float64):
            raise TypeError("ssh must be a float64 CUDA tensor")
        ssh2 = ssh.reshape(-1, self.n).contiguous()
        F = ssh2.shape[0]
        if out is None:
            ox = torch.empty_like(ssh2)
            oy = torch.empty_like(ssh2)
        else:
            ox, oy = out
        st = stream if stream is not None else torch.cuda.current_stream(ssh.device).cuda_stream
        _check(lib().sal_solve(self.handle, C.c_void_p(ssh2.data_ptr()), F, self.n, C.c_void_p(ox.data_ptr()),
                               C.c_void_p(oy.data_ptr()), self.n, int(form), C.c_void_p(st)))
        return ox.view_as(ssh), oy.view_as(ssh)

    def timing(self, enable=-1):
        """Per-pass device milliseconds summed since the last reset:
        (prep+upward, proxy, leaf, total), solves."""
        ms = (C.c_double * 4)()
        n = C.c_int64()
        _check(lib().sal_grid_timing(self.handle, int(enable), ms, C.byref(n)))
        return list(ms), n.value

    def sync(self, stream=None):
        _check(lib().sal_grid_sync(self.handle, C.c_void_p(stream or 0)))

    def solve_host(self, ssh, out_x, out_y, form=FORM_REF):
        """Batched solve on host arrays (F, N) (sal_solve_host): synchronous,
        outputs overwritten.  Pinned arrays make the copies asynchronous."""
        F = ssh.shape[0] if ssh.ndim == 2 else 1
        _check(lib().sal_solve_host(self.handle, _ptr(ssh), F, self.n, _ptr(out_x), _ptr(out_y), self.n, int(form)))

    def tune(self, **changes):
        """The batched form's choices (sal_grid_tune_get) as a dict; keyword
        arguments change them first (sal_grid_tune_set)."""
        t = Tune()
        _check(lib().sal_grid_tune_get(self.handle, C.byref(t)))
        if changes:
            for k, v in changes.items():
                setattr(t, k, int(v))
            _check(lib().sal_grid_tune_set(self.handle, C.byref(t)))
        return t.as_dict()

    def autotune(self, ssh, ntargets=2000, max_rel_err=5e-6):
        """sal_grid_autotune on (F, N) float64 CUDA fields (F <= 64): sets the
        fastest setting whose first field stays within max_rel_err of the FP64
        direct sum; returns (setting, ms of the setting, ms of the start)."""
        ssh2 = ssh.reshape(-1, self.n).contiguous()
        t, mb, ms = Tune(), C.c_double(), C.c_double()
        _check(lib().sal_grid_autotune(self.handle, C.c_void_p(ssh2.data_ptr()), ssh2.shape[0], self.n, int(ntargets),
                                       float(max_rel_err), C.byref(t), C.byref(mb), C.byref(ms)))
        return t.as_dict(), mb.value, ms.value

    def inject_timeout(self, polls):
        """Test hook (sal_grid_inject_timeout): the next FP64 solve's leaf
        pass gives up a staging wait on every group after `polls` polls; the
        host then sees SAL_ETIMEOUT."""
        _check(lib().sal_grid_inject_timeout(self.handle, int(polls)))

    def set_graphs(self, enable=True):
        """CUDA graphs of batched solves, one per call shape (sal_grid_set_graphs):
        the first FORM_MIXED solve of a shape on a non-default stream is
        captured, later ones launch the graph."""
        _check(lib().sal_grid_set_graphs(self.handle, 1 if enable else 0))

    def solve_host_async(self, ssh, out_x, out_y, form=FORM_REF):
        """Pipelined solve on host arrays (sal_solve_host_async): enqueues the
        copies and the solve and returns.  The arrays must be pinned (for
        example numpy views of pinned torch tensors) and left untouched until
        solve_host_wait() returns."""
        F = ssh.shape[0] if ssh.ndim == 2 else 1
        _check(lib().sal_solve_host_async(self.handle, _ptr(ssh), F, self.n, _ptr(out_x), _ptr(out_y), self.n,
                                          int(form)))

    def solve_host_wait(self):
        """Waits for every solve_host_async call of this grid."""
        _check(lib().sal_solve_host_wait(self.handle))

    # ---- host-buffer entry points (synchronous, add into the outputs)
    def fast_sum_host(self, ssh, sal_longrad, sal_latgrad, form=FORM_REF):
        _check(lib().sal_fast_sum_host(self.handle, _ptr(_f64(ssh)), _ptr(sal_longrad), _ptr(sal_latgrad), int(form)))

    def proxy_source_compute_host(self, sshs, weights):
        _check(lib().sal_proxy_source_compute_host(self.handle, _ptr(_f64(sshs)), _ptr(weights)))

    def pc_compute_host(self, weights, sal_x, sal_y):
        _check(lib().sal_pc_compute_host(self.handle, _ptr(_f64(weights)), _ptr(sal_x), _ptr(sal_y)))

    def pp_compute_host(self, sshs, sal_x, sal_y):
        _check(lib().sal_pp_compute_host(self.handle, _ptr(_f64(sshs)), _ptr(sal_x), _ptr(sal_y)))


def solve_joint(grids, sshs, outs=None, stream=None):
    """Batched solves of several grids with one shared leaf-pass launch
    (sal_solve_joint).  grids: Grid objects (max_fields > 32, one degree);
    sshs: (F_k, N_k) float64 CUDA tensors, F_k <= 64.  Returns the list of
    (out_x, out_y) per grid."""
    import torch
    k = len(grids)
    sshs = [s.reshape(-1, g.n).contiguous() for s, g in zip(sshs, grids)]
    if outs is None:
        outs = [(torch.empty_like(s), torch.empty_like(s)) for s in sshs]
    P = C.c_void_p * k
    gh = P(*[g.handle.value for g in grids])
    sp = P(*[s.data_ptr() for s in sshs])
    xp = P(*[o[0].data_ptr() for o in outs])
    yp = P(*[o[1].data_ptr() for o in outs])
    nf = (C.c_int32 * k)(*[s.shape[0] for s in sshs])
    ld = (C.c_int64 * k)(*[g.n for g in grids])
    st = stream if stream is not None else torch.cuda.current_stream(sshs[0].device).cuda_stream
    _check(lib().sal_solve_joint(gh, k, sp, nf, ld, xp, yp, ld, C.c_void_p(st)))
    return outs


def read_values(path, count) -> np.ndarray:
    """The first count values of a one-value-per-line file (the reference's
    input CSVs, code.f90:36-56) or of a raw float64 ".f64" file."""
    out = np.empty(int(count), np.float64)
    _check(lib().sal_read_values(os.fsencode(path), int(count), _ptr(out)))
    return out


def write_values(path, values):
    """Writes values as raw little-endian float64 (the ".f64" form)."""
    v = _f64(values)
    _check(lib().sal_write_values(os.fsencode(path), len(v), _ptr(v)))


def fma_peak(precision=64) -> float:
    """Measured FMA-pipe TFLOP/s of the current device (FP64 or FP32)."""
    v = C.c_double()
    _check(lib().sal_fma_peak(int(precision), C.byref(v)))
    return v.value


NOALLOC_MAX_TARGETS = (1 << 18) // 2   # SAL_NOALLOC_SCRATCH_DOUBLES / 2


def direct_sum_noalloc(xs, ys, zs, w, targets, out_x, out_y, stream=None):
    """direct_sum through sal_direct_sum_noalloc: the library allocates no
    device memory (partial sums go to a fixed 2 MiB array of its own), so the
    caller passes preallocated outputs.  Calls that overlap on the GPU race."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream(xs.device).cuda_stream
    _check(lib().sal_direct_sum_noalloc(C.c_void_p(xs.data_ptr()), C.c_void_p(ys.data_ptr()),
                                        C.c_void_p(zs.data_ptr()), C.c_void_p(w.data_ptr()), xs.numel(),
                                        C.c_void_p(targets.data_ptr()), targets.numel(),
                                        C.c_void_p(out_x.data_ptr()), C.c_void_p(out_y.data_ptr()), C.c_void_p(st)))
    return out_x, out_y


def direct_sum(xs, ys, zs, w, targets, stream=None):
    """FP64 direct sum on the GPU at 0-based targets; inputs are torch CUDA
    tensors (float64 xs, ys, zs, w = area*ssh; int32 targets)."""
    import torch
    nt = targets.numel()
    ox = torch.empty(nt, dtype=torch.float64, device=xs.device)
    oy = torch.empty_like(ox)
    st = stream if stream is not None else torch.cuda.current_stream(xs.device).cuda_stream
    _check(lib().sal_direct_sum(C.c_void_p(xs.data_ptr()), C.c_void_p(ys.data_ptr()), C.c_void_p(zs.data_ptr()),
                                C.c_void_p(w.data_ptr()), xs.numel(), C.c_void_p(targets.data_ptr()), nt,
                                C.c_void_p(ox.data_ptr()), C.c_void_p(oy.data_ptr()), C.c_void_p(st)))
    return ox, oy


# ===================================================================== reference-named entry points
# The reference's four hot routines with its argument lists, through the
# library's reference-signature entry points (include/salgpu.h): each call
# hands over the flattened cube_panel array, the list and the point arrays;
# the library reuses the device grid it built for the same contents.

def _flat_panels(cube_panels, with_points=True):
    """(npanels, ints9, dbl7, pt_off, pt_idx or None) of a Tree or of a dict
    in the Tree.export() layout (the cube_panel array of tree_module.f90:5-28)."""
    e = cube_panels.export() if isinstance(cube_panels, Tree) else cube_panels
    npn = len(e["level"])
    ints = _i32(np.column_stack([e["level"], e["is_leaf"], e["id"], e["parent"], e["child"], e["face"]]).reshape(-1))
    dbl = _f64(np.asarray(e["bounds"]).reshape(-1))
    off = np.ascontiguousarray(e["pt_off"], dtype=np.int64)
    idx = _i32(e["pt_idx"]) if with_points else None
    return npn, ints, dbl, off, idx


def _panel_ptrs(fp):
    npn, ints, dbl, off, idx = fp
    return [npn, _ptr(ints), _ptr(dbl), _ptr(off), None if idx is None else _ptr(idx)]


def dropin_config(form=FORM_REF, mom6_mode=MODE_STT_REF_COMPAT):
    """Arithmetic form of fast_sum (FORM_REF or FORM_ACCURATE) and proxy-weight
    orientation of proxy_source_compute (MODE_STT_REF_COMPAT, the reference's
    transposed store, or MODE_STT_CORRECT)."""
    _check(lib().sal_dropin_config(int(form), int(mom6_mode)))


def dropin_release():
    """Frees the device grids the reference-named entry points keep."""
    _check(lib().sal_dropin_release())


def fast_sum(sal_longrad, sal_latgrad, interaction_list, cube_panels, xs, ys, zs, area, ssh, point_count,
             interp_degree, rank=0, process_count=1, with_points_inside=True):
    """fast_sum_module.f90:291-332.  Adds into sal_longrad/sal_latgrad
    (intent(inout), float64 arrays).  With process_count > 1 only interactions i
    with MOD(i, process_count) == rank are evaluated (:303-304), so the MPI
    Sum_Array that follows in code.f90:99-100 still yields the full sum."""
    L = _i32(np.asarray(interaction_list).reshape(-1))
    xs, ys, zs, area, ssh = _f64(xs), _f64(ys), _f64(zs), _f64(area), _f64(ssh)
    fp = _flat_panels(cube_panels, with_points_inside)
    _check(lib().sal_fast_sum(_ptr(sal_longrad), _ptr(sal_latgrad), _ptr(L), len(L) // 3, *_panel_ptrs(fp),
                              _ptr(xs), _ptr(ys), _ptr(zs), _ptr(area), _ptr(ssh), int(point_count),
                              int(interp_degree), int(rank), int(process_count)))


def proxy_source_compute(proxy_source_weights, tree_panels, points_panels, xs, ys, zs, sshs, areas, interp_degree,
                         point_count, with_points_inside=True):
    """mom6_fast_sum_module.f90:33-74: adds the proxy source weights
    ((d+1)^2 * npanels, panel-major) into proxy_source_weights.  points_panels
    is (nlev, N) as assign_points_to_panels returns it."""
    pp = np.asarray(points_panels)
    nlev = pp.shape[0]
    ppf = _i32(pp.reshape(-1, order="F"))
    xs, ys, zs, sshs, areas = _f64(xs), _f64(ys), _f64(zs), _f64(sshs), _f64(areas)
    fp = _flat_panels(tree_panels, with_points_inside)
    _check(lib().sal_mom6_proxy_source_compute(_ptr(proxy_source_weights), *_panel_ptrs(fp), _ptr(ppf), nlev,
                                               _ptr(xs), _ptr(ys), _ptr(zs), _ptr(sshs), _ptr(areas),
                                               int(interp_degree), int(point_count)))


def pc_compute(sal_longrad, sal_latgrad, pc_interaction_list, cube_panels, xs, ys, zs, interp_degree, proxy_weights,
               with_points_inside=True):
    """mom6_fast_sum_module.f90:153-174: adds the particle-cluster far field."""
    L = _i32(np.asarray(pc_interaction_list).reshape(-1))
    xs, ys, zs, w = _f64(xs), _f64(ys), _f64(zs), _f64(proxy_weights)
    fp = _flat_panels(cube_panels, with_points_inside)
    _check(lib().sal_mom6_pc_compute(_ptr(sal_longrad), _ptr(sal_latgrad), _ptr(L), len(L) // 2, *_panel_ptrs(fp),
                                     _ptr(xs), _ptr(ys), _ptr(zs), len(xs), int(interp_degree), _ptr(w)))


def pp_compute(sal_longrad, sal_latgrad, pp_interaction_list, cube_panels, xs, ys, zs, areas, sshs, e_xs=(), e_ys=(),
               e_zs=(), e_areas=(), e_sshs=(), own_points=None, with_points_inside=True):
    """mom6_fast_sum_module.f90:177-192: adds the near field.  One rank: the
    halo arrays e_* of other ranks' points must be empty."""
    L = _i32(np.asarray(pp_interaction_list).reshape(-1))
    xs, ys, zs, areas, sshs = _f64(xs), _f64(ys), _f64(zs), _f64(areas), _f64(sshs)
    ex = [_f64(a) for a in (e_xs, e_ys, e_zs, e_areas, e_sshs)]
    own = len(xs) if own_points is None else int(own_points)
    fp = _flat_panels(cube_panels, with_points_inside)
    _check(lib().sal_mom6_pp_compute(_ptr(sal_longrad), _ptr(sal_latgrad), _ptr(L), len(L) // 2, *_panel_ptrs(fp),
                                     _ptr(xs), _ptr(ys), _ptr(zs), _ptr(areas), _ptr(sshs),
                                     *[_ptr(a) for a in ex], len(ex[0]), own))


def mom6_grid(tree, pc_list, pp_list, xs, ys, zs, areas, interp_degree, ref_compat=True, device=0) -> Grid:
    """A device grid of the mom6_code.f90 path with both lists, for the
    Grid.proxy_source_compute_host / pc_compute_host / pp_compute_host
    methods."""
    mode = MODE_STT_REF_COMPAT if ref_compat else MODE_STT_CORRECT
    pc, pp = _i32(np.asarray(pc_list).reshape(-1, 2)), _i32(np.asarray(pp_list).reshape(-1, 2))
    return Grid(tree, xs, ys, zs, areas, interp_degree, mode, pc_list=pc, pp_list=pp, device=device)
