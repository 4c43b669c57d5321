"""GPU test of sal_direct_sum_noalloc, the allocation-free direct sum.

Some callers cannot call cudaMalloc: a thread that runs while another
framework's caching allocator already owns the device's memory, or code that
cannot accept the device-wide synchronisation cudaMalloc/cudaFree may cause.
For them the library offers a direct sum whose scratch is a fixed 2 MiB array
in its own device memory.  This test calls that entry point through the C ABI
twice in a row, with different inputs and sizes, and checks each result against
the allocating sal_direct_sum within the FP64 tolerance used for the direct sum
elsewhere (rel-L2 <= 1e-13; the two may split the sources into a different
number of chunks, which changes only the summation order).  It also checks the
size limit is enforced on the host.  The file is named to be collected last.
"""
import numpy as np
import pytest

from conftest import grid_and_ssh, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _case(name, nt, seed):
    import torch
    g, hh = grid_and_ssh(name)
    T = lambda a: torch.tensor(a, device="cuda")
    tg = np.sort(np.random.default_rng(seed).choice(g.n, nt, replace=False)).astype(np.int32)
    return T(g.xs), T(g.ys), T(g.zs), T(g.areas * hh[0]), T(tg)


def test_noalloc_direct_sum_matches_allocating_entry_point_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import salgpu as S
    torch.cuda.set_device(0)
    # first call: 28,673 sources, 3,000 targets (one source chunk)
    # second call: 200,000 sources, 60,000 targets (the scratch limit caps the
    # chunk count below the allocating entry point's)
    for name, nt, seed in (("cfg0", 3000, 1), ("small_200000", 60000, 2)):
        xs, ys, zs, w, tg = _case(name, nt, seed)
        ref_x, ref_y = S.direct_sum(xs, ys, zs, w, tg)
        out_x = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
        out_y = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
        S.direct_sum_noalloc(xs, ys, zs, w, tg, out_x, out_y)
        torch.cuda.synchronize()
        a = [t.cpu().numpy() for t in (out_x, out_y, ref_x, ref_y)]
        assert np.all(np.isfinite(a[0])) and np.all(np.isfinite(a[1]))
        assert rel_l2(a[0], a[1], a[2], a[3]) <= TOL


def test_noalloc_rejects_sizes_beyond_the_scratch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import salgpu as S
    nt = S.NOALLOC_MAX_TARGETS + 1
    xs = torch.zeros(4, dtype=torch.float64, device="cuda")
    tg = torch.zeros(nt, dtype=torch.int32, device="cuda")
    out = torch.zeros(nt, dtype=torch.float64, device="cuda")
    with pytest.raises(S.SalError) as e:
        S.direct_sum_noalloc(xs, xs, xs, xs, tg, out, out)
    assert e.value.code == S.SAL_EINVAL and "scratch limit" in str(e.value)
