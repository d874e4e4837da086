"""The allocation-free entry point against the workspace-taking one.

``sinvb_rgf_z_noalloc`` serves callers that cannot allocate device memory at
call time (inside an allocator hook or host callback that must not re-enter
the allocator, or in a plugin whose host owns all device memory).  Its scratch is a static device array inside the library, so
this test passes only inputs and outputs, calls it twice in a row (the array
keeps the previous call's contents, which must not leak into the next
result), and compares both results with ``sinvb_rgf_z`` at the plain-path
tolerance of the other GPU tests (1e-12 relative Frobenius per block family).

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

from sinv_b200 import _lib, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _with_workspace(lib, d, u, l, n, b, flags, stream):
    import torch
    Gd, Gu, Gl = torch.empty_like(d), torch.empty_like(u), torch.empty_like(l)
    ws = torch.empty(lib.sinvb_rgf_workspace_size(n, b, _lib.C128, flags), dtype=torch.uint8, device="cuda")
    rc = lib.sinvb_rgf_z(d.data_ptr(), u.data_ptr(), l.data_ptr(), n, b, flags, Gd.data_ptr(), Gu.data_ptr(),
                         Gl.data_ptr(), ws.data_ptr(), ws.numel(), stream)
    assert rc == _lib.OK
    return Gd, Gu, Gl


def _without_allocation(lib, d, u, l, n, b, flags, stream, outs, status):
    Gd, Gu, Gl = outs
    rc = lib.sinvb_rgf_z_noalloc(d.data_ptr(), u.data_ptr(), l.data_ptr(), n, b, flags, Gd.data_ptr(),
                                 Gu.data_ptr(), Gl.data_ptr(), status.data_ptr(), stream)
    assert rc == _lib.OK
    return Gd, Gu, Gl


@pytest.mark.parametrize("n,b,sym", [(10, 32, False), (6, 64, False), (5, 17, True), (1, 8, False)])
def test_noalloc_matches_workspace_entry_point(n, b, sym):
    import torch
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    flags = _lib.SAVE_OFFDIAG | (_lib.SYM if sym else 0)
    d, u, l = workloads.dominant(n, b, seed=50 + n + b)
    if sym:
        d = d + np.transpose(d, (0, 2, 1))
        l = np.ascontiguousarray(np.transpose(u, (0, 2, 1)))
    d, u, l = _dev(d), _dev(u), _dev(l)
    ref = _with_workspace(lib, d, u, l, n, b, flags, stream)
    status = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    for call in range(2):   # two calls in a row through the same static scratch
        outs = tuple(torch.full_like(x, float("nan")) for x in (d, u, l))
        got = _without_allocation(lib, d, u, l, n, b, flags, stream, outs, status)
        torch.cuda.synchronize()
        assert int(status.item()) == _lib.OK
        for g, r in zip(got, ref):
            if r.numel():
                assert _rel(g.cpu().numpy(), r.cpu().numpy()) <= TOL, (call, _rel(g.cpu().numpy(), r.cpu().numpy()))


def test_noalloc_reports_pivot_failure_then_recovers():
    import torch
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    d, u, l = workloads.dominant(3, 8, seed=1)
    d[1] = 0.0
    u[0] = 0.0
    dd, uu, ll = _dev(d), _dev(u), _dev(l)
    status = torch.zeros((1,), dtype=torch.int32, device="cuda")
    outs = tuple(torch.empty_like(x) for x in (dd, uu, ll))
    _without_allocation(lib, dd, uu, ll, 3, 8, _lib.SAVE_OFFDIAG, stream, outs, status)
    torch.cuda.synchronize()
    assert int(status.item()) == _lib.STATUS_PIVOT
    # the next call starts from a cleared status word
    d2, u2, l2 = (_dev(x) for x in workloads.dominant(3, 8, seed=1))
    _without_allocation(lib, d2, u2, l2, 3, 8, _lib.SAVE_OFFDIAG, stream, outs, status)
    torch.cuda.synchronize()
    assert int(status.item()) == _lib.OK


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    d, u, l = (_dev(x) for x in workloads.dominant(2, 65, seed=3))
    outs = [torch.empty_like(x) for x in (d, u, l)]
    rc = lib.sinvb_rgf_z_noalloc(d.data_ptr(), u.data_ptr(), l.data_ptr(), 2, 65, _lib.SAVE_OFFDIAG,
                                 outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), None, stream)
    assert rc == _lib.EINVAL
    # off-diagonal outputs are the sweep's per-row storage: required for n > 1
    rc = lib.sinvb_rgf_z_noalloc(d.data_ptr(), u.data_ptr(), l.data_ptr(), 2, 64, 0, outs[0].data_ptr(),
                                 None, None, None, stream)
    assert rc == _lib.EINVAL


def test_noalloc_rejects_outputs_that_overlap_inputs():
    """The sweep keeps per-row products in G_upper / G_lower while it still
    reads A, so an output array over an input (or over another output) would
    give wrong results silently: the call refuses it."""
    import torch
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    d, u, l = (_dev(x) for x in workloads.dominant(4, 16, seed=4))
    Gd, Gu, Gl = (torch.empty_like(x) for x in (d, u, l))
    for outs in [(d, Gu, Gl), (Gd, u, Gl), (Gd, Gu, l), (Gd, Gl, Gl), (Gd, Gu, u[1:])]:
        rc = lib.sinvb_rgf_z_noalloc(d.data_ptr(), u.data_ptr(), l.data_ptr(), 4, 16, _lib.SAVE_OFFDIAG,
                                     outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), None, stream)
        assert rc == _lib.EINVAL
    rc = lib.sinvb_rgf_z_noalloc(d.data_ptr(), u.data_ptr(), l.data_ptr(), 4, 16, _lib.SAVE_OFFDIAG,
                                 Gd.data_ptr(), Gu.data_ptr(), Gl.data_ptr(), None, stream)
    assert rc == _lib.OK
    torch.cuda.synchronize()
