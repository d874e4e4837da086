"""Differentiable RGF: a ``torch.autograd.Function`` with a hand-written adjoint.

The reference has no gradients; this adds dL/dA on the tridiagonal pattern
for any real loss L of the selected blocks (for example the density of
states ``-Im Tr G_ii / pi``).  The forward pass is the ordinary RGF
(``src/sinv/algorithms/rgf/rgf.py:17-64``) that also saves checkpoints of the
left-connected blocks every ceil(sqrt(n)) block rows; the backward pass runs
both sweeps in reverse on the GPU, recomputing the left-connected blocks
between checkpoints instead of storing them.

Gradients follow torch's convention (dL/dA* for complex inputs).  complex128
and float64 run natively; complex64 / float32 are computed in FP64 and the
gradients rounded back.
"""

import ctypes

import torch

from .. import _lib
from . import _device as dev


def _checkpoints(lib, n):
    every, count = ctypes.c_int(0), ctypes.c_int(0)
    _lib.check(lib.sinvb_rgf_checkpoints(n, ctypes.byref(every), ctypes.byref(count)), "sinvb_rgf_checkpoints")
    return every.value, count.value


def _wide(torch, dt):
    return {torch.complex64: torch.complex128, torch.float32: torch.float64}.get(dt, dt)


def _forward(A_diag, A_upper, A_lower, sym_mat, team):
    torch = dev._torch()
    lib = _lib.load()
    dt = _wide(torch, A_diag.dtype)
    code = _lib.dtype_code(dt)
    d = A_diag.detach().to(dt).contiguous()
    n, b = int(d.shape[0]), int(d.shape[1])
    u = A_upper.detach().to(dt).contiguous()
    l = A_lower.detach().to(dt).contiguous()
    flags = _lib.SAVE_OFFDIAG | (_lib.SYM if sym_mat else 0) | {None: 0, "cta": _lib.FORCE_CTA,
                                                               "grid": _lib.FORCE_GRID}[team]
    every, count = _checkpoints(lib, n)
    Gd = torch.empty_like(d)
    Gu = torch.empty_like(u)
    Gl = torch.empty_like(l)
    ck = torch.empty((max(count, 1), b, b), dtype=dt, device=d.device)
    ws = dev.workspace(lib.sinvb_rgf_workspace_size(n, b, code, flags), d.device)
    fn = lib.sinvb_rgf_forward_ckpt_z if code == _lib.C128 else lib.sinvb_rgf_forward_ckpt_d
    rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), n, b, flags, dev.ptr(Gd), dev.ptr(Gu), dev.ptr(Gl),
            ck.data_ptr(), every, dev.ptr(ws), ws.numel(), dev.stream_handle())
    _lib.check(rc, "sinvb_rgf_forward_ckpt")
    dev.raise_for_status(dev.read_status(lib, ws), "rgf (autograd forward)")
    return d, u, l, Gd, Gu, Gl, ck, every, flags


def _adjoint(d, u, l, Gd, Gu, Gl, ck, every, flags, bGd, bGu, bGl):
    torch = dev._torch()
    lib = _lib.load()
    dt = d.dtype
    code = _lib.dtype_code(dt)
    n, b = int(d.shape[0]), int(d.shape[1])

    def prep(x, like):
        return torch.zeros_like(like) if x is None else x.to(dt).contiguous()

    bGd = prep(bGd, Gd)
    bGu = prep(bGu, Gu)
    bGl = prep(bGl, Gl)
    aD = torch.empty_like(d)
    aU = torch.empty_like(u)
    aL = torch.empty_like(l)
    ws = dev.workspace(lib.sinvb_rgf_adjoint_workspace_size(n, b, code, flags), d.device)
    fn = lib.sinvb_rgf_adjoint_z if code == _lib.C128 else lib.sinvb_rgf_adjoint_d
    rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), dev.ptr(Gd), dev.ptr(Gu), dev.ptr(Gl), dev.ptr(bGd), dev.ptr(bGu),
            dev.ptr(bGl), ck.data_ptr(), every, n, b, flags, dev.ptr(aD), dev.ptr(aU), dev.ptr(aL), dev.ptr(ws),
            ws.numel(), dev.stream_handle())
    _lib.check(rc, "sinvb_rgf_adjoint")
    dev.raise_for_status(dev.read_status(lib, ws), "rgf (adjoint)")
    return aD, aU, aL


class RGFFunction(torch.autograd.Function):
    """``(A_diag, A_upper, A_lower) -> (G_diag, G_upper, G_lower)`` with the GPU adjoint."""

    @staticmethod
    def forward(ctx, A_diag, A_upper, A_lower, sym_mat=False, team=None):
        d, u, l, Gd, Gu, Gl, ck, every, flags = _forward(A_diag, A_upper, A_lower, sym_mat, team)
        ctx.save_for_backward(d, u, l, Gd, Gu, Gl, ck)
        ctx.every, ctx.flags = every, flags
        ctx.in_dtypes = (A_diag.dtype, A_upper.dtype, A_lower.dtype)
        out_dt = A_diag.dtype
        return Gd.to(out_dt), Gu.to(out_dt), Gl.to(out_dt)

    @staticmethod
    def backward(ctx, bGd, bGu, bGl):
        d, u, l, Gd, Gu, Gl, ck = ctx.saved_tensors
        aD, aU, aL = _adjoint(d, u, l, Gd, Gu, Gl, ck, ctx.every, ctx.flags, bGd, bGu, bGl)
        dd, du, dl = ctx.in_dtypes
        return aD.to(dd), aU.to(du), aL.to(dl), None, None


def rgf_autograd(A_diag, A_upper, A_lower, sym_mat=False, team=None):
    """Differentiable selected inversion of torch CUDA tensors.

    Returns ``(G_diag, G_upper, G_lower)`` connected to the autograd graph of
    the inputs; ``backward`` runs the GPU adjoint.
    """
    return RGFFunction.apply(A_diag, A_upper, A_lower, sym_mat, team)


# --------------------------------------------------------------------------- batches
def _p(x):
    """Device address of a tensor for a descriptor field (None: absent or empty)."""
    return x.data_ptr() if x is not None and x.numel() > 0 else None


def _forward_batched(instances, sym_mat):
    """Batched forward with checkpoints: one persistent launch over all
    instances (``sinvb_rgf_batched_ckpt_*``)."""
    torch = dev._torch()
    lib = _lib.load()
    dt = _wide(torch, instances[0][0].dtype)
    code = _lib.dtype_code(dt)
    if code not in (_lib.C128, _lib.F64):
        raise TypeError("batched autograd takes complex or real floating tensors")
    flags = _lib.SAVE_OFFDIAG | (_lib.SYM if sym_mat else 0)
    count = len(instances)
    descs = (_lib.BatchDesc * count)()
    cks = (ctypes.c_void_p * count)()
    saved = []
    for k, (A_diag, A_upper, A_lower) in enumerate(instances):
        d = A_diag.detach().to(dt).contiguous()
        n, b = int(d.shape[0]), int(d.shape[1])
        u = A_upper.detach().to(dt).contiguous()
        l = A_lower.detach().to(dt).contiguous()
        every, nck = _checkpoints(lib, n)
        Gd, Gu, Gl = torch.empty_like(d), torch.empty_like(u), torch.empty_like(l)
        ck = torch.empty((max(nck, 1), b, b), dtype=dt, device=d.device)
        descs[k] = _lib.BatchDesc(_p(d), _p(u), _p(l), _p(Gd), _p(Gu), _p(Gl), n, b)
        cks[k] = ck.data_ptr()
        saved.append((d, u, l, Gd, Gu, Gl, ck))
    device = saved[0][0].device
    nbytes = lib.sinvb_rgf_batched_workspace_size(ctypes.cast(descs, ctypes.c_void_p), count, code, flags)
    ws = dev.workspace(nbytes, device)
    status = torch.zeros(count, dtype=torch.int32, device=device)
    fn = lib.sinvb_rgf_batched_ckpt_z if code == _lib.C128 else lib.sinvb_rgf_batched_ckpt_d
    rc = fn(ctypes.cast(descs, ctypes.c_void_p), count, flags, ctypes.cast(cks, ctypes.c_void_p), dev.ptr(ws),
            ws.numel(), dev.ptr(status), dev.stream_handle())
    _lib.check(rc, "sinvb_rgf_batched_ckpt")
    _raise_for_statuses(status, "rgf (batched autograd forward)")
    return saved, flags


def _raise_for_statuses(status, where):
    st = status.cpu().numpy()
    bad = [k for k in range(len(st)) if st[k]]
    if bad:
        import numpy as np
        if st[bad[0]] == _lib.STATUS_PIVOT:
            raise np.linalg.LinAlgError("%s: zero or non-finite pivot in instance %d" % (where, bad[0]))
        raise RuntimeError("%s: instance %d status %d" % (where, bad[0], st[bad[0]]))


def _adjoint_batched(saved, flags, grads):
    """Batched adjoint (``sinvb_rgf_adjoint_batched_*``): one persistent launch."""
    torch = dev._torch()
    lib = _lib.load()
    count = len(saved)
    dt = saved[0][0].dtype
    code = _lib.dtype_code(dt)
    descs = (_lib.AdjointDesc * count)()
    outs, keep = [], []
    for k, ((d, u, l, Gd, Gu, Gl, ck), (bGd, bGu, bGl)) in enumerate(zip(saved, grads)):
        n, b = int(d.shape[0]), int(d.shape[1])
        bGd = torch.zeros_like(Gd) if bGd is None else bGd.to(dt).contiguous()
        bGu = None if bGu is None else bGu.to(dt).contiguous()
        bGl = None if bGl is None else bGl.to(dt).contiguous()
        aD, aU, aL = torch.empty_like(d), torch.empty_like(u), torch.empty_like(l)
        every, nck = _checkpoints(lib, n)
        descs[k] = _lib.AdjointDesc(_p(d), _p(u), _p(l), _p(Gd), _p(Gu), _p(Gl), _p(bGd), _p(bGu), _p(bGl),
                                    _p(ck) if nck else None, _p(aD), _p(aU), _p(aL), n, b)
        keep.append((bGd, bGu, bGl))
        outs.append((aD, aU, aL))
    device = saved[0][0].device
    nbytes = lib.sinvb_rgf_adjoint_batched_workspace_size(ctypes.cast(descs, ctypes.c_void_p), count, code, flags)
    ws = dev.workspace(nbytes, device)
    status = torch.zeros(count, dtype=torch.int32, device=device)
    fn = lib.sinvb_rgf_adjoint_batched_z if code == _lib.C128 else lib.sinvb_rgf_adjoint_batched_d
    rc = fn(ctypes.cast(descs, ctypes.c_void_p), count, flags, dev.ptr(ws), ws.numel(), dev.ptr(status),
            dev.stream_handle())
    _lib.check(rc, "sinvb_rgf_adjoint_batched")
    _raise_for_statuses(status, "rgf (batched adjoint)")
    del keep
    return outs


class RGFBatchFunction(torch.autograd.Function):
    """Many selected inversions with the GPU adjoint, each direction one
    persistent launch: ``(sym_mat, d_0, u_0, l_0, d_1, ...) -> (G_diag_0,
    G_upper_0, G_lower_0, ...)``."""

    @staticmethod
    def forward(ctx, sym_mat, *flat):
        inst = [tuple(flat[3 * k:3 * k + 3]) for k in range(len(flat) // 3)]
        saved, flags = _forward_batched(inst, sym_mat)
        ctx.saved, ctx.flags = saved, flags
        ctx.in_dtypes = [x.dtype for x in flat]
        out = []
        for (d, u, l, Gd, Gu, Gl, ck), (A_d, _, _) in zip(saved, inst):
            out += [Gd.to(A_d.dtype), Gu.to(A_d.dtype), Gl.to(A_d.dtype)]
        return tuple(out)

    @staticmethod
    def backward(ctx, *flat_grads):
        grads = [tuple(flat_grads[3 * k:3 * k + 3]) for k in range(len(ctx.saved))]
        outs = _adjoint_batched(ctx.saved, ctx.flags, grads)
        res = []
        for (aD, aU, aL), k in zip(outs, range(len(outs))):
            res += [aD.to(ctx.in_dtypes[3 * k]), aU.to(ctx.in_dtypes[3 * k + 1]), aL.to(ctx.in_dtypes[3 * k + 2])]
        ctx.saved = None
        return (None, *res)


def rgf_batched_autograd(instances, sym_mat=False):
    """Differentiable selected inversion of many instances (torch CUDA
    tensors, each ``(A_diag, A_upper, A_lower)``, own n and b): one batched
    forward launch, and on ``backward`` one batched adjoint launch.  Returns
    a list of ``(G_diag, G_upper, G_lower)``."""
    flat = [x for inst in instances for x in inst]
    out = RGFBatchFunction.apply(sym_mat, *flat)
    return [tuple(out[3 * k:3 * k + 3]) for k in range(len(instances))]
