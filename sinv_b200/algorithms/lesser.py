"""Lesser Green's function on the tridiagonal blocks: G< = G Sigma< G^H.

No reference counterpart: in a transport code this is the step after ``rgf``
(``src/sinv/algorithms/rgf/rgf.py:17-64``) at every energy point, with the
lesser self-energy Sigma< of the contacts (block-diagonal).  One sweep pair
(``sinvb_rgf_lesser_z``) gives the retarded blocks of ``rgf`` and the lesser
blocks G<_ii, G<_{i,i+1}; G<_{i+1,i} = -(G<_{i,i+1})^H (G< is anti-Hermitian).
``rgf_greater`` is the same computation for the greater self-energy.
``rgf_lesser_batched`` / ``rgf_greater_batched`` take many energies (own n
and b each) in one persistent launch (``sinvb_rgf_lesser_batched_z``).
"""

import ctypes

import numpy as np

from .. import _lib
from . import _device as dev


def rgf_lesser(A_diag, A_upper, A_lower, Sigma_lesser, team=None, check=True, stream=None):
    """``(A blocks, Sigma<_ii blocks) -> (G_diag, G_upper, G_lower, GL_diag, GL_upper, GL_lower)``.

    complex128, numpy or torch (numpy in, numpy out).  ``Sigma_lesser``: (n, b, b).
    ``team``: ``"cta"`` or ``"grid"`` as for ``rgf.rgf_blocks``.
    """
    torch = dev._torch()
    lib = _lib.load()
    tdt = dev.torch_dtype(A_diag)
    if tdt != torch.complex128:
        raise TypeError("rgf_lesser takes complex128 blocks")
    d = dev.to_device(A_diag, tdt)
    n, b = int(d.shape[0]), int(d.shape[1])
    s = dev.to_device(Sigma_lesser, tdt)
    if tuple(s.shape) != (n, b, b):
        raise ValueError("Sigma_lesser must be (%d, %d, %d)" % (n, b, b))
    u = dev.to_device(A_upper, tdt) if n > 1 else None
    l = dev.to_device(A_lower, tdt) if n > 1 else None
    flags = {None: 0, "cta": _lib.FORCE_CTA, "grid": _lib.FORCE_GRID}[team]
    out = [torch.empty((k, b, b), dtype=tdt, device=d.device) for k in (n, n - 1, n - 1, n, n - 1)]
    with torch.cuda.device(d.device):
        ws = dev.workspace(lib.sinvb_rgf_lesser_workspace_size(n, b), d.device)
        rc = lib.sinvb_rgf_lesser_z(dev.ptr(d), dev.ptr(u), dev.ptr(l), dev.ptr(s), n, b, flags,
                                    *(dev.ptr(t) if t.numel() else None for t in out), dev.ptr(ws), ws.numel(),
                                    dev.stream_handle(stream))
        _lib.check(rc, "sinvb_rgf_lesser")
        if check:
            dev.raise_for_status(dev.read_status(lib, ws, stream), "rgf_lesser")
    Gd, Gu, Gl, GLd, GLu = out
    GLl = -GLu.conj().transpose(1, 2).contiguous()
    return tuple(dev.to_output(t, A_diag) for t in (Gd, Gu, Gl, GLd, GLu, GLl))


def rgf_greater(A_diag, A_upper, A_lower, Sigma_greater, team=None, check=True, stream=None):
    """``(A blocks, Sigma>_ii blocks) -> (G_diag, G_upper, G_lower, GG_diag, GG_upper, GG_lower)``:
    the greater Green's function G> = G Sigma> G^H on the tridiagonal blocks.

    Sigma> is anti-Hermitian like Sigma< (both are i times a Hermitian
    broadening), and the recursions of ``rgf_lesser`` use nothing else about
    the self-energy, so the same sweep pair computes G>; GG_lower is
    -(GG_upper)^H.  With Sigma> - Sigma< = Sigma^R - Sigma^A the results obey
    G> - G< = G - G^H.
    """
    return rgf_lesser(A_diag, A_upper, A_lower, Sigma_greater, team=team, check=check, stream=stream)


def rgf_lesser_batched(instances, sigmas, team=None, check=True, stream=None, statuses=None):
    """Many energies at once: ``instances`` a list of ``(A_diag, A_upper,
    A_lower)`` and ``sigmas`` the matching list of Sigma< blocks (n, b, b);
    returns a list of ``(G_diag, G_upper, G_lower, GL_diag, GL_upper,
    GL_lower)``, each as ``rgf_lesser`` returns it for that instance.

    complex128, numpy or torch per instance (numpy in, numpy out).  Inputs
    may be shared between instances (for example the coupling blocks of one
    Hamiltonian at every energy).  ``team``: None (teams sized by block size)
    or ``"cta"`` (one CTA per instance).  With ``check`` a zero or non-finite
    pivot in any instance raises ``numpy.linalg.LinAlgError`` naming it;
    ``statuses`` (a list) receives every instance's status code either way.
    """
    torch = dev._torch()
    lib = _lib.load()
    if len(instances) != len(sigmas) or not instances:
        raise ValueError("rgf_lesser_batched takes matching, non-empty lists of instances and self-energies")
    descs = (_lib.LesserDesc * len(instances))()
    keep, outs = [], []
    device = None
    moved = {}   # one device copy of a host array that several instances share

    def to_dev(x):
        if dev.is_torch(x) and x.is_cuda:
            return dev.to_device(x, torch.complex128)
        if id(x) not in moved:
            moved[id(x)] = (x, dev.to_device(x, torch.complex128))
        return moved[id(x)][1]

    for k, ((A_diag, A_upper, A_lower), sig) in enumerate(zip(instances, sigmas)):
        if dev.torch_dtype(A_diag) != torch.complex128:
            raise TypeError("rgf_lesser_batched takes complex128 blocks (instance %d)" % k)
        d = to_dev(A_diag)
        if device is not None and d.device != device:
            raise ValueError("rgf_lesser_batched: every instance must be on one device (instance %d)" % k)
        n, b = int(d.shape[0]), int(d.shape[1])
        s = to_dev(sig)
        if tuple(s.shape) != (n, b, b):
            raise ValueError("Sigma_lesser of instance %d must be (%d, %d, %d)" % (k, n, b, b))
        u = to_dev(A_upper) if n > 1 else None
        l = to_dev(A_lower) if n > 1 else None
        out = [torch.empty((m, b, b), dtype=torch.complex128, device=d.device) for m in (n, n - 1, n - 1, n, n - 1)]
        descs[k] = _lib.LesserDesc(*(dev.ptr(t) for t in (d, u, l, s)), *(dev.ptr(t) for t in out), n, b)
        keep.append((d, u, l, s))
        outs.append(out)
        device = d.device
    flags = {None: 0, "cta": _lib.FORCE_CTA}[team]
    with torch.cuda.device(device):
        nbytes = lib.sinvb_rgf_lesser_batched_workspace_size(ctypes.cast(descs, ctypes.c_void_p), len(descs), flags)
        ws = dev.workspace(nbytes, device)
        status = torch.zeros(len(descs), dtype=torch.int32, device=device)
        rc = lib.sinvb_rgf_lesser_batched_z(ctypes.cast(descs, ctypes.c_void_p), len(descs), flags, dev.ptr(ws),
                                            ws.numel(), dev.ptr(status), dev.stream_handle(stream))
        _lib.check(rc, "sinvb_rgf_lesser_batched")
        (stream if stream is not None else torch.cuda.current_stream()).synchronize()
        st = status.cpu().numpy()
    if statuses is not None:
        statuses[:] = [int(x) for x in st]
    if check:
        bad = [k for k in range(len(st)) if st[k]]
        if bad:
            dev.raise_for_status(int(st[bad[0]]), "rgf_lesser_batched (instance %d)" % bad[0])
    res = []
    for (Gd, Gu, Gl, GLd, GLu), (A_diag, _, _) in zip(outs, instances):
        GLl = -GLu.conj().transpose(1, 2).contiguous()
        res.append(tuple(dev.to_output(t, A_diag) for t in (Gd, Gu, Gl, GLd, GLu, GLl)))
    del keep, moved
    return res


def rgf_greater_batched(instances, sigmas, team=None, check=True, stream=None, statuses=None):
    """``rgf_lesser_batched`` with the greater self-energies: G> = G Sigma> G^H
    for every instance (see ``rgf_greater``)."""
    return rgf_lesser_batched(instances, sigmas, team=team, check=check, stream=stream, statuses=statuses)
