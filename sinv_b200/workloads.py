"""Seeded synthetic block-tridiagonal workloads.

Five workloads exercise the selected-inversion path:

* ``dominant``      -- uniform [0,1) real and imaginary parts for every block,
  ``2 N I`` added to each diagonal block (diagonally dominant).  n=10, b=32 is
  the CPU-sized case; n=64, b=256 the at-scale plain case.
* ``tight_binding`` -- ``A(E) = (E + i eta) I - H - Sigma`` for a real
  symmetric (hence Hermitian) tight-binding H: onsite blocks ``(R + R^T)/2``
  with ``R ~ N(0,1)``, couplings ``C ~ N(0, 0.5^2)`` above the diagonal and
  ``C^T`` below, ``Sigma = -0.1 i I`` on the first and last diagonal blocks.
* ``energy_batch``  -- 512 energies ``E ~ U[-2, 2]``, block counts
  ``U{16..128}``, block sizes from ``{64, 128, 256, 512}``, one H per instance.
* ``gradient_set``  -- 128 energies on one shared H, n=32, b=128.
* ``large_mixed``   -- 64 instances of n=256, b=1024.

The numpy generators are exact (seeded ``numpy.random.default_rng``) and feed
every parity test.  Instances too large to build on the host are generated on
the device by ``tight_binding_device`` with ``torch.Generator`` streams: same
distributions, different random numbers.
"""

import numpy as np

ETA = 1e-3
SIGMA_EDGE = 0.1
BLOCK_SIZES = (64, 128, 256, 512)


def dominant(n, b, seed=0, dtype=np.complex128):
    """Diagonally dominant random block-tridiagonal matrix (n blocks of b x b).

    Draw order: diag.re, diag.im, upper.re, upper.im, lower.re, lower.im, each
    ``rng.random``; then ``2 n b I`` is added to every diagonal block.
    Real dtypes use only the real draws (same stream positions).
    """
    rng = np.random.default_rng(seed)
    N = n * b

    def c(*shape):
        re = rng.random(shape)
        im = rng.random(shape)
        return re + 1j * im

    d = c(n, b, b) + 2 * N * np.eye(b)
    u = c(max(n - 1, 0), b, b)
    l = c(max(n - 1, 0), b, b)
    if not np.issubdtype(np.dtype(dtype), np.complexfloating):
        d, u, l = d.real, u.real, l.real
    return (np.ascontiguousarray(d, dtype=dtype), np.ascontiguousarray(u, dtype=dtype),
            np.ascontiguousarray(l, dtype=dtype))


def hamiltonian(n, b, seed):
    """Real symmetric tight-binding H as (onsite[n,b,b], coupling[n-1,b,b])."""
    rng = np.random.default_rng(seed)
    R = rng.standard_normal((n, b, b))
    onsite = 0.5 * (R + np.transpose(R, (0, 2, 1)))
    coupling = 0.5 * rng.standard_normal((max(n - 1, 0), b, b))
    return onsite, coupling


def tight_binding(n, b, energy, seed=None, H=None, eta=ETA, sigma=SIGMA_EDGE,
                  dtype=np.complex128):
    """``A(E) = (E + i eta) I - H - Sigma`` as block arrays (diag, upper, lower)."""
    onsite, coupling = H if H is not None else hamiltonian(n, b, seed)
    eye = np.eye(b)
    d = (energy + 1j * eta) * eye[None] - onsite
    d = d.astype(np.complex128)
    d[0] += 1j * sigma * eye
    d[-1] += 1j * sigma * eye
    u = -coupling.astype(np.complex128)
    l = -np.transpose(coupling, (0, 2, 1)).astype(np.complex128)
    return (np.ascontiguousarray(d, dtype=dtype), np.ascontiguousarray(u, dtype=dtype),
            np.ascontiguousarray(l, dtype=dtype))


def energy_batch_spec(count=512, seed=1, nmin=16, nmax=128, sizes=BLOCK_SIZES):
    """Per-instance (energy, n, b, hamiltonian seed) of the energy batch."""
    rng = np.random.default_rng(seed)
    E = rng.uniform(-2.0, 2.0, count)
    ns = rng.integers(nmin, nmax + 1, count)
    bs = rng.choice(np.asarray(sizes), count)
    return [(float(E[k]), int(ns[k]), int(bs[k]), 1000 + k) for k in range(count)]


def gradient_set_spec(count=128, n=32, b=128):
    """Energies and shared Hamiltonian seed of the differentiated workload."""
    E = np.random.default_rng(2).uniform(-2.0, 2.0, count)
    return [float(e) for e in E], n, b, 3


def bcr_batch_spec(count=256):
    """Per-instance (energy, n, b, hamiltonian seed) of the small-matrix BCR batch:
    n in [8, 64], b in {32, 64, 128}, the regime where one matrix's BCR levels
    hold too few block operations to fill the GPU."""
    return energy_batch_spec(count=count, seed=5, nmin=8, nmax=64, sizes=(32, 64, 128))


def large_mixed_spec(count=64, n=256, b=1024):
    """Per-instance (energy, n, b, hamiltonian seed) of the large mixed workload."""
    E = np.random.default_rng(1).uniform(-2.0, 2.0, count)
    return [(float(E[k]), n, b, 2000 + k) for k in range(count)]


def rgf_flops(n, b):
    """Canonical real-flop count of one selected inversion: 8 b^3 (8 (n-1) + n).

    8 (n-1) complex b^3 products at 8 real flops per complex multiply-add
    (the reference's schedule, ``src/sinv/algorithms/rgf/rgf.py:47-62``), plus
    n complex inversions counted as 8 b^3 each.  Fixed regardless of the
    schedule actually run.
    """
    return 8.0 * float(b) ** 3 * (8 * (n - 1) + n)


def rgf_bytes(n, b, itemsize=16):
    """Algorithmic HBM bytes: every input block read once, every output block
    written once, ``2 (3n - 2) b^2`` elements."""
    return 2.0 * (3 * n - 2) * b * b * itemsize


def tight_binding_device(n, b, energy, seed, device="cuda", eta=ETA, sigma=SIGMA_EDGE,
                         out=None):
    """Device-side tight-binding instance (same distributions as
    ``tight_binding``; random numbers from a seeded ``torch.Generator``).

    Returns complex128 ``(diag, upper, lower)`` tensors on ``device``; if
    ``out`` is given the three tensors are filled in place.
    """
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    if out is None:
        d = torch.empty((n, b, b), dtype=torch.complex128, device=device)
        u = torch.empty((max(n - 1, 0), b, b), dtype=torch.complex128, device=device)
        l = torch.empty((max(n - 1, 0), b, b), dtype=torch.complex128, device=device)
    else:
        d, u, l = out
    R = torch.randn((n, b, b), generator=g, dtype=torch.float64, device=device)
    onsite = 0.5 * (R + R.transpose(1, 2))
    del R
    eye = torch.eye(b, dtype=torch.float64, device=device)
    d.real.copy_(energy * eye - onsite)
    d.imag.copy_(eta * eye.expand(n, b, b))
    del onsite
    d[0].imag.add_(sigma * eye)
    d[-1].imag.add_(sigma * eye)
    if n > 1:
        C = 0.5 * torch.randn((n - 1, b, b), generator=g, dtype=torch.float64, device=device)
        u.real.copy_(-C)
        u.imag.zero_()
        l.real.copy_(-C.transpose(1, 2))
        l.imag.zero_()
    return d, u, l
