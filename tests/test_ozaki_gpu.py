"""The mixed-precision complex GEMM on the int8 tensor cores (tcgen05 kind::i8,
Ozaki splitting) against an FP64 product.

Error model: with S digits of 7 bits (the first 6) per value, the relative
error of each entry against |A| |B| is below ~2^-(7S-2) * sqrt(2K); the tests
require the measured relative Frobenius error to fall by at least ~2^-5 per
extra digit and to be at FP64 level (<= 1e-13) with 7 digits.  Inputs that
are exact in few digits give exact products.
"""

import ctypes

import numpy as np
import pytest
import torch

from sinv_b200 import _lib

pytestmark = pytest.mark.gpu


def ozaki(A, B, digits, alpha=1.0, beta=0.0, D=None):
    lib = _lib.load()
    M, K = A.shape
    N = B.shape[1]
    C = torch.empty((M, N), dtype=torch.complex128, device="cuda")
    ws = torch.empty(lib.sinvb_zgemm_ozaki_workspace_size(M, N, K, digits), dtype=torch.uint8, device="cuda")
    rc = lib.sinvb_zgemm_ozaki(M, N, K, alpha, A.data_ptr(), K, B.data_ptr(), N, beta,
                               D.data_ptr() if D is not None else None, N, C.data_ptr(), N, digits,
                               ws.data_ptr(), ws.numel(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, _lib.status_string(rc)
    st = ctypes.c_int(-1)
    assert lib.sinvb_workspace_status(ws.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                      ctypes.byref(st)) == 0
    assert st.value == 0, _lib.status_string(st.value)
    return C


def rand(shape, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    re = torch.randn(shape, generator=g, dtype=torch.float64, device="cuda")
    im = torch.randn(shape, generator=g, dtype=torch.float64, device="cuda")
    return torch.complex(re, im)


def rel(a, b):
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


@pytest.mark.parametrize("M,N,K", [(64, 64, 64), (128, 64, 32), (100, 70, 33), (256, 256, 256), (512, 512, 512),
                                   (5, 3, 7)])
def test_error_falls_with_digits(M, N, K):
    A, B = rand((M, K), 1), rand((K, N), 2)
    ref = A @ B
    errs = [rel(ozaki(A, B, s), ref) for s in (3, 4, 5, 6, 7)]
    for e1, e2 in zip(errs, errs[1:]):
        assert e2 <= e1 / 30 or e2 <= 1e-14, errs
    assert errs[-1] <= 1e-13, errs
    assert errs[3] <= 1e-10, errs


def test_exact_for_short_inputs():
    g = torch.Generator(device="cpu").manual_seed(3)
    A = torch.complex(torch.randint(-8, 8, (96, 80), generator=g).double(),
                      torch.randint(-8, 8, (96, 80), generator=g).double()).cuda()
    B = torch.complex(torch.randint(-8, 8, (80, 72), generator=g).double(),
                      torch.randint(-8, 8, (80, 72), generator=g).double()).cuda()
    assert torch.equal(ozaki(A, B, 3), A @ B)


def test_alpha_beta_addend_and_scaling_spread():
    A, B, D = rand((128, 96), 4), rand((96, 64), 5), rand((128, 64), 6)
    A[3] *= 1e12        # rows / columns of very different magnitude
    B[:, 7] *= 1e-9
    ref = 0.5 * D - 2.0 * (A @ B)
    C = ozaki(A, B, 7, alpha=-2.0, beta=0.5, D=D)
    assert rel(C, ref) <= 1e-12
    # each row keeps its own relative accuracy
    assert rel(C[3], ref[3]) <= 1e-12 and rel(C[5], ref[5]) <= 1e-12
