"""GPU parity of the RGF selected inversion against the CPU oracle.

Tolerances: the plain FP64 path must match the reference rgf on the same
seeded inputs to <= 1e-12 relative Frobenius error per block family
(diagonal, upper, lower); on the reference tests' random banded matrices
(not diagonally dominant) the reference tests' own bar applies
(``np.allclose`` defaults, ``tests/rgf_tests/rgf_test.py:87-94``) together
with a relative bound.  Single precision results are compared at 1e-5.
"""

import numpy as np
import pytest

from oracle import dense, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import rgf
from tests.golden.make_golden import BlockTridiag, RGF_SIZES, banded_case

pytestmark = pytest.mark.gpu

TOL_PLAIN = 1e-12


def _rel(a, b):
    return dense.rel_fro(a, b)


def _check(G, R, tol):
    for x, r in zip(G, R):
        if r.size:
            assert _rel(x, r) <= tol, (_rel(x, r), tol)


@pytest.mark.parametrize("team", [None, "cta", "grid"])
def test_dominant_n10_b32_matches_reference(golden, team):
    d, u, l = workloads.dominant(10, 32, seed=0)
    G = rgf.rgf(d, u, l, team=team)
    ref = (golden["dom_rgf_d"], golden["dom_rgf_u"], golden["dom_rgf_l"])
    _check(G, ref, TOL_PLAIN)
    _check(G, dense.inv_selected(d, u, l), TOL_PLAIN)


def test_save_off_diag_false_leaves_nan(golden):
    d, u, l = workloads.dominant(10, 32, seed=0)
    Gd, Gu, Gl = rgf.rgf(d, u, l, save_off_diag=False)
    assert _rel(Gd, golden["dom_rgf_nooff_d"]) <= TOL_PLAIN
    assert np.all(np.isnan(Gu)) and np.all(np.isnan(Gl))


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("sym", [False, True])
@pytest.mark.parametrize("N,b", RGF_SIZES)
def test_reference_test_matrices(cplx, sym, N, b):
    """The reference tests' sizes and SEED=63 generator, all four variants."""
    A, (d, u, l) = banded_case(N, b, cplx, sym)
    G = rgf.rgf(d, u, l, sym)
    R = rgf_oracle.rgf(d, u, l, sym_mat=sym)
    X = dense.to_blocks(np.linalg.inv(A), b)
    for g, r, x in zip(G, R, X):
        if r.size:
            assert np.allclose(g, x)          # rgf_test.py:87-94 (diagonal asserted too)
            assert _rel(g, r) <= 1e-9


@pytest.mark.parametrize("n,b", [(1, 1), (1, 5), (2, 1), (3, 7), (5, 33), (4, 64), (3, 65), (3, 100), (2, 130)])
@pytest.mark.parametrize("dtype", [np.complex128, np.float64])
def test_ragged_and_edge_sizes(n, b, dtype):
    d, u, l = workloads.dominant(n, b, seed=n * 1000 + b, dtype=dtype)
    for team in (None, "grid"):
        G = rgf.rgf(d, u, l, team=team)
        _check(G, rgf_oracle.rgf(d, u, l), TOL_PLAIN)


@pytest.mark.parametrize("dtype,tol", [(np.complex64, 1e-5), (np.float32, 1e-5)])
def test_single_precision_follows_input_dtype(dtype, tol):
    d, u, l = workloads.dominant(6, 24, seed=4, dtype=dtype)
    G = rgf.rgf(d, u, l)
    assert all(g.dtype == dtype for g in G)
    wide = np.complex128 if dtype == np.complex64 else np.float64
    R = rgf_oracle.rgf(d.astype(wide), u.astype(wide), l.astype(wide))
    _check(G, R, tol)


def test_container_interface_matches_reference_kind(golden):
    d, u, l = workloads.dominant(10, 32, seed=0)
    A = BlockTridiag(d.copy(), u.copy(), l.copy())
    G = rgf.rgf(A)
    assert isinstance(G, BlockTridiag)
    assert _rel(G.d, golden["dom_rgf_d"]) <= TOL_PLAIN
    assert _rel(G.u, golden["dom_rgf_u"]) <= TOL_PLAIN
    assert np.array_equal(A.d, d)        # the input is not modified (rgf.py:41 copies)
    Gn = rgf.rgf(A, False, False)
    assert np.all(np.isnan(Gn.u)) and np.all(np.isnan(Gn.l))


def test_torch_inputs_stay_on_device():
    import torch
    d, u, l = workloads.dominant(4, 16, seed=2)
    td, tu, tl = (torch.from_numpy(x).cuda() for x in (d, u, l))
    G = rgf.rgf(td, tu, tl)
    assert all(g.is_cuda for g in G)
    _check([g.cpu().numpy() for g in G], rgf_oracle.rgf(d, u, l), TOL_PLAIN)


def test_zero_pivot_raises_linalg_error():
    d, u, l = workloads.dominant(3, 4, seed=1)
    d[1] = 0.0
    u[0] = 0.0   # S_1 = A_11 - A_10 g_0 A_01 = 0: a zero pivot in block 1
    with pytest.raises(np.linalg.LinAlgError):
        rgf.rgf(d, u, l)


@pytest.mark.parametrize("n,b", [(64, 256)])
def test_at_scale_plain_matches_oracle(n, b):
    d, u, l = workloads.dominant(n, b, seed=0)
    G = rgf.rgf(d, u, l)
    _check(G, rgf_oracle.rgf(d, u, l), TOL_PLAIN)


@pytest.mark.parametrize("n,b,team", [(1, 8, None), (2, 16, None), (7, 33, None), (6, 70, "grid"), (4, 130, None)])
def test_overwrite_a_in_place(n, b, team):
    import torch
    d, u, l = workloads.dominant(n, b, seed=9 + n)
    td, tu, tl = (torch.from_numpy(x).cuda() for x in (d, u, l))
    G = rgf.rgf_blocks(td, tu, tl, overwrite_a=True, team=team)
    assert G[0].data_ptr() == td.data_ptr()
    _check([g.cpu().numpy() for g in G], rgf_oracle.rgf(d, u, l), TOL_PLAIN)
