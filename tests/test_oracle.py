"""The CPU oracle, pinned against the reference's own outputs (no GPU).

Fixtures: ``tests/golden/reference_outputs.npz`` written by
``tests/golden/make_golden.py`` from the reference ``rgf``
(``src/sinv/algorithms/rgf/rgf.py:17-64``) and ``bcr_serial``
(``src/sinv/algorithms/bcr/bcr_serial.py:19-62``) on the reference tests'
inputs (``SEED = 63`` banded generator) and on the seeded dominant matrix.
"""

import numpy as np
import pytest

from oracle import bcr_oracle, dense, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.utils import matu
from tests.golden.make_golden import (BCR_SIZES, BCR_VARIANTS, RGF_SIZES, RGF_VARIANTS, SEED,
                                      banded_case, checksum)

# Same numpy operations in the same order as the reference: agreement is at
# the level of BLAS rounding differences between runs (usually bit-exact).
PIN_TOL = 1e-13


def _rel(a, b):
    return dense.rel_fro(a, b)


@pytest.mark.parametrize("cplx,sym", RGF_VARIANTS)
@pytest.mark.parametrize("N,b", RGF_SIZES)
def test_rgf_oracle_matches_reference(golden, cplx, sym, N, b):
    A, (d, u, l) = banded_case(N, b, cplx, sym)
    key = f"rgf_c{int(cplx)}_s{int(sym)}_N{N}_b{b}"
    np.testing.assert_allclose(checksum(d, u, l), golden[key + "_in"], rtol=1e-14)
    Gd, Gu, Gl = rgf_oracle.rgf(d, u, l, sym_mat=sym)
    assert _rel(Gd, golden[key + "_d"]) <= PIN_TOL
    if N // b > 1:
        assert _rel(Gu, golden[key + "_u"]) <= PIN_TOL
        assert _rel(Gl, golden[key + "_l"]) <= PIN_TOL


@pytest.mark.parametrize("cplx,sym", BCR_VARIANTS)
@pytest.mark.parametrize("N,b", BCR_SIZES)
def test_bcr_oracle_matches_reference(golden, cplx, sym, N, b):
    A, _ = banded_case(N, b, cplx, sym)
    key = f"bcr_c{int(cplx)}_s{int(sym)}_N{N}_b{b}"
    np.testing.assert_allclose(checksum(A), golden[key + "_in"], rtol=1e-14)
    G = bcr_oracle.bcr_serial(A, b)
    gd, gu, gl = matu.convertDenseToBlkTridiag(G, b)
    assert _rel(gd, golden[key + "_d"]) <= PIN_TOL
    assert _rel(gu, golden[key + "_u"]) <= PIN_TOL
    assert _rel(gl, golden[key + "_l"]) <= PIN_TOL


def test_dominant_case_pins(golden):
    d, u, l = workloads.dominant(10, 32, seed=0)
    np.testing.assert_allclose(checksum(d, u, l), golden["dom_in"], rtol=1e-14)
    Gd, Gu, Gl = rgf_oracle.rgf(d, u, l)
    assert _rel(Gd, golden["dom_rgf_d"]) <= PIN_TOL
    assert _rel(Gu, golden["dom_rgf_u"]) <= PIN_TOL
    assert _rel(Gl, golden["dom_rgf_l"]) <= PIN_TOL
    Gd2, Gu2, _ = rgf_oracle.rgf(d, u, l, save_off_diag=False)
    assert _rel(Gd2, golden["dom_rgf_nooff_d"]) <= PIN_TOL
    assert bool(golden["dom_rgf_nooff_u_isnan"]) and np.all(np.isnan(Gu2))
    bd, bu, bl, blocks = bcr_oracle.bcr_blocks(d, u, l)
    assert _rel(bd, golden["dom_bcr_d"]) <= PIN_TOL
    # blocks of the production tree outside the tridiagonal, as in the dense reference G
    assert _rel(blocks[0, 3], golden["dom_bcr_g_0_3"]) <= PIN_TOL
    assert _rel(blocks[7, 3], golden["dom_bcr_g_7_3"]) <= PIN_TOL


@pytest.mark.parametrize("n,b", [(1, 4), (2, 3), (5, 4), (10, 32)])
@pytest.mark.parametrize("dtype", [np.complex128, np.float64])
def test_oracles_match_dense_inverse(n, b, dtype):
    d, u, l = workloads.dominant(n, b, seed=5, dtype=dtype)
    rd, ru, rl = dense.inv_selected(d, u, l)
    for Gd, Gu, Gl in (rgf_oracle.rgf(d, u, l), bcr_oracle.bcr_blocks(d, u, l)[:3]):
        assert _rel(Gd, rd) <= 1e-13
        if n > 1:
            assert _rel(Gu, ru) <= 1e-13
            assert _rel(Gl, rl) <= 1e-13


def test_pivot_free_gauss_jordan_matches_inverse():
    rng = np.random.default_rng(3)
    a = rng.random((12, 12)) + 1j * rng.random((12, 12)) + 12 * np.eye(12)
    inv, minp = rgf_oracle.gauss_jordan_inverse(a)
    assert _rel(inv, np.linalg.inv(a)) <= 1e-14
    assert minp > 0


def test_bcr_padding_and_schedule():
    # bcr_utils.py:17-40: pad to 2^p - 1 blocks
    assert [bcr_oracle.distance_to_power_of_two(n) for n in (1, 2, 3, 4, 7, 8, 10)] == [0, 1, 0, 3, 0, 7, 5]
    # bcr_utils.py:75-129 on a 15-block tree
    assert bcr_oracle.production_rows(2, 15) == ([7], [3, 11])
    assert bcr_oracle.production_rows(0, 15) == ([1, 3, 5, 7, 9, 11, 13], [0, 2, 4, 6, 8, 10, 12, 14])


def test_matu_generators_follow_reference_seed_semantics():
    # the legacy global seed: same seed, same matrix (matrices_utils.py:37-45)
    a = matu.generateRandomNumpyMat(5, True, True, SEED)
    b = matu.generateRandomNumpyMat(5, True, True, SEED)
    assert np.array_equal(a, b) and np.array_equal(a, a.T)
    band = matu.generateBandedDiagonalMatrix(8, 2, False, False, SEED)
    i, j = np.nonzero(band)
    assert np.all(np.abs(i - j) <= 2)
    d, u, l = matu.convertDenseToBlkTridiag(band, 2)
    assert np.array_equal(matu.convertBlkTridiagToDense(d, u, l), band)


def test_against_live_reference_when_present():
    """Re-run the pin against the reference sources themselves (this container only)."""
    import os
    ref = os.environ.get("SINV_REFERENCE")
    if not ref or not os.path.isdir(os.path.join(ref, "src", "sinv")):
        pytest.skip("SINV_REFERENCE does not name the reference sources")
    from tests.golden import make_golden
    rgf_mod, bcr_mod = make_golden.import_reference(ref)
    d, u, l = workloads.dominant(6, 5, seed=11)
    G = rgf_mod.rgf(make_golden.BlockTridiag(d.copy(), u.copy(), l.copy()), False)
    Gd, Gu, Gl = rgf_oracle.rgf(d, u, l)
    assert _rel(Gd, G.d) <= PIN_TOL and _rel(Gu, G.u) <= PIN_TOL and _rel(Gl, G.l) <= PIN_TOL
    A = dense.to_dense(d, u, l)
    assert _rel(bcr_oracle.bcr_serial(A, 5), bcr_mod.bcr_serial(A.copy(), 5)) <= PIN_TOL
