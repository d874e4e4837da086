"""The PSR oracle pinned on the reference's own outputs (CPU).

``tests/golden/psr_outputs.npz`` holds the reference ``psr_seqsolve``
(``src/sinv/algorithms/psr/psr_seqsolve.py:20-73``) run on 3 and 4 partitions
over the reference test's matrices (``tests/psr_tests/psr_test.py:42-52``,
SEED=63 banded generator) and on a seeded dominant matrix with 3, 4 and 8
partitions; the restatement must reproduce them bit for bit.
"""

import os

import numpy as np
import pytest

from oracle import dense, psr_oracle
from sinv_b200 import workloads
from tests.golden.make_golden import PSR_SIZES, PSR_VARIANTS, banded_case, checksum

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def psr_golden():
    return np.load(os.path.join(HERE, "golden", "psr_outputs.npz"))


CASES = [(c, s, N, b, P) for c, s in PSR_VARIANTS for N, b in PSR_SIZES for P in (3, 4) if N // b >= 3 * P]


@pytest.mark.parametrize("cplx,sym,N,b,P", CASES)
def test_oracle_is_bitwise_reference(psr_golden, cplx, sym, N, b, P):
    key = f"psr_c{int(cplx)}_s{int(sym)}_N{N}_b{b}_P{P}"
    A, (d, u, l) = banded_case(N, b, cplx, sym)
    assert np.array_equal(checksum(A), psr_golden[key + "_in"])
    G = psr_oracle.psr(d, u, l, P)
    for g, s in zip(G, ("_d", "_u", "_l")):
        assert np.array_equal(g, psr_golden[key + s])
    R = dense.inv_selected(d, u, l)
    assert all(np.allclose(g, r) for g, r in zip(G, R))   # psr_test.py:67-70


@pytest.mark.parametrize("P", [3, 4, 8])
def test_oracle_dominant_partitions(psr_golden, P):
    d, u, l = workloads.dominant(24, 16, seed=0)
    assert np.array_equal(checksum(d, u, l), psr_golden["dom_psr_in"])
    G = psr_oracle.psr(d, u, l, P)
    for g, s in zip(G, ("_d", "_u", "_l")):
        assert np.array_equal(g, psr_golden[f"dom_psr_P{P}" + s])
    for g, r in zip(G, dense.inv_selected(d, u, l)):
        assert dense.rel_fro(g, r) <= 1e-13


def test_partitions_and_limits():
    assert psr_oracle.divide(9, 3) == ([0, 3, 6], [3, 3, 3])
    assert psr_oracle.divide(14, 4) == ([0, 5, 8, 11], [5, 3, 3, 3])
    assert psr_oracle.reduced_rows(*psr_oracle.divide(14, 4)) == [4, 5, 7, 8, 10, 11]
    with pytest.raises(ValueError):
        psr_oracle.check(8, 3)
    with pytest.raises(ValueError):
        psr_oracle.check(12, 2)
