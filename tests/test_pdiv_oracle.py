"""The PDIV oracle pinned on the reference's own outputs (CPU).

``tests/golden/pdiv_outputs.npz`` holds the reference ``pdiv_localmap``
(``src/sinv/algorithms/pdiv/pdiv_localmap.py:27-91``) run on 2, 4 and 8
processes over the reference test's matrices
(``tests/pdiv_tests/pdiv_test.py:45-56``, SEED=63 banded generator, each
process given its partition and the bridges as the test does) and on a
seeded dominant matrix with 2, 4, 8 and 16 processes; the restatement must
reproduce them bit for bit.
"""

import os

import numpy as np
import pytest

from oracle import dense, pdiv_oracle
from sinv_b200 import workloads
from tests.golden.make_golden import PDIV_SIZES, PDIV_VARIANTS, banded_case, checksum

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def pdiv_golden():
    return np.load(os.path.join(HERE, "golden", "pdiv_outputs.npz"))


CASES = [(c, s, N, b, P) for c, s in PDIV_VARIANTS for N, b in PDIV_SIZES for P in (2, 4, 8) if N // b >= P]


@pytest.mark.parametrize("cplx,sym,N,b,P", CASES)
def test_oracle_is_bitwise_reference(pdiv_golden, cplx, sym, N, b, P):
    key = f"pdiv_c{int(cplx)}_s{int(sym)}_N{N}_b{b}_P{P}"
    A, (d, u, l) = banded_case(N, b, cplx, sym)
    assert np.array_equal(checksum(A), pdiv_golden[key + "_in"])
    G = pdiv_oracle.pdiv(d, u, l, P)
    for g, s in zip(G, ("_d", "_u", "_l")):
        assert np.array_equal(g, pdiv_golden[key + s])
    R = dense.inv_selected(d, u, l)
    assert all(np.allclose(g, r) for g, r in zip(G, R))   # pdiv_test.py:134-136


@pytest.mark.parametrize("P", [1, 2, 4, 8, 16])
def test_oracle_dominant_processes(pdiv_golden, P):
    d, u, l = workloads.dominant(16, 12, seed=0)
    assert np.array_equal(checksum(d, u, l), pdiv_golden["dom_pdiv_in"])
    G = pdiv_oracle.pdiv(d, u, l, P)
    if P > 1:
        for g, s in zip(G, ("_d", "_u", "_l")):
            assert np.array_equal(g, pdiv_golden[f"dom_pdiv_P{P}" + s])
    for g, r in zip(G, dense.inv_selected(d, u, l)):
        assert dense.rel_fro(g, r) <= 1e-13


def test_limits():
    with pytest.raises(ValueError):
        pdiv_oracle.check(12, 3)     # not a power of two
    with pytest.raises(ValueError):
        pdiv_oracle.check(3, 4)      # fewer blocks than processes
    assert pdiv_oracle.middle(0, 1) == 0 and pdiv_oracle.middle(0, 3) == 1 and pdiv_oracle.middle(4, 7) == 5
