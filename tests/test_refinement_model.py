"""Why the mixed-precision path has no refinement step on G_ii (CPU, numpy).

The mixed path computes every block product of the RGF sweeps to about
3e-14 relative error (int8 Ozaki digits) and every block inverse in FP64.
This test models that on the CPU: the 6-product RGF schedule of the library
(``X_i = g_i A_{i,i+1}``, ``P_{i+1} = A_{i+1,i} g_i`` kept from the forward
sweep) with a relative perturbation of 3e-14 on each product, against the
dense FP64 inverse.  It then applies the one refinement step that the
selected blocks allow, an FP64 residual correction of each diagonal block

    R_i  = I - A_{i,i-1} G_{i-1,i} - A_ii G_ii - A_{i,i+1} G_{i+1,i}
    G_ii <- G_ii + G_ii R_i

(and its column form), and shows that it leaves the error where it was: the
error is accumulated along the chain of Schur complements, and the Newton
step X + X (I - A X) of the whole inverse needs the full block column i of
G to form its diagonal block, which a selected inversion never holds.
"""

import numpy as np
import pytest

from oracle import dense
from sinv_b200 import workloads

EPS = 3e-14


def _rgf6(d, u, l, rng):
    """The library's product schedule; each product perturbed by EPS when rng is given."""
    def mm(a, b):
        c = a @ b
        if rng is None:
            return c
        s = np.linalg.norm(c) / np.sqrt(c.size)
        return c + EPS * s * (rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)) / np.sqrt(2)

    n = d.shape[0]
    g, X, P = [None] * n, [None] * n, [None] * n
    g[0] = np.linalg.inv(d[0])
    for i in range(1, n):
        X[i - 1] = mm(g[i - 1], u[i - 1])
        P[i] = mm(l[i - 1], g[i - 1])
        g[i] = np.linalg.inv(d[i] - mm(P[i], u[i - 1]))
    Gd, Gu, Gl = [None] * n, [None] * (n - 1), [None] * (n - 1)
    Gd[n - 1] = g[n - 1]
    for i in range(n - 2, -1, -1):
        Gl[i] = -mm(Gd[i + 1], P[i + 1])
        Gu[i] = -mm(X[i], Gd[i + 1])
        Gd[i] = g[i] - mm(X[i], Gl[i])
    return np.array(Gd), np.array(Gu), np.array(Gl)


def _refine(d, u, l, Gd, Gu, Gl, column=False):
    n, b = d.shape[0], d.shape[1]
    out = Gd.copy()
    for i in range(n):
        if column:   # (G A)_ii = I
            R = np.eye(b) - Gd[i] @ d[i]
            if i > 0:
                R -= Gl[i - 1] @ u[i - 1]
            if i < n - 1:
                R -= Gu[i] @ l[i]
            out[i] = Gd[i] + R @ Gd[i]
        else:        # (A G)_ii = I
            R = np.eye(b) - d[i] @ Gd[i]
            if i > 0:
                R -= l[i - 1] @ Gu[i - 1]
            if i < n - 1:
                R -= u[i] @ Gl[i]
            out[i] = Gd[i] + Gd[i] @ R
    return out


@pytest.mark.parametrize("n,b,energy", [(12, 24, 0.3), (16, 32, -1.1), (24, 16, 1.7)])
def test_local_refinement_of_G_ii_does_not_reduce_the_mixed_error(n, b, energy):
    d, u, l = workloads.tight_binding(n, b, energy, seed=7)
    exact = dense.inv_selected(d, u, l)[0]
    fp64 = _rgf6(d, u, l, None)
    mixed = _rgf6(d, u, l, np.random.default_rng(n * b))
    e64 = dense.rel_fro(fp64[0], exact)
    emix = dense.rel_fro(mixed[0], exact)
    assert emix > 5 * e64, (emix, e64)   # the perturbed products dominate the error
    for column in (False, True):
        eref = dense.rel_fro(_refine(d, u, l, *mixed, column=column), exact)
        assert 0.9 * emix <= eref <= 1.1 * emix, (column, emix, eref)
