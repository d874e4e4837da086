"""CPU oracle for the selected-inversion path (test infrastructure only).

This package restates, in plain numpy, the reference algorithms that the
CUDA library replaces:

* ``rgf_oracle.rgf``        follows ``src/sinv/algorithms/rgf/rgf.py:17-64``
* ``bcr_oracle.bcr_serial`` follows ``src/sinv/algorithms/bcr/bcr_serial.py:19-467``
  with ``src/sinv/algorithms/bcr/bcr_utils.py:17-129``
* ``dense.inv_selected``    is the reference tests' own oracle: a dense
  ``numpy.linalg.inv`` cut into block-tridiagonal pieces
  (``tests/rgf_tests/rgf_test.py:81``, ``tests/bcr_tests/bcr_serial_test.py:68``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this package, and only as
the checker or as the timed CPU baseline.  The shipped library never calls it:
``sinv_b200`` raises when its CUDA extension is missing instead of falling
back to anything here.

Parity pin: the restatements are checked against outputs of the reference
itself (imported from its sources with two import shims), committed as
fixtures under ``tests/golden/`` by ``tests/golden/make_golden.py``.
"""
