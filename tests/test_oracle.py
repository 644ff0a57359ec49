"""The CPU oracle, pinned against the reference's own tests and golden data (CPU only).

* When the reference sources are present (development checkout), the reference's 20 unit tests
  (``tests/test_linearization.py``) run unchanged on the reference's own class with the oracle
  as its native module.
* Always: the oracle reproduces the committed fixtures of the reference class
  (``tests/golden/reference_8x9.npz``) and satisfies properties the reference relies on.
* With ``PYEULERALE_SLOW=1`` and the reference present: one CI example end to end against its
  committed golden output (byte for byte).
"""

from __future__ import annotations

import os
import unittest

import numpy as np
import pytest

from oracle import refload

HAVE_REF = refload.reference_available()


@pytest.mark.skipif(not HAVE_REF, reason="reference sources not present")
def test_reference_unit_tests_pass_on_oracle():
    refload.load_reference_package()
    import importlib.util

    path = refload.DEFAULT_REFERENCE / "tests" / "test_linearization.py"
    spec = importlib.util.spec_from_file_location("ref_test_linearization", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    suite = unittest.defaultTestLoader.loadTestsFromTestCase(mod.TestJacobi)
    assert suite.countTestCases() == 20
    result = unittest.TextTestRunner(verbosity=0).run(suite)
    assert result.wasSuccessful(), [str(f[0]) for f in result.failures + result.errors]


def _ref_case(reference_8x9, golden_grids):
    X = np.asfortranarray(golden_grids["naca0012_8x9"], dtype=complex)
    U = np.asfortranarray(reference_8x9["states"], dtype=complex)
    return X, np.zeros_like(X), U


def test_oracle_reproduces_reference_fixture(oracle, reference_8x9, golden_grids):
    X, V, U = _ref_case(reference_8x9, golden_grids)
    M, N = U.shape[1:]
    oracle.aoa[...] = 1.25
    R = np.asfortranarray(np.zeros((4, M, N), dtype=complex))
    oracle.compute_odes(0.5, X, V, U, R)
    np.testing.assert_array_equal(R.real, reference_8x9["odes"])
    J = np.asfortranarray(np.zeros((4, 4, M, N, 9)))
    oracle.compute_odes_wrt_states(0.5, X, V, U, J)
    np.testing.assert_array_equal(J, reference_8x9["odes_wrt_states"])


def test_convert_matches_dense_definition(oracle, reference_8x9):
    """O(nnz) BSR conversion == the reference's O((MN)^2) scan semantics (f90:765-814)."""
    J = np.asfortranarray(reference_8x9["odes_wrt_states"])
    M, N = J.shape[2], J.shape[3]
    nnzb = (9 * M - 6) * N
    data = np.asfortranarray(np.zeros((4, 4, nnzb)))
    idx = np.zeros(nnzb, dtype=np.int32)
    ptr = np.zeros(M * N + 1, dtype=np.int32)
    oracle.convert_odes_wrt_states(J, data, idx, ptr)
    # the reference's double loop, restated literally
    e_data, e_idx, e_ptr, p = [], [], [1], 1
    for n_row in range(1, N + 1):
        for m_row in range(1, M + 1):
            col = 0
            for n_col in range(1, N + 1):
                for m_col in range(1, M + 1):
                    col += 1
                    if m_col == m_row and (n_col - n_row + 1) % N == 0:
                        k = 2
                    elif m_col == m_row and (n_col - n_row + 2) % N == 0:
                        k = 3
                    elif m_col == m_row - 1 and n_col == n_row:
                        k = 6
                    elif m_col == m_row - 2 and n_col == n_row:
                        k = 7
                    elif m_col == m_row and n_col == n_row:
                        k = 1
                    elif m_col == m_row + 1 and n_col == n_row:
                        k = 8
                    elif m_col == m_row + 2 and n_col == n_row:
                        k = 9
                    elif m_col == m_row and (n_col - n_row - 1) % N == 0:
                        k = 4
                    elif m_col == m_row and (n_col - n_row - 2) % N == 0:
                        k = 5
                    else:
                        continue
                    e_data.append(J[:, :, m_row - 1, n_row - 1, k - 1])
                    e_idx.append(col)
                    p += 1
            e_ptr.append(p)
    np.testing.assert_array_equal(idx, e_idx)
    np.testing.assert_array_equal(ptr, e_ptr)
    np.testing.assert_array_equal(np.moveaxis(data, -1, 0), np.array(e_data))


def test_free_stream_is_steady_on_uniform_grid(oracle, golden_grids):
    """Free stream on a static grid has a residual at round-off level away from the wall."""
    X = np.asfortranarray(golden_grids["naca0012_8x9"], dtype=complex)
    M, N = X.shape[1] - 1, X.shape[2] - 1
    U = np.asfortranarray(np.zeros((4, M, N), dtype=complex))
    oracle.aoa[...] = 0.0
    oracle.set_free_stream_state(0.5, U)
    R = np.asfortranarray(np.zeros((4, M, N), dtype=complex))
    oracle.compute_odes(0.5, X, np.zeros_like(X), U, R)
    assert np.all(np.isfinite(R))
    assert np.max(np.abs(R[:, M - 1, :])) < 1e-10 * np.max(np.abs(U))


@pytest.mark.skipif(not (HAVE_REF and os.environ.get("PYEULERALE_SLOW")),
                    reason="set PYEULERALE_SLOW=1 with the reference present")
def test_gain_example_golden_output(tmp_path):
    import contextlib
    import io
    import runpy
    import shutil
    import sys

    refload.load_reference_package()
    root = refload.DEFAULT_REFERENCE
    work = tmp_path / "examples" / "gain"
    work.mkdir(parents=True)
    (tmp_path / "examples" / "grids").symlink_to(root / "examples" / "grids")
    shutil.copy(root / "examples" / "gain" / "run.py", work / "run.py")
    cwd, argv = os.getcwd(), sys.argv
    buf = io.StringIO()
    try:
        os.chdir(work)
        sys.argv = ["run.py", "../grids/naca0012_129x129.plot3d", "10.", "0.1"]
        with contextlib.redirect_stdout(buf):
            runpy.run_path("run.py", run_name="__main__")
    finally:
        os.chdir(cwd)
        sys.argv = argv
    golden = (refload.DEFAULT_REFERENCE / "examples" / "gain" / "Ma0p10.out").read_text()
    assert buf.getvalue() == golden
