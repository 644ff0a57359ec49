"""The pressure-coefficient export against the output of the reference's own export function
(CPU)."""

from __future__ import annotations

import gzip
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).parent / "golden"


def test_export_matches_reference_output(tmp_path, golden_grids, reference_8x9):
    from pyeulerale_b200.export import export_pressure_coefficients, format_pressure_coefficients

    args = (golden_grids["naca0012_8x9"], reference_8x9["cp"], reference_8x9["cp_wrt/result"])
    expected = (GOLDEN / "cp_export_8x9.txt").read_bytes()
    assert format_pressure_coefficients(*args) == expected
    export_pressure_coefficients(tmp_path / "cp.gz", *args)
    assert gzip.decompress((tmp_path / "cp.gz").read_bytes()) == expected


def test_export_rejects_mismatched_shapes(golden_grids):
    import pytest

    from pyeulerale_b200.export import format_pressure_coefficients

    with pytest.raises(ValueError):
        format_pressure_coefficients(golden_grids["naca0012_8x9"], np.zeros((3, 3)),
                                     np.zeros((3, 3), dtype=complex))
