"""Post-processing output: the pressure-coefficient export of the response example.

``export_pressure_coefficients`` writes the format of ``export_pressure_coefficients`` in
examples/response/run.py:32-63 of the reference: for every cell (radial index outer, angular
index inner) four lines, one per cell vertex in the order (m, n), (m, n+1), (m+1, n+1),
(m+1, n), with the columns ``x z cp Re(dcp/dalpha) Im(dcp/dalpha)`` printed as ``%+.5e``
separated by single spaces, then an empty line; the file is gzip-compressed. Plotting (the
reference's gnuplot scripts) stays outside this library.
"""

from __future__ import annotations

import gzip
from pathlib import Path

import numpy as np


def format_pressure_coefficients(vertices: np.ndarray, pressure_coef: np.ndarray,
                                 pressure_coef_wrt_aoa: np.ndarray) -> bytes:
    """The uncompressed text of the export (see the module docstring)."""
    v = np.asarray(vertices, dtype=float)
    cp = np.asarray(pressure_coef, dtype=float)
    dcp = np.asarray(pressure_coef_wrt_aoa, dtype=complex)
    M, N = cp.shape
    if v.shape != (2, M + 1, N + 1) or dcp.shape != (M, N):
        raise ValueError("vertices must be (2, M+1, N+1) and the coefficients (M, N)")
    # corners (M, N, 4, 2) in the order (m, n), (m, n+1), (m+1, n+1), (m+1, n)
    corners = np.stack([v[:, :-1, :-1], v[:, :-1, 1:], v[:, 1:, 1:], v[:, 1:, :-1]], axis=-1)
    corners = np.moveaxis(corners, 0, -1)
    data = np.stack([cp, dcp.real, dcp.imag], axis=-1)               # (M, N, 3)
    rows = np.concatenate([corners, np.broadcast_to(data[:, :, None, :], (M, N, 4, 3))], axis=-1)
    line = "%+.5e %+.5e %+.5e %+.5e %+.5e\n"
    cell = line * 4 + "\n"
    flat = rows.reshape(M * N, 20)
    return "".join(cell % tuple(r) for r in flat.tolist()).encode()


def export_pressure_coefficients(file_name: str | Path, vertices: np.ndarray,
                                 pressure_coef: np.ndarray,
                                 pressure_coef_wrt_aoa: np.ndarray) -> None:
    """Writes the gzip-compressed export (examples/response/run.py:32-63)."""
    with gzip.open(file_name, mode="wb") as fh:
        fh.write(format_pressure_coefficients(vertices, pressure_coef, pressure_coef_wrt_aoa))
