"""O-grid input: the reference's PLOT3D reader and a seeded NACA-00tt O-grid generator.

``read_plot3d`` follows ``SpatialDiscretization._read_grid`` (src/py_euler_ale/core.py:213-227):
a single-block 2D PLOT3D text file whose second line holds the radial and angular point counts,
followed by all x then all z coordinates with the radial index running fastest in the file
(C-order reshape to ``(2, radial_pts, angular_pts)``).

``naca_ogrid`` builds the synthetic benchmark grids (the reference ships fixed grids only):
a symmetric NACA 4-digit section with cosine clustering, ordered trailing edge -> lower side ->
leading edge -> upper side and closed (first angular column equals the last), geometric radial
stretching from a given first spacing out to a far-field circle, blended by linear transfinite
interpolation. The thickness polynomial uses the closed-trailing-edge last coefficient
(-0.1036) so the surface closes exactly.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

NUM_DIM = 2
NUM_VAR = 4
HEAT_RATIO = 1.4


def read_plot3d(grid_file: str | Path) -> np.ndarray:
    """Reads the vertex coordinates ``(2, radial_pts, angular_pts)`` (Fortran order, float64)."""
    with open(grid_file) as fh:
        fh.readline()
        radial_pts, angular_pts = (int(v) for v in fh.readline().split())
        values = np.array(fh.read().split(), dtype=np.float64)
    if values.size != NUM_DIM * radial_pts * angular_pts:
        raise ValueError(f"{grid_file}: expected {NUM_DIM * radial_pts * angular_pts} values, "
                         f"got {values.size}")
    return np.asfortranarray(values.reshape((NUM_DIM, radial_pts, angular_pts)))


def write_plot3d(grid_file: str | Path, vertices: np.ndarray) -> None:
    """Writes vertices ``(2, radial_pts, angular_pts)`` in the layout ``read_plot3d`` reads."""
    v = np.asarray(vertices, dtype=np.float64)
    with open(grid_file, "w") as fh:
        fh.write("1\n")
        fh.write(f"{v.shape[1]} {v.shape[2]}\n")
        np.savetxt(fh, v.reshape(-1), fmt="%.17e")


def naca_thickness(x: np.ndarray, t: float) -> np.ndarray:
    """Half thickness of a symmetric NACA 4-digit section of unit chord (closed trailing edge)."""
    return 5.0 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x**2 + 0.2843 * x**3
                      - 0.1036 * x**4)


def _stretching(first: float, total: float, cells: int) -> np.ndarray:
    """Normalised geometric distribution s_0 = 0 < ... < s_cells = 1 with first step `first/total`."""
    h = first / total
    if h * cells >= 1.0:
        return np.linspace(0.0, 1.0, cells + 1)
    lo, hi = 1.0 + 1e-12, 2.0
    while (h * (hi**cells - 1) / (hi - 1)) < 1.0:
        hi *= 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if h * (r**cells - 1) / (r - 1) > 1.0:
            hi = r
        else:
            lo = r
    r = 0.5 * (lo + hi)
    s = np.concatenate(([0.0], np.cumsum(h * r ** np.arange(cells))))
    return s / s[-1]


def naca_ogrid(radial_pts: int, angular_pts: int, thickness: float = 0.12, chord: float = 1.0,
               far_radius: float = 20.0, first_spacing: float = 0.01) -> np.ndarray:
    """NACA-00tt O-grid vertices ``(2, radial_pts, angular_pts)`` in Fortran order.

    ``far_radius`` and ``first_spacing`` are in grid units (multiply by the chord for values
    given in chords). The far-field circle is centred at mid-chord.
    """
    theta = np.linspace(0.0, 2.0 * np.pi, angular_pts)
    xs = 0.5 * (1.0 + np.cos(theta))              # 1 -> 0 -> 1: TE, LE, TE (cosine clustering)
    zs = naca_thickness(np.clip(xs, 0.0, 1.0), thickness)
    zs = np.where(theta <= np.pi, -zs, zs)        # lower side first, then upper side
    surf = np.stack([xs * chord, zs * chord])
    surf[:, -1] = surf[:, 0]
    far = np.stack([0.5 * chord + far_radius * np.cos(theta), -far_radius * np.sin(theta)])
    far[:, -1] = far[:, 0]
    s = _stretching(first_spacing, far_radius, radial_pts - 1)
    grid = (1.0 - s)[None, :, None] * surf[:, None, :] + s[None, :, None] * far[:, None, :]
    return np.asfortranarray(grid)


def free_stream_state(mach: float, aoa_deg: float) -> np.ndarray:
    """Free-stream conserved state (make_free_stream_state, src/spatial_discretization.f90:250-259)."""
    speed = mach * np.sqrt(HEAT_RATIO)
    a = 0.0174532925199432957692369 * aoa_deg
    return np.array([1.0, speed * np.cos(a), speed * np.sin(a),
                     1.0 / (HEAT_RATIO - 1.0) + speed * speed / 2.0])


def perturbed_states(M: int, N: int, mach: float, aoa_deg: float, rel: float,
                     rng: np.random.Generator) -> np.ndarray:
    """Free stream times (1 + rel * N(0, 1)) componentwise, shape (4, M, N), Fortran order."""
    fs = free_stream_state(mach, aoa_deg)
    U = fs[:, None, None] * (1.0 + rel * rng.standard_normal((NUM_VAR, M, N)))
    return np.asfortranarray(U)


def smooth_velocities(vertices: np.ndarray, rng: np.random.Generator, modes: int = 8,
                      amplitude: float = 0.05) -> np.ndarray:
    """Seeded smooth vertex velocity field: `modes` angular Fourier modes with radial decay."""
    _, mp, npts = vertices.shape
    n = np.arange(npts) / (npts - 1) * 2.0 * np.pi
    m = np.arange(mp) / max(mp - 1, 1)
    V = np.zeros((NUM_DIM, mp, npts))
    for d in range(NUM_DIM):
        for k in range(1, modes + 1):
            a, b = rng.standard_normal(2) / k
            V[d] += (a * np.cos(k * n) + b * np.sin(k * n))[None, :] * np.exp(-3.0 * m)[:, None]
    V[:, :, -1] = V[:, :, 0]
    return np.asfortranarray(amplitude * V)
