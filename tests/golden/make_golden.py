"""Generates the committed golden fixtures from the PyEulerALE reference checkout.

Run with ``PYEULERALE_REFERENCE`` naming a checkout of the reference sources:

    PYEULERALE_REFERENCE=<reference checkout> python tests/golden/make_golden.py

It writes, next to this script:

* ``grids.npz`` -- the reference's shipped grids used by its tests and CI examples
  (``tests/naca0012_8x9.plot3d``, ``examples/grids/naca0004_129x129.plot3d``,
  ``examples/grids/naca0012_129x129.plot3d``) as float64 vertex arrays;
* ``*.out`` -- the reference's committed golden outputs of its CI examples
  (``examples/response/Ma0p05.out``, ``Ma0p5.out``, ``examples/gain/Ma0p10.out``,
  ``Ma0p50.out``), the end-to-end pins of the residual history, transfer functions and gains;
* ``cp_export_8x9.txt`` -- the uncompressed output of the reference's own
  ``export_pressure_coefficients`` (examples/response/run.py:32-63, taken from that file
  unmodified) for the 8x9 state below, its pressure coefficients and their tangent along a
  seeded direction;
* ``reference_8x9.npz`` -- outputs of the reference's own Python class
  (``src/py_euler_ale/core.py``, unmodified) running on the C++ oracle for the state of its
  unit tests (``tests/test_linearization.py:26-33``: seed 1, 0.5 % noise): residual, forces,
  every Jacobian, and the 13 second-order routines (the reference's finite-difference
  formulas) for seeded directions.
"""

from __future__ import annotations

import ast
import gzip
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle.refload import DEFAULT_REFERENCE, load_reference_package  # noqa: E402

GRIDS = {
    "naca0012_8x9": "tests/naca0012_8x9.plot3d",
    "naca0004_129x129": "examples/grids/naca0004_129x129.plot3d",
    "naca0012_129x129": "examples/grids/naca0012_129x129.plot3d",
}
OUTS = {
    "response_Ma0p05.out": "examples/response/Ma0p05.out",
    "response_Ma0p5.out": "examples/response/Ma0p5.out",
    "gain_Ma0p10.out": "examples/gain/Ma0p10.out",
    "gain_Ma0p50.out": "examples/gain/Ma0p50.out",
}

SECOND_ORDER = [
    ("compute_odes_wrt_states_inner_product_wrt_mach", "odes", "states"),
    ("compute_odes_wrt_states_inner_product_wrt_states", "odes", "states"),
    ("compute_odes_wrt_states_inner_product_wrt_vertices", "odes", "states"),
    ("compute_odes_wrt_vertices_inner_product_wrt_mach", "odes", "vertices"),
    ("compute_odes_wrt_vertices_inner_product_wrt_states", "odes", "vertices"),
    ("compute_odes_wrt_vertices_inner_product_wrt_vertices", "odes", "vertices"),
    ("compute_odes_wrt_velocities_inner_product_wrt_mach", "odes", "velocities"),
    ("compute_odes_wrt_velocities_inner_product_wrt_states", "odes", "velocities"),
    ("compute_odes_wrt_velocities_inner_product_wrt_vertices", "odes", "velocities"),
    ("compute_forces_wrt_states_inner_product_wrt_states", "forces", "states"),
    ("compute_forces_wrt_states_inner_product_wrt_vertices", "forces", "states"),
    ("compute_forces_wrt_vertices_inner_product_wrt_states", "forces", "vertices"),
    ("compute_forces_wrt_vertices_inner_product_wrt_vertices", "forces", "vertices"),
]


def _reference_function(path: Path, name: str):
    """One top-level function of a reference script, compiled from its source unmodified (the
    script itself parses command-line arguments and runs a workload when executed)."""
    tree = ast.parse(path.read_text())
    node = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == name)
    module = ast.Module(body=[node], type_ignores=[])
    namespace = {"np": np, "gzip": gzip}
    exec(compile(module, str(path), "exec"), namespace)
    return namespace[name]


def main(root: Path | None = DEFAULT_REFERENCE) -> None:
    if root is None:
        raise SystemExit("set PYEULERALE_REFERENCE to a checkout of the reference sources")
    grids = {}
    for key, rel in GRIDS.items():
        pts = np.loadtxt(root / rel, dtype=int, skiprows=1, max_rows=1)
        vals = np.loadtxt(root / rel, dtype=float, skiprows=2)
        grids[key] = vals.reshape((2, int(pts[0]), int(pts[1])))
    np.savez_compressed(HERE / "grids.npz", **grids)
    for key, rel in OUTS.items():
        shutil.copyfile(root / rel, HERE / key)

    pkg = load_reference_package(root)
    rng = np.random.default_rng(seed=1)
    s = pkg.SpatialDiscretization(grid_file=root / GRIDS["naca0012_8x9"])
    s.states[:] *= (rng.random(s.states.shape) - 0.5) * 0.01 + 1.
    s.compute_odes()
    s.compute_forces()
    s.linearize()
    out = {
        "states": s.states.copy(), "odes": s.odes.copy(), "forces": s.forces.copy(),
        "odes_wrt_mach": s._odes_wrt_mach.copy(), "odes_wrt_states": s._odes_wrt_states.copy(),
        "odes_wrt_vertices": s._odes_wrt_vertices.copy(),
        "odes_wrt_velocities": s._odes_wrt_velocities.copy(),
        "forces_wrt_states": s._forces_wrt_states.copy(),
        "forces_wrt_vertices": s._forces_wrt_vertices.copy(),
    }

    def rnd(shape):
        a = np.empty(shape, order="F", dtype=complex)
        a[:] = rng.random(shape) + rng.random(shape) * 1j
        return a

    shapes = {"odes": s._odes.shape, "forces": s._forces.shape, "states": s._states.shape,
              "vertices": s._vertices.shape, "velocities": s._velocities.shape}
    for name, cot, direction in SECOND_ORDER:
        w, d = rnd(shapes[cot]), rnd(shapes[direction])
        out[f"{name}/cotangent"] = w
        out[f"{name}/direction"] = d
        out[f"{name}/result"] = getattr(s, name)(w, d)
    # one resolvent pair (test_solve, tests/test_linearization.py:332-356)
    shift = 0.3 + 0.7j
    b = rnd(shapes["odes"])
    out["solve/shift"] = np.array(shift)
    out["solve/rhs"] = b
    out["solve/fwd"] = s.solve_odes_wrt_states_fwd(b, shift=shift)
    out["solve/adj"] = s.solve_odes_wrt_states_adj(b, shift=shift)
    # pressure coefficients, their tangent, and the reference's export of both
    d = rnd(shapes["states"])
    out["cp"] = s.compute_pressure_coefficients()
    out["cp_wrt/direction"] = d
    out["cp_wrt/result"] = s.apply_pressure_coefficients_wrt_states_fwd(d)
    export = _reference_function(root / "examples" / "response" / "run.py",
                                 "export_pressure_coefficients")
    with tempfile.TemporaryDirectory() as tmp:
        export(file_name=str(Path(tmp) / "cp.gz"), vertices=s.vertices,
               pressure_coef=out["cp"], pressure_coef_wrt_aoa=out["cp_wrt/result"])
        (HERE / "cp_export_8x9.txt").write_bytes(gzip.decompress((Path(tmp) / "cp.gz").read_bytes()))
    np.savez_compressed(HERE / "reference_8x9.npz", **out)
    print("wrote", sorted(p.name for p in HERE.iterdir()))


if __name__ == "__main__":
    main()
