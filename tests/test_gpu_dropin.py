"""The drop-in class against the reference class's own outputs (GPU).

``tests/golden/reference_8x9.npz`` holds what PyEulerALE's unmodified ``core.py`` returns for the
state of its unit tests (seed 1, 0.5 % noise on the 8x9 grid), including its finite-difference
second-order routines; the drop-in must agree within the reference's own test tolerances
(``atol=1e-6, rtol=1e-5``, tests/test_linearization.py) for the second-order terms and to
round-off for everything else.
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver(cuda, golden_grids, reference_8x9):
    from pyeulerale_b200 import SpatialDiscretization

    s = SpatialDiscretization(golden_grids["naca0012_8x9"])
    s.states[:] = reference_8x9["states"]
    s.compute_odes()
    s.compute_forces()
    s.linearize()
    return s


def test_residual_forces_and_mirrors(solver, reference_8x9):
    assert rel_err(solver.odes, reference_8x9["odes"]) <= 1e-12
    assert rel_err(solver.forces, reference_8x9["forces"]) <= 1e-12
    for key in ["odes_wrt_mach", "odes_wrt_states", "odes_wrt_vertices", "odes_wrt_velocities",
                "forces_wrt_states", "forces_wrt_vertices"]:
        got = getattr(solver, "_" + key)
        assert got.shape == reference_8x9[key].shape and got.flags.f_contiguous
        assert rel_err(got, reference_8x9[key]) <= 1e-10, key


SECOND = [
    "compute_odes_wrt_states_inner_product_wrt_mach",
    "compute_odes_wrt_states_inner_product_wrt_states",
    "compute_odes_wrt_states_inner_product_wrt_vertices",
    "compute_odes_wrt_vertices_inner_product_wrt_mach",
    "compute_odes_wrt_vertices_inner_product_wrt_states",
    "compute_odes_wrt_vertices_inner_product_wrt_vertices",
    "compute_odes_wrt_velocities_inner_product_wrt_mach",
    "compute_odes_wrt_velocities_inner_product_wrt_states",
    "compute_odes_wrt_velocities_inner_product_wrt_vertices",
    "compute_forces_wrt_states_inner_product_wrt_states",
    "compute_forces_wrt_states_inner_product_wrt_vertices",
    "compute_forces_wrt_vertices_inner_product_wrt_states",
    "compute_forces_wrt_vertices_inner_product_wrt_vertices",
]


@pytest.mark.parametrize("name", SECOND)
def test_second_order_matches_reference_fd(solver, reference_8x9, name):
    w = np.asfortranarray(reference_8x9[f"{name}/cotangent"])
    d = np.asfortranarray(reference_8x9[f"{name}/direction"])
    got = getattr(solver, name)(w, d)
    ref = reference_8x9[f"{name}/result"]
    np.testing.assert_allclose(got, ref, atol=1e-6, rtol=1e-5)


def test_resolvent_matches_reference(solver, reference_8x9):
    shift = complex(reference_8x9["solve/shift"])
    b = np.asfortranarray(reference_8x9["solve/rhs"])
    np.testing.assert_allclose(solver.solve_odes_wrt_states_fwd(b, shift=shift),
                               reference_8x9["solve/fwd"], rtol=1e-9)
    np.testing.assert_allclose(solver.solve_odes_wrt_states_adj(b, shift=shift),
                               reference_8x9["solve/adj"], rtol=1e-9)


def test_check_array_errors_like_reference(solver):
    with pytest.raises(RuntimeError, match="Incorrect shape"):
        solver.apply_odes_wrt_states_fwd(np.zeros((4, 2, 2), dtype=complex))
    with pytest.raises(RuntimeError, match="Incorrect data type"):
        solver.apply_odes_wrt_states_fwd(np.asfortranarray(np.zeros(solver.states.shape)))
    with pytest.raises(RuntimeError, match="FORTRAN-contiguous"):
        solver.apply_odes_wrt_states_fwd(np.zeros(solver.states.shape, dtype=complex, order="C"))


def test_pressure_coefficients_on_device(solver, reference_8x9):
    cp = solver.compute_pressure_coefficients()
    assert cp.flags.f_contiguous and cp.dtype == np.float64
    assert rel_err(cp, reference_8x9["cp"]) <= 1e-12  # same bar as residual and forces
    d = np.asfortranarray(reference_8x9["cp_wrt/direction"])
    got = solver.apply_pressure_coefficients_wrt_states_fwd(d)
    assert rel_err(got, reference_8x9["cp_wrt/result"]) <= 1e-12
