"""Workload drivers as library calls: batched frequency response and the adjoint lift gradient
against the one-shift-at-a-time path and the forward tangent (GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver(cuda):
    from pyeulerale_b200 import SpatialDiscretization
    from pyeulerale_b200 import grid as G

    X = G.naca_ogrid(33, 33, thickness=0.12, chord=1.0, far_radius=20.0, first_spacing=0.01)
    s = SpatialDiscretization(X, mach_number=0.5, angle_of_attack=1.25, coefficient_length=1.0,
                              coefficient_center=(0.25, 0.0))
    rng = np.random.default_rng(5)
    s.states[:] = G.perturbed_states(32, 32, 0.5, 1.25, 0.01, rng)
    s.compute_odes()
    s.compute_forces()
    s.linearize()
    return s


def test_frequency_response_batched_matches_plain(solver):
    from pyeulerale_b200 import drivers

    ks = np.logspace(-2, 1, 7)
    cl_p, cm_p = drivers.frequency_response(solver, 1.0, 0.25, ks)
    cl_b, cm_b = drivers.frequency_response_batched(solver, 1.0, 0.25, ks, group=3)
    assert rel_err(cl_b, cl_p) <= 1e-10, (cl_b, cl_p)
    assert rel_err(cm_b, cm_p) <= 1e-10, (cm_b, cm_p)


def test_adjoint_lift_gradient_dot_product(solver):
    """<dc_l/dX, dX> (one adjoint solve) == the forward tangent of c_l along dX."""
    from pyeulerale_b200 import drivers

    grad = drivers.adjoint_lift_gradient(solver)
    assert grad.shape == solver.vertices.shape
    rng = np.random.default_rng(8)
    for _ in range(2):
        dX = np.asfortranarray(rng.standard_normal(solver.vertices.shape).astype(complex))
        g = solver.compute_lift_coefficient_wrt_forces()
        dU = -solver.solve_odes_wrt_states_fwd(solver.apply_odes_wrt_vertices_fwd(d_vertices=dX))
        fwd = np.vdot(g, solver.apply_forces_wrt_vertices_fwd(d_vertices=dX)
                      + solver.apply_forces_wrt_states_fwd(d_states=dU)).real
        adj = float(np.sum(grad * dX.real))
        assert abs(adj - fwd) <= 1e-9 * abs(fwd), (adj, fwd)
