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


@pytest.mark.parametrize("per_anchor", [1, 3, 8])
def test_frequency_response_anchored_matches_direct(solver, per_anchor):
    """GMRES preconditioned by the nearest anchor's ring-LU factors gives the direct solves'
    transfer function (every system to 1e-10 relative residual), one to eight shifts per anchor
    (one per anchor: the anchor is the shift itself)."""
    from pyeulerale_b200 import drivers

    ks = np.logspace(-2, 1, 16)
    cl_d, cm_d = drivers.frequency_response_batched(solver, 1.0, 0.25, ks, group=8)
    stats = {}
    cl_a, cm_a = drivers.frequency_response_batched(solver, 1.0, 0.25, ks, method="anchored",
                                                    per_anchor=per_anchor, stats=stats)
    assert stats["anchors"] == -(-len(ks) // per_anchor)
    assert rel_err(cl_a, cl_d) <= 1e-9, (cl_a, cl_d)
    assert rel_err(cm_a, cm_d) <= 1e-9, (cm_a, cm_d)
    if per_anchor == 1:  # the preconditioner is the inverse: done by the first check (5 steps)
        assert max(stats["iterations"]) <= 5 and stats["direct"] == 0, stats


def test_anchored_lift_gradient_matches_adjoint_driver(solver):
    """The lift gradient from the shift-0 factors of the anchored call equals
    adjoint_lift_gradient's, and the transfer function is the one without it."""
    from pyeulerale_b200 import drivers

    ks = np.logspace(-2, 1, 9)
    cl, cm, grad = drivers.frequency_response_batched(solver, 1.0, 0.25, ks, method="anchored",
                                                      lift_gradient=True)
    cl0, cm0 = drivers.frequency_response_batched(solver, 1.0, 0.25, ks, method="anchored")
    assert rel_err(cl, cl0) <= 1e-10 and rel_err(cm, cm0) <= 1e-10
    ref = drivers.adjoint_lift_gradient(solver)
    assert rel_err(grad, ref) <= 1e-9, rel_err(grad, ref)


def test_anchored_gmres_residuals_and_fallback(solver, cuda):
    """solve_anchored reports true residuals at the tolerance; with an iteration limit too small
    to converge it returns EB_ERR_NOCONV per system (no exception), and the driver's direct
    fallback still gives the direct result."""
    from pyeulerale_b200 import drivers
    from pyeulerale_b200.solver import RingLUMany, anchor_shifts, solve_anchored

    M, N = solver.num_radial, solver.num_angular
    rng = np.random.default_rng(12)
    shifts = 1j * np.logspace(-1, -0.6, 6)  # groups of three within a factor 1.6
    rhs = cuda.from_numpy((rng.standard_normal((6, 8 * M * N)))).cuda()
    anchors, sa = anchor_shifts(shifts, 3)
    np.testing.assert_array_equal(sa, [0, 0, 0, 1, 1, 1])
    lu = RingLUMany(solver._batch(), capacity=len(anchors))
    lu.factor(solver._dJ_u, anchors)
    x, info = solve_anchored(solver._batch(), solver._dJ_u, rhs, shifts, lu, sa)
    assert all(i["converged"] and i["rel_residual"] <= 1e-10 for i in info), info
    lu.factor(solver._dJ_u, shifts[:2])
    xd, _ = lu.solve(rhs[:2].contiguous())
    assert rel_err(x[:2].cpu().numpy(), xd.cpu().numpy()) <= 1e-8
    lu.factor(solver._dJ_u, anchors)
    _, info = solve_anchored(solver._batch(), solver._dJ_u, rhs, shifts, lu, sa, maxiter=1,
                             raise_on_failure=False)
    # (the middle shift of a log-spaced group is its anchor and converges at once)
    assert not all(i["converged"] for i in info), info


def test_anchored_sweep_graph_matches_direct_launches(solver, cuda, monkeypatch):
    """The anchored preconditioner's sweep replayed from its CUDA graph gives the same bits as
    the sweep launched directly (EB_RINGLU_GRAPHS=0)."""
    from pyeulerale_b200.solver import RingLUMany, anchor_shifts, solve_anchored

    M, N = solver.num_radial, solver.num_angular
    rng = np.random.default_rng(21)
    shifts = 1j * np.logspace(-1, -0.6, 6)
    rhs = cuda.from_numpy(rng.standard_normal((6, 8 * M * N))).cuda()
    anchors, sa = anchor_shifts(shifts, 3)
    lu = RingLUMany(solver._batch(), capacity=len(anchors))
    lu.factor(solver._dJ_u, anchors)
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("EB_RINGLU_GRAPHS", flag)
        x, info = solve_anchored(solver._batch(), solver._dJ_u, rhs, shifts, lu, sa)
        out.append((x.cpu().numpy(), info.iterations))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


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


def test_ptc_and_adjoint_batched_match_single(cuda):
    """Three uneven instances (two of one grid size, factored together): the batched PTC
    histories, steady states and adjoint lift gradients equal the drop-in's per instance."""
    from pyeulerale_b200 import SpatialDiscretization, drivers
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    specs = [InstanceSpec(G.naca_ogrid(33, 33, 0.12, 1.0, 20.0, 0.01), 0.5, 1.25, 1.0, (0.25, 0.0)),
             InstanceSpec(G.naca_ogrid(21, 25, 0.08, 1.0, 15.0, 0.02), 0.4, -1.0, 1.0, (0.25, 0.0)),
             InstanceSpec(G.naca_ogrid(33, 33, 0.10, 1.0, 20.0, 0.01), 0.45, 2.0, 1.0, (0.25, 0.0))]
    inst = InstanceSet(specs)
    res = drivers.ptc_batched(inst, rtol=1e-10, max_iter=40, workspace_bytes=1 << 30)
    grads = drivers.adjoint_lift_gradients_batched(inst, res, workspace_bytes=1 << 30)
    states = inst.unpack_cells(res.states.cpu().numpy())
    for k, sp in enumerate(specs):
        s = SpatialDiscretization(sp.vertices, mach_number=sp.mach, angle_of_attack=sp.aoa_deg,
                                  coefficient_length=sp.chord, coefficient_center=sp.center)
        hist = drivers.ptc(s, rtol=1e-10, max_iter=40)
        assert res.rel_norms[k][-1] <= 1e-10 and hist.rel_norms[-1] <= 1e-10
        assert abs(len(res.rel_norms[k]) - hist.iterations) <= 1, (k, res.rel_norms[k],
                                                                    hist.rel_norms)
        early = [i for i, r in enumerate(hist.rel_norms) if r > 1e-7 and i < len(res.rel_norms[k])]
        assert np.allclose([res.rel_norms[k][i] for i in early],
                           [hist.rel_norms[i] for i in early], rtol=1e-6), k
        assert rel_err(states[k], s.states.real) <= 1e-9, k
        ref = drivers.adjoint_lift_gradient(s)
        assert rel_err(grads[k], ref) <= 1e-8, (k, rel_err(grads[k], ref))


def test_ptc_batched_large_grids_match_single(cuda):
    """The two largest grid sizes of the uneven workload, a 257x257 and a 513x257 O-grid
    (12.9 GB and 25.8 GB of ring-LU factors each), through the batched PTC and adjoint: the same
    histories, steady states and adjoint lift gradients as the drop-in one instance at a time."""
    from pyeulerale_b200 import SpatialDiscretization, drivers
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    specs = [InstanceSpec(G.naca_ogrid(257, 257, 0.12, 1.0, 20.0, 0.01), 0.5, 1.25, 1.0,
                          (0.25, 0.0)),
             InstanceSpec(G.naca_ogrid(513, 257, 0.08, 1.0, 20.0, 0.01), 0.4, 1.0, 1.0,
                          (0.25, 0.0))]
    inst = InstanceSet(specs)
    res = drivers.ptc_batched(inst, rtol=1e-10, max_iter=30, workspace_bytes=28 << 30)
    grads = drivers.adjoint_lift_gradients_batched(inst, res, workspace_bytes=28 << 30)
    states = inst.unpack_cells(res.states.cpu().numpy())
    batched = res.rel_norms
    del res
    cuda.cuda.empty_cache()
    for k, sp in enumerate(specs):
        s = SpatialDiscretization(sp.vertices, mach_number=sp.mach, angle_of_attack=sp.aoa_deg,
                                  coefficient_length=sp.chord, coefficient_center=sp.center)
        hist = drivers.ptc(s, rtol=1e-10, max_iter=30)
        assert batched[k][-1] <= 1e-10 and hist.rel_norms[-1] <= 1e-10, (k, batched[k],
                                                                          hist.rel_norms)
        assert abs(len(batched[k]) - hist.iterations) <= 1, (k, batched[k], hist.rel_norms)
        early = [i for i, r in enumerate(hist.rel_norms) if r > 1e-7 and i < len(batched[k])]
        assert np.allclose([batched[k][i] for i in early], [hist.rel_norms[i] for i in early],
                           rtol=1e-6), k
        assert rel_err(states[k], s.states.real) <= 1e-9, k
        ref = drivers.adjoint_lift_gradient(s)
        assert rel_err(grads[k], ref) <= 1e-8, (k, rel_err(grads[k], ref))
        del s
        cuda.cuda.empty_cache()


def test_ptc_device_loop_matches_host_loop(cuda):
    """The device PTC loop (eb_ptc_run: one captured step replayed, control values on the
    device) gives the host-driven loop's history, steady state and final residual."""
    from pyeulerale_b200 import SpatialDiscretization, drivers
    from pyeulerale_b200 import grid as G

    X = G.naca_ogrid(33, 41, 0.10, 1.0, 20.0, 0.01)
    a = SpatialDiscretization(X, mach_number=0.5, angle_of_attack=1.25)
    b = SpatialDiscretization(X, mach_number=0.5, angle_of_attack=1.25)
    ha = drivers.ptc(a, rtol=1e-10, max_iter=40, device=True)
    hb = drivers.ptc(b, rtol=1e-10, max_iter=40, device=False)
    assert ha.rel_norms[-1] <= 1e-10 and hb.rel_norms[-1] <= 1e-10
    assert abs(ha.iterations - hb.iterations) <= 1, (ha.rel_norms, hb.rel_norms)
    early = [i for i, r in enumerate(hb.rel_norms) if r > 1e-7 and i < ha.iterations]
    assert np.allclose([ha.rel_norms[i] for i in early], [hb.rel_norms[i] for i in early],
                       rtol=1e-6)
    assert np.allclose(ha.norms[:len(early)], hb.norms[:len(early)], rtol=1e-6)
    assert rel_err(a.states.real, b.states.real) <= 1e-9
    assert np.max(np.abs(a.odes)) / np.max(np.abs(b.odes)) < 10.0  # both round-off level


def test_ptc_device_loop_stops_on_nan_and_at_the_step_limit(cuda):
    """A non-finite state ends the device loop with EB_ERR_NAN after recording a NaN norm; a
    loop cut by max_steps returns EB_OK with max_steps entries (as the example driver)."""
    from pyeulerale_b200 import _lib, grid as G, solver
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    X = G.naca_ogrid(33, 41, 0.10, 1.0, 20.0, 0.01)  # its PTC converges (a 17x21 grid diverges)
    inst = InstanceSet([InstanceSpec(X, 0.5, 1.25)])
    dX = cuda.from_numpy(inst.pack_vertices()).cuda()
    dV = cuda.zeros_like(dX)
    f64 = dict(dtype=cuda.float64, device="cuda")
    U = cuda.empty(4 * inst.n_cells, **f64)
    inst.call("eb_set_free_stream_state", U)
    R, J = cuda.empty(4 * inst.n_cells, **f64), cuda.empty(144 * inst.n_cells, **f64)
    norms, rels, rc = solver.ptc_run(inst.batch, dX, dV, U, R, J, rtol=1e-30, max_steps=3)
    assert rc == _lib.EB_OK and len(rels) == 3 and rels[0] == 1.0
    U[5] = float("nan")
    norms, rels, rc = solver.ptc_run(inst.batch, dX, dV, U, R, J, rtol=1e-10, max_steps=5)
    assert rc == _lib.EB_ERR_NAN and len(rels) == 1 and np.isnan(rels[0])
