"""The adjoint workload at full size: NACA-0012 257x257 O-grid (chord 1, far field 20 chords,
first spacing 0.01), Ma 0.6, alpha 2 deg, the PTC state plus a seeded 1e-3 relative
perturbation, a seeded smooth grid-velocity field (GPU). The reference's PTC law reaches a
relative residual of 2.8e-5 on this transonic case and then leaves the basin (its residual
grows and the density turns negative), so the checks start from the iterate at rel <= 1e-4;
the 1e-3 perturbation dominates the remaining residual either way.

Checks: the reverse products of R (U, X, V, Ma) and F (U, X) against the oracle's reverse
products of its complex-step Jacobians; dot-product tests of every forward / reverse pair;
central finite differences (h = 1e-6) of <w, R>; the adjoint lift gradient against the forward
tangent; the second-order gradient grad_U <w, dR/dU . d> against finite differences of the
first-order product.
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import crandn, oracle_eval, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def steady(cuda):
    from pyeulerale_b200 import SpatialDiscretization, drivers
    from pyeulerale_b200 import grid as G

    X = G.naca_ogrid(257, 257, thickness=0.12, chord=1.0, far_radius=20.0, first_spacing=0.01)
    s = SpatialDiscretization(X, mach_number=0.6, angle_of_attack=2.0, coefficient_length=1.0,
                              coefficient_center=(0.25, 0.0))
    hist = drivers.ptc(s, rtol=1e-4, max_iter=20)
    assert hist.rel_norms[-1] <= 1e-4, hist.rel_norms
    rng = np.random.default_rng(257)
    s.states[:] = s.states * (1.0 + 1e-3 * rng.standard_normal(s.states.shape))
    s.velocities[:] = G.smooth_velocities(X, rng)
    s.compute_odes()
    s.compute_forces()
    s.linearize()
    return s, rng


def test_reverse_products_match_oracle(steady, oracle):
    s, rng = steady
    o = oracle_eval(oracle, dict(X=s.vertices.real, V=s.velocities.real, U=s.states.real,
                                 mach=s.mach_number, aoa=s.angle_of_attack))
    assert rel_err(s.odes.real, o["R"]) <= 1e-12
    w = crandn(rng, s.odes.shape)
    wf = crandn(rng, s.forces.shape)
    pairs = [("apply_odes_wrt_states_rev", "J_u", w, s.states.shape),
             ("apply_odes_wrt_vertices_rev", "J_x", w, s.vertices.shape),
             ("apply_odes_wrt_velocities_rev", "J_v", w, s.velocities.shape),
             ("apply_odes_wrt_mach_rev", "J_ma", w, (1,)),
             ("apply_forces_wrt_states_rev", "JF_u", wf, s.states.shape),
             ("apply_forces_wrt_vertices_rev", "JF_x", wf, s.vertices.shape)]
    for name, key, cot, shape in pairs:
        got = getattr(s, name)(cot)
        ref = np.asfortranarray(np.zeros(shape, dtype=complex))
        oname = name.replace("velocities", "vertices")
        getattr(oracle, oname)(o[key], cot, ref)
        assert rel_err(got, ref) <= 1e-10, (name, rel_err(got, ref))


def test_dot_products(steady):
    s, rng = steady
    w = crandn(rng, s.odes.shape)
    wf = crandn(rng, s.forces.shape)
    for fwd, rev, src_shape, cot in [
            ("apply_odes_wrt_states_fwd", "apply_odes_wrt_states_rev", s.states.shape, w),
            ("apply_odes_wrt_vertices_fwd", "apply_odes_wrt_vertices_rev", s.vertices.shape, w),
            ("apply_odes_wrt_velocities_fwd", "apply_odes_wrt_velocities_rev", s.velocities.shape, w),
            ("apply_odes_wrt_mach_fwd", "apply_odes_wrt_mach_rev", (1,), w),
            ("apply_forces_wrt_states_fwd", "apply_forces_wrt_states_rev", s.states.shape, wf),
            ("apply_forces_wrt_vertices_fwd", "apply_forces_wrt_vertices_rev", s.vertices.shape, wf)]:
        d = crandn(rng, src_shape)
        lhs = np.sum(cot * getattr(s, fwd)(d))
        rhs = np.sum(getattr(s, rev)(cot) * d)
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1e-300), (fwd, lhs, rhs)


def test_finite_differences_of_residual(steady, cuda):
    """<w, R(x + h d) - R(x - h d)> / 2h, h = 1e-6, against the reverse products. R is smooth
    in X, V and Ma here (1e-6). In U it is smooth only piecewise: the reference's max_c keeps
    the second argument unless the first exceeds it by 1e-8 (f90:111-120), so R jumps by
    ~1e-8 where a face's spectral radii or sensors cross that margin, and a perturbation of all
    65536 cells crosses some of them; the finite difference then differs by ~1e-4 relative
    whatever h is (a jump of size 1e-8 crossed with probability ~h contributes ~1e-8 / h).
    In X the kinks of |u.n| at faces whose normal velocity is near zero give ~1e-5. The
    localized test below checks U to round-off."""
    h = 1e-6
    tol = {"U": 5e-4, "X": 1e-4, "V": 1e-8, "mach": 1e-8}
    from pyeulerale_b200 import autograd
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    s, rng = steady
    inst = InstanceSet([InstanceSpec(s.vertices.real, s.mach_number, s.angle_of_attack, 1.0,
                                     (0.25, 0.0))])
    t = dict(U=cuda.from_numpy(inst.pack_cells([s.states.real])).cuda(),
             X=cuda.from_numpy(inst.pack_vertices()).cuda(),
             V=cuda.from_numpy(inst.pack_vertices([s.velocities.real])).cuda(),
             mach=cuda.tensor([s.mach_number], dtype=cuda.float64))
    leaves = {k: v.clone().requires_grad_(True) for k, v in t.items()}
    R = autograd.residual(leaves["U"], leaves["X"], leaves["V"], leaves["mach"], inst)
    w = cuda.from_numpy(rng.standard_normal(R.numel())).cuda()
    grads = cuda.autograd.grad((R * w).sum(), [leaves[k] for k in ("U", "X", "V", "mach")])
    errors = {}
    for k, (key, g) in enumerate(zip(("U", "X", "V", "mach"), grads)):
        base = t[key]
        d = cuda.from_numpy(rng.standard_normal(base.numel())).to(base.device)
        if key == "U":
            d = d * base  # relative perturbation of the conserved variables
        args = dict(t)
        with cuda.no_grad():
            args[key] = base + h * d
            fp = float((autograd.residual(args["U"], args["X"], args["V"], args["mach"], inst) * w).sum())
            args[key] = base - h * d
            fm = float((autograd.residual(args["U"], args["X"], args["V"], args["mach"], inst) * w).sum())
        inst.set_mach(t["mach"])
        fd = (fp - fm) / (2 * h)
        an = float((g * d).sum())
        errors[key] = abs(fd - an) / abs(an)
    assert all(errors[k] <= tol[k] for k in errors), errors


def _block(shape, rng, scale=None, m=(120, 136), n=(40, 56)):
    """A direction confined to cells [m0, m1) x [n0, n1) (with the cell-state scale if given)."""
    e = np.zeros(shape)
    sub = rng.standard_normal((shape[0], m[1] - m[0], n[1] - n[0]))
    e[:, m[0]:m[1], n[0]:n[1]] = sub * (scale[:, m[0]:m[1], n[0]:n[1]] if scale is not None else 1)
    return np.asfortranarray(e.astype(complex))


def test_localized_finite_differences_states(steady):
    """The same check for U on a 16 x 16 block of the smooth outer flow, with the cotangent on
    the block's stencil neighbourhood only (small sums, so h = 1e-8 keeps its round-off low)."""
    s, rng = steady
    w = _block(s.odes.shape, rng, m=(118, 138), n=(38, 58))
    e = _block(s.states.shape, rng, scale=s.states.real)
    grad = s.apply_odes_wrt_states_rev(w)
    base = s.states.copy()
    h = 1e-8
    vals = []
    for sign in (1.0, -1.0):
        s.states[:] = base + sign * h * e
        s.compute_odes()
        vals.append(float(np.sum(w * s.odes).real))
    s.states[:] = base
    s.compute_odes()
    fd = (vals[0] - vals[1]) / (2 * h)
    an = float(np.sum(grad * e).real)
    assert abs(fd - an) <= 1e-5 * abs(an), (fd, an)


def test_adjoint_lift_gradient(steady):
    from pyeulerale_b200 import drivers

    s, rng = steady
    grad = drivers.adjoint_lift_gradient(s)
    dX = np.asfortranarray(rng.standard_normal(s.vertices.shape).astype(complex))
    g = s.compute_lift_coefficient_wrt_forces()
    dU = -s.solve_odes_wrt_states_fwd(s.apply_odes_wrt_vertices_fwd(d_vertices=dX))
    fwd = np.vdot(g, s.apply_forces_wrt_vertices_fwd(d_vertices=dX)
                  + s.apply_forces_wrt_states_fwd(d_states=dU)).real
    assert abs(float(np.sum(grad * dX.real)) - fwd) <= 1e-8 * abs(fwd)


def test_second_order_gradient_finite_differences(steady):
    """grad_U <w, dR/dU . d> against central differences (h = 1e-8) of the first-order product
    along a direction confined to a 16 x 16 block of cells in the smooth outer flow, with the
    cotangent on the block's neighbourhood: dR/dU itself jumps by O(1) where a max_c branch,
    sign(u.n) or the sign of a sensor's pressure second difference flips (the last is common
    in smooth flow), so a direction over all cells, or a larger step, measures those jumps
    rather than the derivative."""
    s, rng = steady
    w = _block(s.odes.shape, rng, m=(116, 140), n=(36, 60))
    d = np.asfortranarray(rng.standard_normal(s.states.shape).astype(complex))
    grad = s.compute_odes_wrt_states_inner_product_wrt_states(d_odes=w, d_states=d)
    e = _block(s.states.shape, rng, scale=s.states.real)
    base = s.states.copy()
    h = 1e-8
    vals = []
    for sign in (1.0, -1.0):
        s.states[:] = base + sign * h * e
        s.linearize()
        vals.append(np.sum(w * s.apply_odes_wrt_states_fwd(d)).real)
    s.states[:] = base
    s.linearize()
    fd = (vals[0] - vals[1]) / (2 * h)
    an = float(np.sum(grad * e).real)
    assert abs(fd - an) <= 1e-5 * abs(an), (fd, an)
