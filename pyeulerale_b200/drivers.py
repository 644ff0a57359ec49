"""Workload drivers as library calls: PTC/SER steady state, frequency response, static gain.

These are the callers of the hot path in the reference's examples
(``examples/response/run.py`` and ``examples/gain/run.py``), written as functions over the
drop-in ``SpatialDiscretization``: everything runs through the device (residual, Jacobians,
ring-block LU resolvent, exact second-order terms). ``response_report`` / ``gain_report``
print the same report as the reference's example scripts, so a run can be compared with the
reference's committed golden outputs line by line.
"""

from __future__ import annotations

import io
from dataclasses import dataclass, field

import numpy as np

from .grid import HEAT_RATIO


@dataclass
class PtcResult:
    """History of the pseudo-transient continuation."""

    norms: list[float] = field(default_factory=list)
    rel_norms: list[float] = field(default_factory=list)

    @property
    def iterations(self) -> int:
        return len(self.norms)


def ptc(solver, rtol: float = 1e-9, max_iter: int = 100, out=None, ser: float = 0.1,
        safeguard: bool = False, growth: float = 10.0, max_retries: int = 8,
        device: bool = True) -> PtcResult:
    """Pseudo-transient continuation with switched evolution relaxation
    (examples/response/run.py:84-123): the time step is ``ser`` / (relative infinity-norm of the
    residual), each step solves (dR/dU - dt^-1 I) dU = -R on the device, and the loop stops at
    rel <= rtol (or NaN), leaving the solver linearized at the final state.

    With ``device`` (the default) the whole loop runs on the GPU (``eb_ptc_run``: residual,
    infinity norm, shift, Jacobian, ring-block LU solve and update with their control values in
    device memory, one CUDA graph replayed per step); the states, residual and history come back
    once at the end. ``device=False`` runs the same loop step by step from the host.

    ``safeguard`` (off by default, which is the reference's loop) rejects a step whose residual
    is not finite or grows by more than ``growth``, and retries it with a ten times larger shift
    (a smaller pseudo time step), up to ``max_retries`` times; the larger shift then decays by
    half per accepted step. This keeps the iterates of cases whose undamped steps overshoot
    into negative densities finite; whether they then converge depends on the case."""
    res = PtcResult()
    if device and not safeguard:
        return _ptc_device(solver, rtol, max_iter, out, ser)
    solver.compute_odes()
    norm_free_stream = np.max(np.abs(solver.odes))
    if out is not None:
        print(f"\nPseudo-transient continuation:\n{'it':>6} {'residual':>15} "
              f"{'rel residual':>15}", file=out)
    floor = 0.0
    for it in range(max_iter):
        solver.compute_odes()
        norm = np.max(np.abs(solver.odes))
        rel = norm / norm_free_stream
        res.norms.append(float(norm))
        res.rel_norms.append(float(rel))
        if out is not None:
            print(f"{it:>6} {norm:>15.1e} {rel:>15.1e}", file=out)
        solver.linearize()
        solver.compute_forces()
        if rel <= rtol or np.isnan(rel):
            break
        time_step = ser * rel**-1.
        shift = time_step**-1.
        if not safeguard:
            update = solver.solve_odes_wrt_states_fwd(d_odes=-solver.odes, shift=shift)
            solver.states[:] += update
            continue
        shift = max(shift, floor)
        base, rhs = solver.states.copy(), -solver.odes
        for _ in range(max_retries + 1):
            solver.states[:] = base + solver.solve_odes_wrt_states_fwd(d_odes=rhs, shift=shift)
            solver.compute_odes()
            trial = np.max(np.abs(solver.odes)) / norm_free_stream
            if np.isfinite(trial) and trial <= growth * rel:
                break
            shift *= 10.0
        floor = shift / 2.0 if shift > rel / ser else floor / 2.0
    return res


def _ptc_device(solver, rtol: float, max_iter: int, out, ser: float) -> PtcResult:
    """``ptc`` through the device loop of one instance (``solver.ptc_run``)."""
    from . import solver as solver_mod

    solver._upload()
    norms, rels, _ = solver_mod.ptc_run(solver._batch(), solver._dX, solver._dV, solver._dU,
                                        solver._dR, solver._dJ_u, ser=ser, rtol=rtol,
                                        max_steps=max_iter)
    solver._states[...] = np.reshape(solver._dU.cpu().numpy(), solver._states.shape, order="F")
    res = PtcResult(norms=[float(v) for v in norms], rel_norms=[float(v) for v in rels])
    if out is not None:
        print(f"\nPseudo-transient continuation:\n{'it':>6} {'residual':>15} "
              f"{'rel residual':>15}", file=out)
        for it, (norm, rel) in enumerate(zip(res.norms, res.rel_norms)):
            print(f"{it:>6} {norm:>15.1e} {rel:>15.1e}", file=out)
    # the solver's host residual, Jacobians and forces at the final state
    solver.compute_odes()
    solver.linearize()
    solver.compute_forces()
    return res


@dataclass
class BatchedPtcResult:
    """Per-instance histories of ``ptc_batched`` and the packed device states."""

    rel_norms: list = field(default_factory=list)   # one list of relative norms per instance
    states: object = None                             # packed float64 device tensor
    vertices: object = None
    velocities: object = None

    @property
    def iterations(self) -> list[int]:
        return [len(h) for h in self.rel_norms]


def _shape_groups(instances) -> dict:
    groups: dict = {}
    for i, sp in enumerate(instances.specs):
        groups.setdefault((sp.M, sp.N), []).append(i)
    return groups


def _batched_solves(instances, J, shifts_of, rhs_of, out_of, adjoint: bool, workspace,
                    tol: float, on_fail=None) -> None:
    """Solves (J_i - s_i I) x_i = b_i (or the adjoint) for the instances in ``shifts_of``, the
    instances of one grid size together per factorisation call, as many per call as the
    ``workspace`` (one uint8 device tensor) holds. If a call fails (a singular or non-finite
    system, a solve that misses ``tol``), its systems are retried one at a time and those that
    still fail are passed to ``on_fail`` (or re-raised without one)."""
    from . import _lib
    from .solver import RingLUMany, ringlu_workspace_bytes

    groups = _shape_groups(instances)
    for (M, N), members in groups.items():
        todo = [i for i in members if i in shifts_of]
        if not todo:
            continue
        stride = (ringlu_workspace_bytes(M, N) + 255) // 256 * 256
        cap = max(1, min(len(todo), workspace.numel() // stride))
        if workspace.numel() < stride:
            raise ValueError(f"workspace of {workspace.numel()} bytes is below one {M}x{N} system")
        batch = _lib.single_batch(_lib.make_instance(M, N, 0.5, 0.0))
        lu = RingLUMany(batch, capacity=cap, tol=tol, workspace=workspace)
        nc = M * N

        def run(chunk):
            offs = [instances.cell_offsets[i] for i in chunk]
            lu.factor([J[144 * o:144 * (o + nc)] for o in offs], [shifts_of[i] for i in chunk])
            xs, _ = lu.solve([rhs_of(i) for i in chunk], adjoint=adjoint)
            for i, x in zip(chunk, xs):
                out_of(i, x)

        for c0 in range(0, len(todo), cap):
            chunk = todo[c0:c0 + cap]
            try:
                run(chunk)
            except _lib.EulerB200Error:
                for i in chunk:
                    try:
                        run([i])
                    except _lib.EulerB200Error:
                        if on_fail is None:
                            raise
                        on_fail(i)


def ptc_batched(instances, states=None, rtol: float = 1e-10, max_iter: int = 100,
                ser: float = 0.1, workspace_bytes: int = 64 << 30, tol: float = 1e-10,
                velocities=None) -> BatchedPtcResult:
    """The PTC/SER loop of ``ptc`` for every instance of an ``InstanceSet`` at once.

    Each iteration evaluates the residuals and d(odes)/d(states) of all instances in one launch
    each, takes every unconverged instance's relative infinity norm (one segmented reduction),
    and solves each instance's (dR/dU - dt^-1 I) dU = -R with the ring-block LU, the instances
    of one grid size factored together (``eb_ringlu_factor_many`` with one Jacobian per
    system) within ``workspace_bytes`` of factor storage. Instances stop individually at
    rel <= rtol (or NaN). ``states`` (packed, host or device) defaults to the free stream.
    """
    import torch

    inst = instances
    f64 = dict(dtype=torch.float64, device="cuda")
    dX = torch.from_numpy(inst.pack_vertices()).cuda()
    dV = (torch.zeros_like(dX) if velocities is None
          else torch.as_tensor(velocities, dtype=torch.float64).cuda())
    dU = torch.empty(4 * inst.n_cells, **f64)
    if states is None:
        inst.call("eb_set_free_stream_state", dU)
    else:
        dU.copy_(torch.as_tensor(states, dtype=torch.float64))
    R = torch.empty(4 * inst.n_cells, **f64)
    J = torch.empty(144 * inst.n_cells, **f64)
    lengths = torch.tensor([4 * sp.M * sp.N for sp in inst.specs], device="cuda")
    seg_max = lambda v: torch.segment_reduce(v.abs(), "max", lengths=lengths)  # noqa: E731
    workspace = torch.empty(int(workspace_bytes) // 256 * 256, dtype=torch.uint8, device="cuda")
    inst.call("eb_compute_odes", dX, dV, dU, R)
    norm0 = seg_max(R).cpu().numpy()
    res = BatchedPtcResult(rel_norms=[[] for _ in inst.specs])
    active = set(range(len(inst)))
    for _ in range(max_iter):
        inst.call("eb_compute_odes", dX, dV, dU, R)
        rel = seg_max(R).cpu().numpy() / norm0
        for i in sorted(active):
            res.rel_norms[i].append(float(rel[i]))
        active = {i for i in active if not (rel[i] <= rtol or np.isnan(rel[i]))}
        if not active:
            break
        inst.call("eb_compute_odes_wrt_states", dX, dV, dU, J)
        shifts = {i: (ser * rel[i]**-1.)**-1. for i in active}

        def rhs_of(i):
            o, n = inst.cell_offsets[i], 4 * inst.specs[i].M * inst.specs[i].N
            b = torch.zeros(2 * n, **f64)
            b[0::2] = -R[4 * o:4 * o + n]
            return b

        def update(i, x):
            o, n = inst.cell_offsets[i], 4 * inst.specs[i].M * inst.specs[i].N
            dU[4 * o:4 * o + n] += x[0::2]

        def failed(i):  # a singular shifted Jacobian: the instance stops here, as diverged
            o, n = inst.cell_offsets[i], 4 * inst.specs[i].M * inst.specs[i].N
            dU[4 * o:4 * o + n] = float("nan")

        _batched_solves(inst, J, shifts, rhs_of, update, False, workspace, tol, failed)
    res.states, res.vertices, res.velocities = dU, dX, dV
    return res


def adjoint_lift_gradients_batched(instances, result: BatchedPtcResult,
                                   workspace_bytes: int = 64 << 30,
                                   tol: float = 1e-10) -> list[np.ndarray]:
    """``adjoint_lift_gradient`` of every instance at the states of ``result``: the forces
    Jacobians, d(odes)/d(states) and d(odes)/d(vertices) of all instances in one launch each,
    the adjoint solves at shift 0 with the instances of one grid size factored together, and
    the reverse products over all instances. Returns one (2, M+1, N+1) array per instance, or
    None for an instance whose PTC did not converge (or whose adjoint system is singular)."""
    import torch

    inst = instances
    f64 = dict(dtype=torch.float64, device="cuda")
    dX, dV, dU = result.vertices, result.velocities, result.states
    nc, nv, nw = inst.n_cells, inst.n_verts, inst.n_wall
    g = torch.zeros(4 * nw, **f64)  # complex (2, N) per instance: d c_l / d F_z = 1 / (q c)
    for sp, w in zip(inst.specs, inst.wall_offsets):
        q = sp.mach**2 * HEAT_RATIO / 2
        g[4 * w + 2:4 * (w + sp.N):4] = 1.0 / (q * sp.chord)
    JFu, JFx = torch.empty(8 * nw, **f64), torch.empty(8 * nw, **f64)
    inst.call("eb_compute_forces_wrt_states", dX, dU, JFu)
    inst.call("eb_compute_forces_wrt_vertices", dX, dU, JFx)
    gU = torch.empty(8 * nc, **f64)
    inst.call("eb_apply_forces_wrt_states_rev", JFu, g, gU)
    J = torch.empty(144 * nc, **f64)
    inst.call("eb_compute_odes_wrt_states", dX, dV, dU, J)
    lam = torch.empty(8 * nc, **f64)

    def rhs_of(i):
        o, n = inst.cell_offsets[i], 8 * inst.specs[i].M * inst.specs[i].N
        return gU[8 * o:8 * o + n]

    def store(i, x):
        o, n = inst.cell_offsets[i], 8 * inst.specs[i].M * inst.specs[i].N
        lam[8 * o:8 * o + n] = x

    ok = {i for i, h in enumerate(result.rel_norms) if h and np.isfinite(h[-1])}
    bad = set(range(len(inst))) - ok
    workspace = torch.empty(int(workspace_bytes) // 256 * 256, dtype=torch.uint8, device="cuda")
    _batched_solves(inst, J, {i: 0.0 for i in sorted(ok)}, rhs_of, store, True, workspace, tol,
                    bad.add)
    del workspace, J
    Jx = torch.empty(32 * nc, **f64)
    inst.call("eb_compute_odes_wrt_vertices", dX, dV, dU, Jx)
    gX_r, gX_f = torch.empty(4 * nv, **f64), torch.empty(4 * nv, **f64)
    inst.call("eb_apply_odes_wrt_vertices_rev", Jx, lam, gX_r)
    inst.call("eb_apply_forces_wrt_vertices_rev", JFx, g, gX_f)
    grad = (gX_f - gX_r)[0::2].cpu().numpy()
    out, o = [], 0
    for k, sp in enumerate(inst.specs):
        n = 2 * (sp.M + 1) * (sp.N + 1)
        out.append(None if k in bad else np.asfortranarray(
            np.reshape(grad[o:o + n], (2, sp.M + 1, sp.N + 1), order="F")))
        o += n
    return out


def pitch_vertices(solver, axis_location: float) -> np.ndarray:
    """dX/dalpha of a rigid pitch about (axis_location, 0), per radian."""
    v = np.empty_like(solver.vertices, dtype=complex)
    v[1] = -(solver.vertices[0] - axis_location)
    v[0] = solver.vertices[1]
    return v


def frequency_response(solver, chord: float, axis_location: float,
                       reduced_frequencies, out=None, cp_file=None) -> tuple[np.ndarray, np.ndarray]:
    """Pitch-to-(c_l, c_m) transfer function at s = i k V_inf / (c/2)
    (examples/response/run.py:125-176). Returns (c_l(s), c_m(s)). With ``cp_file``, writes the
    steady pressure coefficients and their pitch response at the last frequency in the
    example's export format (examples/response/run.py:178-186)."""
    speed = solver.mach_number * HEAT_RATIO**0.5
    dX = pitch_vertices(solver, axis_location)
    cl_grad = solver.compute_lift_coefficient_wrt_forces()
    cm_grad = solver.compute_moment_coefficient_wrt_forces()
    cm_grad_x = solver.compute_moment_coefficient_wrt_vertices()
    if out is not None:
        print(f"\nFrequency response:\n{'red frequency':>15} {'lift coefficient':>25} "
              f"{'moment coefficient':>25}", file=out)
    cls, cms = [], []
    rhs_x = solver.apply_odes_wrt_vertices_fwd(d_vertices=dX)
    dF_x = solver.apply_forces_wrt_vertices_fwd(d_vertices=dX)
    for k in reduced_frequencies:
        s = 1j * k * speed / (chord / 2)
        dU = -solver.solve_odes_wrt_states_fwd(
            shift=s, d_odes=rhs_x + solver.apply_odes_wrt_velocities_fwd(d_velocities=s * dX))
        dF = dF_x + solver.apply_forces_wrt_states_fwd(d_states=dU)
        cl = np.vdot(cl_grad, dF)
        cm = np.vdot(cm_grad, dF) + np.vdot(cm_grad_x, dX)
        cls.append(cl)
        cms.append(cm)
        if out is not None:
            print(f"{k:>15.3e} {cl:>+25.3e} {cm:>+25.3e}", file=out)
    if cp_file is not None and len(cls):
        from .export import export_pressure_coefficients

        export_pressure_coefficients(cp_file, solver.vertices, solver.compute_pressure_coefficients(),
                                     solver.apply_pressure_coefficients_wrt_states_fwd(dU))
    return np.array(cls), np.array(cms)


def _device_apply(solver, name: str, jac, x, out_numel: int):
    """y = jac-product(x) on the device; x, y interleaved complex float64 tensors."""
    import torch

    y = torch.empty(2 * out_numel, dtype=torch.float64, device="cuda")
    solver._call(name, jac.data_ptr(), x.data_ptr(), y.data_ptr())
    return y


def frequency_response_batched(solver, chord: float, axis_location: float,
                               reduced_frequencies, group: int = 16,
                               tol: float = 1e-10, method: str = "direct",
                               per_anchor: int = 3, stats: dict | None = None,
                               lift_gradient: bool = False):
    """``frequency_response`` with the shifts factored and solved together on the device.

    The pitch-to-(c_l, c_m) transfer function at s = i k V_inf / (c/2) for every reduced
    frequency k (examples/response/run.py:135-176): each shift solves
    (dR/dU - s I) dU = -(dR/dX + s dR/dV) dX/dalpha; c_l(s) = <grad_F c_l, dF/dX dX + dF/dU dU>,
    c_m(s) likewise plus <grad_X c_m, dX>. Right-hand sides, solutions and force perturbations
    stay on the device, only the 2 x len(k) coefficients come back. The solver must be
    linearized at the state of interest.

    method "direct": ``group`` shifts share each factorisation call (``RingLUMany``: one launch
    per elimination step for the whole group). method "anchored": the shifts, ordered by
    magnitude, go in groups of ``per_anchor`` around one factorised anchor shift each, and all
    shifts are solved by GMRES preconditioned with their anchor's factors
    (``solver.solve_anchored``) to tol / 100; a shift whose GMRES does not converge is solved
    directly.
    ``stats`` (optional dict) receives the anchored solve's iteration counts.

    ``lift_gradient=True`` (anchored method) also returns the adjoint lift gradient
    (``adjoint_lift_gradient``): shift 0 is factored in the same batched call as the anchors and
    its adjoint solve uses those factors. Returns ``(cl, cm)`` or ``(cl, cm, gradient)``.
    """
    import torch

    from .solver import RingLUMany, anchor_shifts, solve_anchored

    ks = np.atleast_1d(np.asarray(reduced_frequencies, dtype=float))
    speed = solver.mach_number * HEAT_RATIO**0.5
    shifts = 1j * ks * speed / (chord / 2)
    nc = solver.num_radial * solver.num_angular
    nf = solver.forces.size
    dX = pitch_vertices(solver, axis_location)
    dXd = solver._cvec(dX)
    rx = torch.view_as_complex(_device_apply(
        solver, "eb_apply_odes_wrt_vertices_fwd", solver._dJ_x, dXd, 4 * nc).view(-1, 2))
    rv = torch.view_as_complex(_device_apply(
        solver, "eb_apply_odes_wrt_vertices_fwd", solver._dJ_v, dXd, 4 * nc).view(-1, 2))
    dFx = torch.view_as_complex(_device_apply(
        solver, "eb_apply_forces_wrt_vertices_fwd", solver._dJF_x, dXd, nf).view(-1, 2))
    to_dev = lambda a: torch.from_numpy(  # noqa: E731
        np.ascontiguousarray(np.asarray(a, dtype=complex).ravel(order="F"))).to("cuda")
    cl_grad = to_dev(solver.compute_lift_coefficient_wrt_forces())
    cm_grad = to_dev(solver.compute_moment_coefficient_wrt_forces())
    cm_x = complex(np.vdot(solver.compute_moment_coefficient_wrt_vertices(), dX))
    cl = np.empty(len(shifts), dtype=complex)
    cm = np.empty(len(shifts), dtype=complex)

    def rhs_of(chunk):
        st = torch.from_numpy(np.asarray(chunk)).to("cuda")[:, None]
        return torch.view_as_real(-(rx[None, :] + st * rv[None, :])).reshape(len(chunk), -1) \
            .contiguous()

    def coefficients(idx, x):
        dF = torch.stack([torch.view_as_complex(_device_apply(
            solver, "eb_apply_forces_wrt_states_fwd", solver._dJF_u, x[k], nf).view(-1, 2))
            for k in range(len(idx))]) + dFx[None, :]
        cl[idx] = (dF @ cl_grad.conj()).cpu().numpy()
        cm[idx] = (dF @ cm_grad.conj()).cpu().numpy() + cm_x

    if method == "direct":
        lu = RingLUMany(solver._batch(), capacity=min(group, len(shifts)), tol=tol)
        for g0 in range(0, len(shifts), lu.capacity):
            chunk = shifts[g0:g0 + lu.capacity]
            lu.factor(solver._dJ_u, chunk)
            x, _ = lu.solve(rhs_of(chunk))
            coefficients(np.arange(g0, g0 + len(chunk)), x)
        return cl, cm
    if method != "anchored":
        raise ValueError(f"unknown method {method!r}")
    anchors, sys_anchor = anchor_shifts(shifts, per_anchor)
    factored = list(anchors) + ([0.0] if lift_gradient else [])  # shift 0: the adjoint's
    lu = RingLUMany(solver._batch(), capacity=len(factored), tol=tol)
    lu.factor(solver._dJ_u, factored)
    # GMRES to tol / 100: the direct solves stop at tol too, and two solutions within tol of
    # the same system differ by the system's conditioning times tol; the margin keeps the
    # transfer function within ~tol of the direct one
    x, info = solve_anchored(solver._batch(), solver._dJ_u, rhs_of(shifts), shifts, lu,
                             sys_anchor, tol=tol * 1e-2, raise_on_failure=False)
    grad = None
    if lift_gradient:  # the adjoint lift gradient on the shift-0 factors, before any re-factoring
        g = solver.compute_lift_coefficient_wrt_forces().astype(complex)
        b = solver._cvec(solver.apply_forces_wrt_states_rev(d_forces=g))
        lam, _ = lu.solve_one(len(anchors), b, adjoint=True)
        lam_h = np.reshape(lam.cpu().numpy().view(np.complex128), solver.odes.shape, order="F")
        grad = np.asfortranarray((solver.apply_forces_wrt_vertices_rev(d_forces=g)
                                  - solver.apply_odes_wrt_vertices_rev(d_odes=lam_h)).real)
    bad = [k for k, i in enumerate(info) if not i["converged"]]
    for g0 in range(0, len(bad), lu.capacity):  # direct solves of the unconverged shifts
        idx = bad[g0:g0 + lu.capacity]
        lu.factor(solver._dJ_u, shifts[idx])
        xd, _ = lu.solve(rhs_of(shifts[idx]))
        for j, k in enumerate(idx):
            x[k] = xd[j]
    del lu
    if stats is not None:
        stats.update(anchors=len(anchors), iterations=info.iterations, direct=len(bad))
    coefficients(np.arange(len(shifts)), x)
    return (cl, cm, grad) if lift_gradient else (cl, cm)


def adjoint_lift_gradient(solver) -> np.ndarray:
    """Gradient of the steady-state lift coefficient with respect to the grid vertices.

    With R(U, X) = 0 at the solver's (converged, linearized) state, dc_l/dX =
    (dF/dX)^T g - (dR/dX)^T lam with g = grad_F c_l and (dR/dU)^T lam = (dF/dU)^T g: one adjoint
    solve (solve_odes_wrt_states_adj at shift 0) and three reverse products, the device
    counterpart of the adjoint of examples/gain/run.py:107-109. Returns (2, M+1, N+1).
    """
    g = solver.compute_lift_coefficient_wrt_forces().astype(complex)
    lam = solver.solve_odes_wrt_states_adj(solver.apply_forces_wrt_states_rev(d_forces=g))
    grad = (solver.apply_forces_wrt_vertices_rev(d_forces=g)
            - solver.apply_odes_wrt_vertices_rev(d_odes=lam.astype(complex)))
    return np.asfortranarray(grad.real)


def static_gain(solver, out=None) -> tuple[float, float]:
    """Lift slope dc_l/dalpha and its Mach derivative at zero angle of attack
    (examples/gain/run.py:81-145), with the adjoint of c_l and the exact second-order terms."""
    dX = pitch_vertices(solver, 0.0)
    cl_grad = solver.compute_lift_coefficient_wrt_forces()
    dU_a = -solver.solve_odes_wrt_states_fwd(d_odes=solver.apply_odes_wrt_vertices_fwd(
        d_vertices=dX))
    cl_a = np.vdot(cl_grad, solver.apply_forces_wrt_vertices_fwd(d_vertices=dX)
                   + solver.apply_forces_wrt_states_fwd(d_states=dU_a))
    dU_m = -solver.solve_odes_wrt_states_fwd(
        d_odes=solver.apply_odes_wrt_mach_fwd(d_mach=np.asarray([1. + 0j])))
    adj = -solver.solve_odes_wrt_states_adj(solver.apply_forces_wrt_states_rev(d_forces=cl_grad))
    cl_a_m = (
        -2 / solver.mach_number * cl_a
        + np.vdot(solver.compute_forces_wrt_states_inner_product_wrt_states(
            d_forces=cl_grad, d_states=dU_a), dU_m)
        + np.vdot(solver.compute_forces_wrt_vertices_inner_product_wrt_states(
            d_forces=cl_grad, d_vertices=dX), dU_m)
        + solver.compute_odes_wrt_states_inner_product_wrt_mach(d_odes=adj, d_states=dU_a).item()
        + np.vdot(solver.compute_odes_wrt_states_inner_product_wrt_states(
            d_odes=adj, d_states=dU_m), dU_a)
        + solver.compute_odes_wrt_vertices_inner_product_wrt_mach(
            d_odes=adj, d_vertices=dX).item()
        + np.vdot(solver.compute_odes_wrt_states_inner_product_wrt_vertices(
            d_odes=adj, d_states=dU_m), dX)
    )
    if out is not None:
        print("\nLift coefficient derivatives:", file=out)
        print(f"{'wrt pitch angle:':<36} {cl_a.real:.4f} (1/rad)", file=out)
        print(f"{'wrt pitch angle wrt Mach number:':<36} {cl_a_m.real:.4f} (1/rad)", file=out)
    return float(cl_a.real), float(cl_a_m.real)


def response_report(grid, mesh_name: str, chord: float, mach: float, axis_location: float,
                    rtol: float = 1e-9, max_iter: int = 100, **solver_kw) -> str:
    """The report of the response example for one grid (PTC + 11-point frequency response)."""
    from .core import SpatialDiscretization

    out = io.StringIO()
    print(f"{'Mesh file:':<25} {mesh_name}", file=out)
    print(f"{'Chord / L:':<25} {chord}", file=out)
    print(f"{'Mach number:':<25} {mach}", file=out)
    print(f"{'Axis location / L:':<25} {axis_location}", file=out)
    s = SpatialDiscretization(grid, mach_number=mach, angle_of_attack=0., coefficient_length=chord,
                              coefficient_center=(axis_location, 0.0), **solver_kw)
    ptc(s, rtol, max_iter, out)
    frequency_response(s, chord, axis_location, np.logspace(-2, 0, 11), out)
    return out.getvalue()


def gain_report(grid, mesh_name: str, chord: float, mach: float, rtol: float = 1e-9,
                max_iter: int = 100, **solver_kw) -> str:
    """The report of the gain example for one grid (PTC + lift slope and its Mach derivative)."""
    from .core import SpatialDiscretization

    out = io.StringIO()
    print(f"{'Mesh file:':<25} {mesh_name}", file=out)
    print(f"{'Chord / L:':<25} {chord}", file=out)
    print(f"{'Mach number:':<25} {mach}", file=out)
    s = SpatialDiscretization(grid, mach_number=mach, angle_of_attack=0., coefficient_length=chord,
                              **solver_kw)
    ptc(s, rtol, max_iter, out)
    static_gain(s, out)
    return out.getvalue()
