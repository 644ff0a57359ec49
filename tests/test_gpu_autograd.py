"""torch.autograd of the residual and the wall forces against the oracle's reverse products
(complex-step Jacobians) and central finite differences (GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import oracle_eval, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def packed(cuda, golden_grids):
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    rng = np.random.default_rng(21)
    grids = [G.naca_ogrid(33, 33, 0.12, 1.0, 20.0, 0.01), G.naca_ogrid(20, 13, 0.06, 2.0, 30.0, 0.05),
             golden_grids["naca0012_8x9"]]
    flows = [(0.6, 2.0), (0.3, -2.0), (0.5, 1.25)]
    specs = [InstanceSpec(X, ma, a) for X, (ma, a) in zip(grids, flows)]
    states = [G.perturbed_states(s.M, s.N, s.mach, s.aoa_deg, 0.01, rng) for s in specs]
    vels = [G.smooth_velocities(X, rng) for X in grids]
    inst = InstanceSet(specs)
    t = dict(U=cuda.from_numpy(inst.pack_cells(states)).cuda(),
             X=cuda.from_numpy(inst.pack_vertices()).cuda(),
             V=cuda.from_numpy(inst.pack_vertices(vels)).cuda(),
             mach=cuda.tensor([f[0] for f in flows], dtype=cuda.float64))
    return inst, specs, states, vels, t, rng


def _split_verts(inst, flat):
    out, o = [], 0
    for s in inst.specs:
        n = 2 * (s.M + 1) * (s.N + 1)
        out.append(np.reshape(flat[o:o + n], (2, s.M + 1, s.N + 1), order="F"))
        o += n
    return out


def test_residual_vjp_matches_oracle(cuda, oracle, packed):
    from pyeulerale_b200 import autograd

    inst, specs, states, vels, t, rng = packed
    leaves = {k: v.clone().requires_grad_(True) for k, v in t.items()}
    R = autograd.residual(leaves["U"], leaves["X"], leaves["V"], leaves["mach"], inst)
    w = cuda.from_numpy(rng.standard_normal(R.numel())).cuda()
    (R * w).sum().backward()
    gU = inst.unpack_cells(leaves["U"].grad.cpu().numpy())
    gX = _split_verts(inst, leaves["X"].grad.cpu().numpy())
    gV = _split_verts(inst, leaves["V"].grad.cpu().numpy())
    gM = leaves["mach"].grad.numpy()
    ws = inst.unpack_cells(w.cpu().numpy())
    for k, s in enumerate(specs):
        o = oracle_eval(oracle, dict(X=s.vertices, V=vels[k], U=states[k], mach=s.mach,
                                     aoa=s.aoa_deg))
        wk = np.asfortranarray(ws[k].astype(complex))
        for key, fn, got in [("J_u", "apply_odes_wrt_states_rev", gU[k]),
                             ("J_x", "apply_odes_wrt_vertices_rev", gX[k]),
                             ("J_v", "apply_odes_wrt_vertices_rev", gV[k])]:
            ref = np.asfortranarray(np.zeros(got.shape, dtype=complex))
            getattr(oracle, fn)(o[key], wk, ref)
            assert rel_err(got, ref.real) <= 1e-10, (k, key, rel_err(got, ref.real))
        refm = np.zeros(1, dtype=complex)
        oracle.apply_odes_wrt_mach_rev(o["J_ma"], wk, refm)
        assert abs(gM[k] - refm[0].real) <= 1e-10 * abs(refm[0].real), (k, gM[k], refm)


def test_residual_vjp_finite_difference(cuda, packed):
    from pyeulerale_b200 import autograd

    inst, _, _, _, t, rng = packed
    U = t["U"].clone().requires_grad_(True)
    R = autograd.residual(U, t["X"], t["V"], t["mach"], inst)
    w = cuda.from_numpy(rng.standard_normal(R.numel())).cuda()
    (gU,) = cuda.autograd.grad((R * w).sum(), U)
    d = cuda.from_numpy(rng.standard_normal(U.numel())).cuda() * t["U"]
    h = 1e-7
    with cuda.no_grad():
        fp = (autograd.residual(t["U"] + h * d, t["X"], t["V"], t["mach"], inst) * w).sum()
        fm = (autograd.residual(t["U"] - h * d, t["X"], t["V"], t["mach"], inst) * w).sum()
    fd = float((fp - fm) / (2 * h))
    an = float((gU * d).sum())
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)


def test_forces_vjp_matches_oracle(cuda, oracle, packed):
    from pyeulerale_b200 import autograd

    inst, specs, states, vels, t, rng = packed
    U = t["U"].clone().requires_grad_(True)
    X = t["X"].clone().requires_grad_(True)
    F = autograd.forces(U, X, inst)
    assert F.numel() == 2 * inst.n_wall
    wf = cuda.from_numpy(rng.standard_normal(F.numel())).cuda()
    (F * wf).sum().backward()
    gU = inst.unpack_cells(U.grad.cpu().numpy())
    gX = _split_verts(inst, X.grad.cpu().numpy())
    wfn = wf.cpu().numpy()
    for k, s in enumerate(specs):
        o = oracle_eval(oracle, dict(X=s.vertices, V=vels[k], U=states[k], mach=s.mach,
                                     aoa=s.aoa_deg))
        off = inst.wall_offsets[k]
        wk = np.asfortranarray(np.reshape(wfn[2 * off:2 * (off + s.N)], (2, s.N),
                                          order="F").astype(complex))
        refu = np.asfortranarray(np.zeros((4, s.M, s.N), dtype=complex))
        oracle.apply_forces_wrt_states_rev(o["JF_u"], wk, refu)
        refx = np.asfortranarray(np.zeros((2, s.M + 1, s.N + 1), dtype=complex))
        oracle.apply_forces_wrt_vertices_rev(o["JF_x"], wk, refx)
        assert rel_err(gU[k], refu.real) <= 1e-10, k
        assert rel_err(gX[k], refx.real) <= 1e-10, k
