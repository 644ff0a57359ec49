"""Parity of the CUDA kernels with the oracle, through the C ABI (GPU)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from helpers import Gpu, crandn, make_case, oracle_eval, rel_err

pytestmark = pytest.mark.gpu

CASES = ["ref8x9", "naca0012_33", "naca0012_33_moving", "naca0004_129", "naca0004_33_sym",
         "min4x5"]

# Tolerances: residual / forces differ from the reference arithmetic by summation order and
# the real-vs-complex evaluation only; Jacobians are exact dual-number derivatives compared
# with h = 1e-12 complex-step derivatives.
TOL_R = 1e-12
TOL_J = 1e-10
TOL_APPLY = 1e-13


@pytest.fixture(scope="module", params=CASES)
def evaluated(request, cuda, oracle, golden_grids):
    case = make_case(request.param, golden_grids, seed=7)
    gpu = Gpu(cuda, case)
    return request.param, case, gpu, gpu.evaluate(), oracle_eval(oracle, case)


def test_residual(evaluated):
    name, _, _, g, o = evaluated
    assert rel_err(g["R"], o["R"]) <= TOL_R, name


def test_forces(evaluated):
    name, _, _, g, o = evaluated
    assert rel_err(g["F"], o["F"]) <= TOL_R, name


@pytest.mark.parametrize("key", ["J_ma", "J_u", "J_x", "J_v", "JF_u", "JF_x"])
def test_jacobians(evaluated, key):
    name, _, _, g, o = evaluated
    assert rel_err(g[key], o[key]) <= TOL_J, (name, key, rel_err(g[key], o[key]))


def test_apply_products(evaluated, oracle):
    """GPU Jacobian products against the oracle's products on the same (GPU) Jacobians."""
    name, case, gpu, g, _ = evaluated
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(3)
    torch = gpu.torch
    sh = {"odes": (4, M, N), "states": (4, M, N), "vertices": (2, M + 1, N + 1),
          "forces": (2, N), "mach": (1,)}
    products = [
        ("eb_apply_odes_wrt_mach_fwd", "apply_odes_wrt_mach_fwd", "J_ma", "mach", "odes"),
        ("eb_apply_odes_wrt_mach_rev", "apply_odes_wrt_mach_rev", "J_ma", "odes", "mach"),
        ("eb_apply_odes_wrt_states_fwd", "apply_odes_wrt_states_fwd", "J_u", "states", "odes"),
        ("eb_apply_odes_wrt_states_rev", "apply_odes_wrt_states_rev", "J_u", "odes", "states"),
        ("eb_apply_odes_wrt_vertices_fwd", "apply_odes_wrt_vertices_fwd", "J_x", "vertices",
         "odes"),
        ("eb_apply_odes_wrt_vertices_rev", "apply_odes_wrt_vertices_rev", "J_x", "odes",
         "vertices"),
        ("eb_apply_odes_wrt_vertices_fwd", "apply_odes_wrt_vertices_fwd", "J_v", "vertices",
         "odes"),
        ("eb_apply_forces_wrt_states_fwd", "apply_forces_wrt_states_fwd", "JF_u", "states",
         "forces"),
        ("eb_apply_forces_wrt_states_rev", "apply_forces_wrt_states_rev", "JF_u", "forces",
         "states"),
        ("eb_apply_forces_wrt_vertices_fwd", "apply_forces_wrt_vertices_fwd", "JF_x",
         "vertices", "forces"),
        ("eb_apply_forces_wrt_vertices_rev", "apply_forces_wrt_vertices_rev", "JF_x", "forces",
         "vertices"),
    ]
    for cname, oname, jkey, src, dst in products:
        x = crandn(rng, sh[src])
        y = torch.zeros(2 * int(np.prod(sh[dst])), dtype=torch.float64, device="cuda")
        gpu.call(cname, g["_dev"][jkey], gpu.dev(x), y)
        got = gpu.host(y, sh[dst], complex_=True)
        ref = np.asfortranarray(np.zeros(sh[dst], dtype=complex))
        getattr(oracle, oname)(g[jkey], x, ref)
        assert rel_err(got, ref) <= TOL_APPLY, (name, cname, rel_err(got, ref))


def test_tangent_kernel(evaluated):
    """Matrix-free forward tangent == sum of the Jacobian products (complex direction)."""
    name, case, gpu, g, o = evaluated
    check_tangent(name, gpu, o)


@pytest.mark.parametrize("name", ["naca0004_33_sym", "naca0012_33"])
def test_tangent_at_exact_free_stream(cuda, oracle, golden_grids, name):
    """At an exact free stream many sensor numerators cancel to exactly zero and abs_c takes
    its derivative sign from a zero (positive, as the reference's complex step does): the
    tangent of the tiled dual kernel matches the complex-step Jacobian products there too."""
    from pyeulerale_b200 import grid as G

    case = make_case(name, golden_grids)
    M, N = case["U"].shape[1], case["U"].shape[2]
    case["U"] = G.perturbed_states(M, N, case["mach"], case["aoa"], 0.0,
                                   np.random.default_rng(0))
    check_tangent(name + "_free_stream", Gpu(cuda, case), oracle_eval(oracle, case))


@pytest.mark.parametrize("entry", ["eb_compute_odes_wrt_states",
                                   "eb_compute_odes_wrt_states_untiled"])
@pytest.mark.parametrize("name", ["naca0004_33_sym", "naca0012_33", "ref8x9"])
def test_states_jacobian_at_exact_free_stream(cuda, oracle, golden_grids, name, entry):
    """At an exact free stream sensor numerators cancel to exactly zero and abs_c takes its
    derivative sign from a zero: every entry of d(odes)/d(states) matches the complex-step
    Jacobian there (a branch taken differently changes an entry by O(1), not by rounding)."""
    from pyeulerale_b200 import grid as G

    case = make_case(name, golden_grids)
    M, N = case["U"].shape[1], case["U"].shape[2]
    case["U"] = G.perturbed_states(M, N, case["mach"], case["aoa"], 0.0,
                                   np.random.default_rng(0))
    gpu = Gpu(cuda, case)
    J = gpu.empty(144 * M * N)
    gpu.call(entry, gpu.X, gpu.V, gpu.U, J)
    got = gpu.host(J, (4, 4, M, N, 9))
    ref = oracle_eval(oracle, case)["J_u"]
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) <= TOL_J * scale, (name, entry)


def test_states_jacobian_tiled_uneven_batch(cuda, oracle, golden_grids):
    """The tiled states Jacobian over one launch of instances of uneven sizes (partial tiles in
    both directions, grids down to M = 4, N = 5) and different flows, moving grids: each
    instance's blocks match the oracle's complex-step Jacobian and the per-cell kernel's."""
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    rng = np.random.default_rng(19)
    grids = [G.naca_ogrid(33, 41, 0.12, 1.0, 20.0, 0.01), G.naca_ogrid(20, 13, 0.06, 2.0, 30.0, 0.05),
             G.naca_ogrid(5, 6, 0.12, 1.0, 10.0, 0.05), G.naca_ogrid(70, 37, 0.10, 1.0, 15.0, 0.02),
             golden_grids["naca0004_129x129"]]
    flows = [(0.5, 1.25), (0.3, -2.0), (0.45, 0.5), (0.6, 3.0), (0.5, 0.0)]
    specs = [InstanceSpec(X, ma, a) for X, (ma, a) in zip(grids, flows)]
    states = [G.perturbed_states(s.M, s.N, s.mach, s.aoa_deg, 0.01, rng) for s in specs]
    vels = [G.smooth_velocities(X, rng) for X in grids]
    inst = InstanceSet(specs)
    dX = cuda.from_numpy(inst.pack_vertices()).cuda()
    dV = cuda.from_numpy(inst.pack_vertices(vels)).cuda()
    dU = cuda.from_numpy(inst.pack_cells(states)).cuda()
    Jt = cuda.full((144 * inst.n_cells,), np.nan, dtype=cuda.float64, device="cuda")
    Ju = cuda.zeros(144 * inst.n_cells, dtype=cuda.float64, device="cuda")
    inst.call("eb_compute_odes_wrt_states", dX, dV, dU, Jt)
    inst.call("eb_compute_odes_wrt_states_untiled", dX, dV, dU, Ju)
    got = inst.unpack_cells(Jt.cpu().numpy(), per_cell=144)
    plain = inst.unpack_cells(Ju.cpu().numpy(), per_cell=144)
    for k, (s, X, V, U) in enumerate(zip(specs, grids, vels, states)):
        shape = (4, 4, s.M, s.N, 9)
        g = np.reshape(got[k].ravel(order="F"), shape, order="F")
        u = np.reshape(plain[k].ravel(order="F"), shape, order="F")
        assert np.all(np.isfinite(g)), k
        ref = oracle_eval(oracle, dict(X=X, V=V, U=U, mach=s.mach, aoa=s.aoa_deg))["J_u"]
        assert rel_err(g, ref) <= TOL_J, (k, rel_err(g, ref))
        assert rel_err(g, u) <= 1e-12, (k, rel_err(g, u))


def run_adjoint(gpu, w, is_complex=True):
    """d_states, d_vertices, d_velocities, d_mach of the matrix-free adjoint (host arrays)."""
    M, N = gpu.M, gpu.N
    f = 2 if is_complex else 1
    gU, gX, gV, gM = (gpu.empty(f * n) for n in (4 * M * N, 2 * (M + 1) * (N + 1),
                                                 2 * (M + 1) * (N + 1), 1))
    gpu.call("eb_apply_odes_adjoint", gpu.X, gpu.V, gpu.U, gpu.dev(w), 1 if is_complex else 0,
             gU, gX, gV, gM)
    sv = (2, M + 1, N + 1)
    return (gpu.host(gU, (4, M, N), is_complex), gpu.host(gX, sv, is_complex),
            gpu.host(gV, sv, is_complex), gpu.host(gM, (1,), is_complex))


def test_adjoint_kernel_matches_reverse_products(evaluated, oracle):
    """The matrix-free adjoint equals the reverse products with the oracle's complex-step
    Jacobians (apply_odes_wrt_states_rev, _vertices_rev with J_x and J_v, _mach_rev)."""
    name, case, gpu, g, o = evaluated
    M, N = gpu.M, gpu.N
    w = crandn(np.random.default_rng(11), (4, M, N))
    got = run_adjoint(gpu, w)
    for (fn, key, shape), y in zip([("apply_odes_wrt_states_rev", "J_u", (4, M, N)),
                                    ("apply_odes_wrt_vertices_rev", "J_x", (2, M + 1, N + 1)),
                                    ("apply_odes_wrt_vertices_rev", "J_v", (2, M + 1, N + 1)),
                                    ("apply_odes_wrt_mach_rev", "J_ma", (1,))], got):
        ref = np.asfortranarray(np.zeros(shape, dtype=complex))
        getattr(oracle, fn)(o[key], w, ref)
        assert rel_err(y, ref) <= TOL_J, (name, key, rel_err(y, ref))


def test_adjoint_kernel_dot_product_with_tangent(evaluated):
    """<w, dR(d)> from the tiled tangent equals <dR^T w, d> from the adjoint, for complex w and
    complex directions on U, X, V and Ma together (bilinear, no conjugation)."""
    name, case, gpu, g, o = evaluated
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(13)
    w = crandn(rng, (4, M, N))
    d = [crandn(rng, (4, M, N)), crandn(rng, (2, M + 1, N + 1)), crandn(rng, (2, M + 1, N + 1)),
         np.array([0.4 + 0.1j])]
    dR = gpu.empty(8 * M * N)
    gpu.call("eb_apply_odes_tangent", gpu.X, gpu.V, gpu.U, *[gpu.dev(a) for a in d], dR, None)
    lhs = np.sum(w * gpu.host(dR, (4, M, N), complex_=True))
    rhs = sum(np.sum(a * b) for a, b in zip(run_adjoint(gpu, w), d))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0), (name, lhs, rhs)


def test_adjoint_kernel_real_cotangent(evaluated):
    """A real cotangent (is_complex = 0) gives the real parts of the complex products."""
    name, case, gpu, g, o = evaluated
    M, N = gpu.M, gpu.N
    w = crandn(np.random.default_rng(17), (4, M, N))
    full = run_adjoint(gpu, w)
    real = run_adjoint(gpu, np.asfortranarray(w.real), is_complex=False)
    for a, b in zip(real, full):
        np.testing.assert_array_equal(a, b.real)


def test_adjoint_kernel_uneven_batch(cuda, oracle, golden_grids):
    """One launch over uneven instances (partial tiles, M = 4 / N = 5, moving grids): each
    instance's reverse products equal the oracle's with its complex-step Jacobians."""
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    rng = np.random.default_rng(29)
    grids = [G.naca_ogrid(33, 41, 0.12, 1.0, 20.0, 0.01), G.naca_ogrid(5, 6, 0.12, 1.0, 10.0, 0.05),
             G.naca_ogrid(70, 37, 0.10, 1.0, 15.0, 0.02), G.naca_ogrid(20, 13, 0.06, 2.0, 30.0, 0.05)]
    flows = [(0.5, 1.25), (0.45, 0.5), (0.6, 3.0), (0.3, -2.0)]
    specs = [InstanceSpec(X, ma, a) for X, (ma, a) in zip(grids, flows)]
    states = [G.perturbed_states(s.M, s.N, s.mach, s.aoa_deg, 0.01, rng) for s in specs]
    vels = [G.smooth_velocities(X, rng) for X in grids]
    ws = [crandn(rng, (4, s.M, s.N)) for s in specs]
    inst = InstanceSet(specs)
    dX = cuda.from_numpy(inst.pack_vertices()).cuda()
    dV = cuda.from_numpy(inst.pack_vertices(vels)).cuda()
    dU = cuda.from_numpy(inst.pack_cells(states)).cuda()
    dw = cuda.from_numpy(inst.pack_cells(ws).view(np.float64)).cuda()
    f64 = dict(dtype=cuda.float64, device="cuda")
    gU = cuda.full((8 * inst.n_cells,), np.nan, **f64)
    gX = cuda.full((4 * inst.n_verts,), np.nan, **f64)
    gV = cuda.full((4 * inst.n_verts,), np.nan, **f64)
    gM = cuda.full((2 * len(specs),), np.nan, **f64)
    inst.call("eb_apply_odes_adjoint", dX, dV, dU, dw, 1, gU, gX, gV, gM)
    hU, hX, hV, hM = (a.cpu().numpy().view(np.complex128) for a in (gU, gX, gV, gM))
    for k, (s, X, V, U, w) in enumerate(zip(specs, grids, vels, states, ws)):
        o = oracle_eval(oracle, dict(X=X, V=V, U=U, mach=s.mach, aoa=s.aoa_deg))
        M, N = s.M, s.N
        c0, v0 = inst.cell_offsets[k], inst.vert_offsets[k]
        nv = (M + 1) * (N + 1)
        got = [np.reshape(hU[4 * c0:4 * (c0 + M * N)], (4, M, N), order="F"),
               np.reshape(hX[2 * v0:2 * (v0 + nv)], (2, M + 1, N + 1), order="F"),
               np.reshape(hV[2 * v0:2 * (v0 + nv)], (2, M + 1, N + 1), order="F"),
               hM[k:k + 1]]
        for (fn, key, shape), y in zip([("apply_odes_wrt_states_rev", "J_u", (4, M, N)),
                                        ("apply_odes_wrt_vertices_rev", "J_x", (2, M + 1, N + 1)),
                                        ("apply_odes_wrt_vertices_rev", "J_v", (2, M + 1, N + 1)),
                                        ("apply_odes_wrt_mach_rev", "J_ma", (1,))], got):
            ref = np.asfortranarray(np.zeros(shape, dtype=complex))
            getattr(oracle, fn)(o[key], np.asfortranarray(w), ref)
            assert rel_err(y, ref) <= TOL_J, (k, key, rel_err(y, ref))


def check_tangent(name, gpu, o):
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(5)
    dU = crandn(rng, (4, M, N))
    dX = crandn(rng, (2, M + 1, N + 1))
    dV = crandn(rng, (2, M + 1, N + 1))
    dMa = np.array([0.3 - 0.2j])
    torch = gpu.torch
    dR = torch.zeros(8 * M * N, dtype=torch.float64, device="cuda")
    gpu.call("eb_apply_odes_tangent", gpu.X, gpu.V, gpu.U, gpu.dev(dU), gpu.dev(dX),
             gpu.dev(dV), gpu.dev(dMa), dR, None)
    got = gpu.host(dR, (4, M, N), complex_=True)
    # reference: complex-step Jacobians applied with the oracle's own routines
    from oracle.shim import SpatialDiscretizationModule

    ora = SpatialDiscretizationModule()
    parts = []
    for fn, J, x in [("apply_odes_wrt_states_fwd", o["J_u"], dU),
                     ("apply_odes_wrt_vertices_fwd", o["J_x"], dX),
                     ("apply_odes_wrt_vertices_fwd", o["J_v"], dV),
                     ("apply_odes_wrt_mach_fwd", o["J_ma"], dMa)]:
        y = np.asfortranarray(np.zeros((4, M, N), dtype=complex))
        getattr(ora, fn)(J, x, y)
        parts.append(y)
    ref = parts[0] + parts[1] + parts[2] + parts[3]
    assert rel_err(got, ref) <= TOL_J, (name, rel_err(got, ref))


def test_bsr_conversion_bit_exact(evaluated, oracle):
    """convert_odes_wrt_states: identical data, indices and index pointers."""
    name, _, gpu, g, _ = evaluated
    M, N = gpu.M, gpu.N
    nnzb = (9 * M - 6) * N
    torch = gpu.torch
    data = torch.zeros(16 * nnzb, dtype=torch.float64, device="cuda")
    idx = torch.zeros(nnzb, dtype=torch.int32, device="cuda")
    ptr = torch.zeros(M * N + 1, dtype=torch.int32, device="cuda")
    gpu.call("eb_convert_odes_wrt_states", g["_dev"]["J_u"], data, idx, ptr)
    r_data = np.asfortranarray(np.zeros((4, 4, nnzb)))
    r_idx = np.zeros(nnzb, dtype=np.int32)
    r_ptr = np.zeros(M * N + 1, dtype=np.int32)
    oracle.convert_odes_wrt_states(g["J_u"], r_data, r_idx, r_ptr)
    np.testing.assert_array_equal(idx.cpu().numpy(), r_idx)
    np.testing.assert_array_equal(ptr.cpu().numpy(), r_ptr)
    np.testing.assert_array_equal(np.reshape(data.cpu().numpy(), (4, 4, nnzb), order="F"),
                                  r_data)


def test_bsr_shifted_spmv(evaluated, oracle):
    name, _, gpu, g, _ = evaluated
    M, N = gpu.M, gpu.N
    nnzb = (9 * M - 6) * N
    torch = gpu.torch
    data = torch.zeros(16 * nnzb, dtype=torch.float64, device="cuda")
    idx = torch.zeros(nnzb, dtype=torch.int32, device="cuda")
    ptr = torch.zeros(M * N + 1, dtype=torch.int32, device="cuda")
    gpu.call("eb_convert_odes_wrt_states", g["_dev"]["J_u"], data, idx, ptr)
    rng = np.random.default_rng(11)
    x = crandn(rng, (4, M, N))
    y = torch.zeros(8 * M * N, dtype=torch.float64, device="cuda")
    shift = 0.25 - 1.5j
    from pyeulerale_b200 import _lib

    _lib.call("eb_bsr_shifted_spmv", M * N, data.data_ptr(), idx.data_ptr(), ptr.data_ptr(),
              shift.real, shift.imag, gpu.dev(x).data_ptr(), y.data_ptr(), None)
    got = gpu.host(y, (4, M, N), complex_=True)
    ref = np.asfortranarray(np.zeros((4, M, N), dtype=complex))
    oracle.apply_odes_wrt_states_fwd(g["J_u"], x, ref)
    ref = ref - shift * x
    assert rel_err(got, ref) <= TOL_APPLY, name


@pytest.mark.parametrize("entry", ["eb_compute_odes", "eb_compute_odes_untiled"])
def test_residual_uneven_batch(cuda, oracle, golden_grids, entry):
    """One launch over instances of uneven sizes (partial tiles) and different flows."""
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    rng = np.random.default_rng(17)
    grids = [G.naca_ogrid(33, 41, 0.12, 1.0, 20.0, 0.01), G.naca_ogrid(20, 13, 0.06, 2.0, 30.0, 0.05),
             golden_grids["naca0004_129x129"], G.naca_ogrid(70, 37, 0.10, 1.0, 15.0, 0.02)]
    flows = [(0.5, 1.25), (0.3, -2.0), (0.6, 3.0), (0.45, 0.0)]
    specs = [InstanceSpec(X, ma, a) for X, (ma, a) in zip(grids, flows)]
    states = [G.perturbed_states(s.M, s.N, s.mach, s.aoa_deg, 0.01, rng) for s in specs]
    vels = [G.smooth_velocities(X, rng) for X in grids]
    inst = InstanceSet(specs)
    dX = cuda.from_numpy(inst.pack_vertices()).cuda()
    dV = cuda.from_numpy(inst.pack_vertices(vels)).cuda()
    dU = cuda.from_numpy(inst.pack_cells(states)).cuda()
    dR = cuda.zeros(4 * inst.n_cells, dtype=cuda.float64, device="cuda")
    inst.call(entry, dX, dV, dU, dR)
    got = inst.unpack_cells(dR.cpu().numpy())
    for k, (s, X, V, U) in enumerate(zip(specs, grids, vels, states)):
        ref = oracle_eval(oracle, dict(X=X, V=V, U=U, mach=s.mach, aoa=s.aoa_deg))["R"]
        assert rel_err(got[k], ref) <= TOL_R, (entry, k, rel_err(got[k], ref))


def test_residual_pipeline_matches_direct_calls(cuda, golden_grids):
    """Streaming steps (overlapped copies and launches) give each step's own residual."""
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec
    from pyeulerale_b200.pipeline import ResidualPipeline

    rng = np.random.default_rng(23)
    X = golden_grids["naca0004_129x129"]
    specs = [InstanceSpec(X, 0.5, 0.0), InstanceSpec(X, 0.45, 1.0)]
    inst = InstanceSet(specs)
    hX = cuda.from_numpy(inst.pack_vertices()).pin_memory()
    hV = cuda.from_numpy(inst.pack_vertices([G.smooth_velocities(X, rng)] * 2)).pin_memory()
    steps = []
    for k in range(5):
        U = [G.perturbed_states(s.M, s.N, s.mach, s.aoa_deg, 0.01, rng) for s in specs]
        steps.append((cuda.from_numpy(inst.pack_cells(U)).pin_memory(),
                      cuda.empty(4 * inst.n_cells, dtype=cuda.float64).pin_memory()))
    pipe = ResidualPipeline(inst, depth=2)
    for hU, hR in steps:
        pipe.submit(hX, hV, hU, hR)
    pipe.synchronize()
    dR = cuda.empty(4 * inst.n_cells, dtype=cuda.float64, device="cuda")
    for hU, hR in steps:
        inst.call("eb_compute_odes", hX.cuda(), hV.cuda(), hU.cuda(), dR)
        np.testing.assert_array_equal(hR.numpy(), dR.cpu().numpy())


@pytest.mark.parametrize("M,N", [(3, 8), (8, 4), (0, 0)])
def test_undersized_grids_are_rejected(cuda, M, N):
    """Grids below M = 4, N = 5 (where the reference indexes out of bounds) fail on the host
    with EB_ERR_ARG before any launch."""
    from pyeulerale_b200 import _lib

    b = _lib.single_batch(_lib.make_instance(M, N, 0.5, 0.0))
    t = cuda.zeros(64, dtype=cuda.float64, device="cuda")
    with pytest.raises(_lib.EulerB200Error) as err:
        _lib.call("eb_compute_odes", ctypes.byref(b), t.data_ptr(), t.data_ptr(), t.data_ptr(),
                  t.data_ptr(), None)
    assert err.value.code == _lib.EB_ERR_ARG


def test_states_jacobian_variants_agree_and_autotune(cuda, golden_grids, monkeypatch):
    """The two dual widths of the tiled states Jacobian give bit-identical blocks, and the
    autotuner times both on the first call of a new size and reports its choice."""
    from pyeulerale_b200 import _lib

    case = make_case("naca0012_33", golden_grids, seed=2)
    gpu = Gpu(cuda, case)
    n = 144 * gpu.M * gpu.N
    out = []
    for v in ("v0", "v1"):
        monkeypatch.setenv("EB_AUTOTUNE", v)
        J = gpu.empty(n)
        gpu.call("eb_compute_odes_wrt_states", gpu.X, gpu.V, gpu.U, J)
        out.append(J.cpu().numpy())
    np.testing.assert_array_equal(out[0], out[1])
    monkeypatch.delenv("EB_AUTOTUNE")
    J = gpu.empty(n)
    gpu.call("eb_compute_odes_wrt_states", gpu.X, gpu.V, gpu.U, J)
    np.testing.assert_array_equal(J.cpu().numpy(), out[0])
    report = _lib.autotune_report()
    line = [s for s in report.splitlines() if f"jac_states_tiled ({gpu.M * gpu.N}," in s]
    assert line and "width 4" in line[0] and "width 2" in line[0] and "(kept)" in line[0]


def test_adjoint_variants_agree(cuda, golden_grids, monkeypatch):
    """The two occupancy variants of the matrix-free adjoint (two CTAs per SM at 128 registers,
    one CTA per SM uncapped) give bit-identical products, and the autotuner lists its choice."""
    from pyeulerale_b200 import _lib

    case = make_case("naca0012_33", golden_grids, seed=3)
    gpu = Gpu(cuda, case)
    w = crandn(np.random.default_rng(31), (4, gpu.M, gpu.N))
    out = []
    for v in ("v0", "v1"):
        monkeypatch.setenv("EB_AUTOTUNE", v)
        out.append(run_adjoint(gpu, w))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)
    monkeypatch.delenv("EB_AUTOTUNE")
    for a, b in zip(run_adjoint(gpu, w), out[0]):
        np.testing.assert_array_equal(a, b)
    report = _lib.autotune_report()
    line = [s for s in report.splitlines()
            if f"residual_adjoint complex ({gpu.M * gpu.N}," in s]
    assert line and "1 CTA/SM" in line[0] and "(kept)" in line[0]


@pytest.mark.parametrize("case_name", ["naca0012_33_moving", "min4x5"])
def test_residual_variants_agree(cuda, golden_grids, monkeypatch, case_name):
    """The residual kernel's two launch variants (loads per use, own cell preloaded) give
    bit-identical residuals, full and partial tiles alike, and the autotuner lists its choice."""
    from pyeulerale_b200 import _lib

    case = make_case(case_name, golden_grids, seed=4)
    gpu = Gpu(cuda, case)
    M, N = gpu.M, gpu.N
    out = []
    for v in ("v0", "v1"):
        monkeypatch.setenv("EB_AUTOTUNE", v)
        R = gpu.empty(4 * M * N)
        gpu.call("eb_compute_odes", gpu.X, gpu.V, gpu.U, R)
        out.append(R.cpu().numpy())
    np.testing.assert_array_equal(out[0], out[1])
    monkeypatch.delenv("EB_AUTOTUNE")
    R = gpu.empty(4 * M * N)
    gpu.call("eb_compute_odes", gpu.X, gpu.V, gpu.U, R)
    np.testing.assert_array_equal(R.cpu().numpy(), out[0])
    assert any(f"residual_tiled ({M * N}," in s and "(kept)" in s
               for s in _lib.autotune_report().splitlines())
