"""Device GMRES resolvent against the direct sparse solve of the oracle Jacobian (GPU)."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from helpers import Gpu, crandn, make_case, rel_err

pytestmark = pytest.mark.gpu


def bsr_matrix(oracle, J: np.ndarray) -> sp.csr_matrix:
    """The reference's CSR assembly (core.py:512-531) from the oracle's BSR conversion."""
    M, N = J.shape[2], J.shape[3]
    nnzb = (9 * M - 6) * N
    data = np.asfortranarray(np.zeros((4, 4, nnzb)))
    idx = np.zeros(nnzb, dtype=np.int32)
    ptr = np.zeros(M * N + 1, dtype=np.int32)
    oracle.convert_odes_wrt_states(J, data, idx, ptr)
    return sp.bsr_matrix((np.moveaxis(data, -1, 0), idx - 1, ptr - 1)).tocsr()


@pytest.mark.parametrize("name,shift", [("ref8x9", 0.3 + 0.7j), ("ref8x9", 2.0),
                                        ("ref8x9", 0.05j), ("naca0012_33", 60.0)])
@pytest.mark.parametrize("adjoint", [False, True])
def test_gmres_matches_direct_solve(cuda, oracle, golden_grids, name, shift, adjoint):
    """Block-Jacobi GMRES where it converges (small grids, or large shifts)."""
    from pyeulerale_b200 import solver

    case = make_case(name, golden_grids, seed=2)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(9)
    b = crandn(rng, (4, M, N))
    x, info = solver.solve_shifted(gpu.batch, g["_dev"]["J_u"], gpu.dev(b), [shift],
                                   adjoint=adjoint, tol=1e-10, restart=60, maxiter=5000)
    got = gpu.host(x, (4, M, N), complex_=True)
    A = bsr_matrix(oracle, g["J_u"]).astype(complex)
    n = A.shape[0]
    if adjoint:
        op = (A - np.conj(shift) * sp.eye(n)).T.tocsc()
    else:
        op = (A - shift * sp.eye(n)).tocsc()
    bf = b.ravel(order="F")
    res = np.linalg.norm(bf - op @ got.ravel(order="F")) / np.linalg.norm(bf)
    assert res <= 1e-10, (info, res)
    ref = spla.spsolve(op, bf)
    assert rel_err(got.ravel(order="F"), ref) <= 1e-7, info


def test_gmres_batched_shifts_match_single(cuda, golden_grids):
    """Several shifts in one call give the same solutions as one call per shift."""
    from pyeulerale_b200 import solver

    case = make_case("ref8x9", golden_grids, seed=4)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(1)
    shifts = [0.5j, 1.0 + 0.2j, 3.0, 0.1 - 0.4j]
    rhs = [crandn(rng, (4, M, N)) for _ in shifts]
    packed = cuda.cat([gpu.dev(r) for r in rhs])
    xb, info_b = solver.solve_shifted(gpu.batch, g["_dev"]["J_u"], packed, shifts,
                                      sys_inst=[0] * len(shifts))
    n = 8 * M * N
    for k, (s, r) in enumerate(zip(shifts, rhs)):
        x1, _ = solver.solve_shifted(gpu.batch, g["_dev"]["J_u"], gpu.dev(r), [s])
        a = xb[k * n:(k + 1) * n].cpu().numpy()
        c = x1.cpu().numpy()
        assert rel_err(a, c) <= 1e-8, (k, info_b)


@pytest.mark.parametrize("name", ["ref8x9", "naca0012_33", "naca0012_33_moving", "naca0004_129",
                                  "min4x5"])
@pytest.mark.parametrize("shift", [0.3 + 0.7j, 2.0, 0.0, 0.0012j])
def test_ringlu_direct_solve(cuda, oracle, golden_grids, name, shift):
    """Ring-block LU resolvent: 1e-10 residual and agreement with SuperLU, both directions."""
    from pyeulerale_b200 import solver

    case = make_case(name, golden_grids, seed=2)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(9)
    b = crandn(rng, (4, M, N))
    lu = solver.RingLU(gpu.batch, tol=1e-10)
    lu.factor(g["_dev"]["J_u"], shift)
    A = bsr_matrix(oracle, g["J_u"]).astype(complex)
    n = A.shape[0]
    bf = b.ravel(order="F")
    for adjoint in (False, True):
        x, rel = lu.solve(gpu.dev(b), adjoint=adjoint)
        got = gpu.host(x, (4, M, N), complex_=True).ravel(order="F")
        op = ((A - np.conj(shift) * sp.eye(n)).T if adjoint else (A - shift * sp.eye(n))).tocsc()
        res = np.linalg.norm(bf - op @ got) / np.linalg.norm(bf)
        assert res <= 1e-10 and rel <= 1e-10, (name, shift, adjoint, res, rel)
        if n <= 20000:
            ref = spla.spsolve(op, bf)
            assert rel_err(got, ref) <= 1e-7, (name, shift, adjoint)


def test_ringlu_odd_ring_size(cuda, oracle):
    """A ring of 4 N unknowns that is not a multiple of the pivot kernel's row tile (N = 13)."""
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200 import solver

    X = G.naca_ogrid(21, 14, 0.12, 1.0, 20.0, 0.01)
    rng = np.random.default_rng(6)
    case = dict(X=X, V=np.zeros_like(X), U=G.perturbed_states(20, 13, 0.5, 1.25, 0.01, rng),
                mach=0.5, aoa=1.25)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    b = crandn(rng, (4, 20, 13))
    lu = solver.RingLU(gpu.batch, tol=1e-10)
    shift = 0.2 + 0.4j
    lu.factor(g["_dev"]["J_u"], shift)
    x, rel = lu.solve(gpu.dev(b))
    A = bsr_matrix(oracle, g["J_u"]).astype(complex)
    op = (A - shift * sp.eye(A.shape[0])).tocsc()
    ref = spla.spsolve(op, b.ravel(order="F"))
    got = gpu.host(x, (4, 20, 13), complex_=True).ravel(order="F")
    assert rel <= 1e-10 and rel_err(got, ref) <= 1e-8, rel


@pytest.mark.parametrize("name", ["naca0012_33", "naca0004_129"])
def test_ringlu_many_matches_single(cuda, golden_grids, name):
    """Concurrent multi-shift factor / solve == one factorisation per shift, both directions."""
    from pyeulerale_b200 import solver

    case = make_case(name, golden_grids, seed=3)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(12)
    shifts = [1j * k for k in (0.01, 0.3, 4.0)] + [0.0, 2.0 - 0.5j]
    rhs = [gpu.dev(crandn(rng, (4, M, N))) for _ in shifts]
    many = solver.RingLUMany(gpu.batch, capacity=len(shifts), tol=1e-10)
    many.factor(g["_dev"]["J_u"], shifts)
    one = solver.RingLU(gpu.batch, tol=1e-10)
    for adjoint in (False, True):
        xs, rels = many.solve(rhs, adjoint=adjoint)
        assert max(rels) <= 1e-10, rels
        for k, s in enumerate(shifts):
            one.factor(g["_dev"]["J_u"], s)
            x1, _ = one.solve(rhs[k], adjoint=adjoint)
            assert rel_err(xs[k].cpu().numpy(), x1.cpu().numpy()) <= 1e-9, (name, k, adjoint)


@pytest.mark.parametrize("grid", ["naca0012_33", "wide"])
def test_ringlu_blocked_matches_single(cuda, golden_grids, grid):
    """16 shifts (two stream groups of 8) take the blocked Gauss-Jordan inversion (64-column
    blocks, ZGEMM trailing updates); one shift at a time takes the unblocked one. Both agree,
    both directions, on K = 128 (16-column panels) and K = 1024 (8-column panels)."""
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200 import solver

    rng = np.random.default_rng(21)
    if grid == "wide":
        X = G.naca_ogrid(9, 257, 0.12, 1.0, 20.0, 0.05)
        case = dict(X=X, V=np.zeros_like(X), U=G.perturbed_states(8, 256, 0.6, 2.0, 0.01, rng),
                    mach=0.6, aoa=2.0)
    else:
        case = make_case(grid, golden_grids, seed=5)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    M, N = gpu.M, gpu.N
    assert (4 * N) % 64 == 0
    shifts = [1j * k for k in np.logspace(-2, 1, 14)] + [0.0, 1.5 - 0.25j]
    rhs = [gpu.dev(crandn(rng, (4, M, N))) for _ in shifts]
    many = solver.RingLUMany(gpu.batch, capacity=len(shifts), tol=1e-10)
    many.factor(g["_dev"]["J_u"], shifts)
    one = solver.RingLU(gpu.batch, tol=1e-10)
    for adjoint in (False, True):
        xs, rels = many.solve(rhs, adjoint=adjoint)
        assert max(rels) <= 1e-10, rels
        for k in (0, 7, 8, 15):  # first and last shift of each group
            one.factor(g["_dev"]["J_u"], shifts[k])
            x1, _ = one.solve(rhs[k], adjoint=adjoint)
            assert rel_err(xs[k].cpu().numpy(), x1.cpu().numpy()) <= 1e-9, (grid, k, adjoint)


def test_ringlu_wide_rings(cuda, oracle):
    """Rings of 4 N = 1024 unknowns (N = 256: the two-rows-per-thread panel path)."""
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200 import solver

    X = G.naca_ogrid(9, 257, 0.12, 1.0, 20.0, 0.05)
    rng = np.random.default_rng(16)
    case = dict(X=X, V=np.zeros_like(X), U=G.perturbed_states(8, 256, 0.6, 2.0, 0.01, rng),
                mach=0.6, aoa=2.0)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    b = crandn(rng, (4, 8, 256))
    A = bsr_matrix(oracle, g["J_u"]).astype(complex)
    for shift in (0.0, 0.05j):
        lu = solver.RingLU(gpu.batch, tol=1e-10)
        lu.factor(g["_dev"]["J_u"], shift)
        for adjoint in (False, True):
            x, rel = lu.solve(gpu.dev(b), adjoint=adjoint)
            op = ((A - np.conj(shift) * sp.eye(A.shape[0])).T if adjoint
                  else (A - shift * sp.eye(A.shape[0]))).tocsc()
            ref = spla.spsolve(op, b.ravel(order="F"))
            got = gpu.host(x, (4, 8, 256), complex_=True).ravel(order="F")
            assert rel <= 1e-10 and rel_err(got, ref) <= 1e-8, (shift, adjoint, rel)


def test_ringlu_graph_replay(cuda, golden_grids, monkeypatch):
    """Eager, captured and replayed factorisations of the same workspace give the same
    solutions for different shifts (the shifts live in device memory, the graph does not)."""
    from pyeulerale_b200 import solver

    case = make_case("naca0012_33", golden_grids, seed=8)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(2)
    rhs = [gpu.dev(crandn(rng, (4, M, N))) for _ in range(2)]
    shifts = [[0.1j, 2.0], [0.3 - 0.2j, 0.0], [1.5j, 0.02], [0.7, 0.05j]]
    many = solver.RingLUMany(gpu.batch, capacity=2, tol=1e-10)
    got = []
    for sh in shifts:  # call 1 eager, call 2 captured, calls 3-4 replayed
        many.factor(g["_dev"]["J_u"], sh)
        got.append([x.cpu().numpy() for x in many.solve(rhs)[0]])
    monkeypatch.setenv("EB_RINGLU_GRAPHS", "0")
    for sh, xs in zip(shifts, got):
        many.factor(g["_dev"]["J_u"], sh)
        ref = [x.cpu().numpy() for x in many.solve(rhs)[0]]
        for a, b in zip(xs, ref):
            assert rel_err(a, b) <= 1e-12, sh
