"""Scratch-free GMRES entry point (``eb_gmres_solve_noalloc``) against ``eb_gmres_solve`` (GPU).

Callers that cannot allocate device memory (their memory belongs to another runtime's pool, or
their loop may not allocate once running) use the entry point whose workspace is the library's
fixed 48 MiB device array. Two calls in a row must give the same solutions as the allocating
entry point: the array keeps the previous call's contents, so anything left over must not leak
into the next solve. This file is collected last so that a failure here cannot hide others.
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import Gpu, crandn, make_case, rel_err

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_solver_twice(cuda, golden_grids):
    from pyeulerale_b200 import _lib, solver

    case = make_case("ref8x9", golden_grids, seed=3)
    gpu = Gpu(cuda, case)
    g = gpu.evaluate()
    J = g["_dev"]["J_u"]
    M, N = gpu.M, gpu.N
    rng = np.random.default_rng(21)
    calls = [([0.3 + 0.7j, 2.0], False), ([0.05j, 1.5 - 0.5j, 4.0], True)]
    for shifts, adjoint in calls:
        rhs = cuda.cat([gpu.dev(crandn(rng, (4, M, N))) for _ in shifts])
        ref, info_ref = solver.solve_shifted(gpu.batch, J, rhs, shifts, adjoint=adjoint,
                                             sys_inst=[0] * len(shifts))
        x = cuda.full_like(rhs, np.nan)  # stale values must not matter
        got, info = solver.solve_shifted_noalloc(gpu.batch, J, rhs, shifts, adjoint=adjoint,
                                                 sys_inst=[0] * len(shifts), x=x)
        assert info.max_rel_residual <= 1e-10
        assert rel_err(got.cpu().numpy(), ref.cpu().numpy()) <= 1e-10, (info, info_ref)


def test_noalloc_rejects_oversized_systems(cuda):
    from pyeulerale_b200 import _lib, solver

    inst = _lib.make_instance(256, 256, 0.5, 0.0)
    b = _lib.single_batch(inst)
    J = cuda.zeros(8, dtype=cuda.float64, device="cuda")
    rhs = cuda.zeros(8 * 256 * 256, dtype=cuda.float64, device="cuda")
    with pytest.raises(_lib.EulerB200Error, match="48 MiB"):
        solver.solve_shifted_noalloc(b, J, rhs, [1.0], restart=60)
