"""Scratch-free GMRES entry point (``eb_gmres_solve_noalloc``) against ``eb_gmres_solve`` (GPU).

Callers that cannot allocate device memory (their memory belongs to another runtime's pool, or
their loop may not allocate once running) use the entry point whose workspace is the library's
fixed 48 MiB device array. Two calls in a row must give the same solutions as the allocating
entry point: the array keeps the previous call's contents, so anything left over must not leak
into the next solve. After its first call on a device, a call must leave the device's free
memory unchanged. This file is collected last so that a failure here cannot hide others.
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


def test_noalloc_two_instances_allocates_nothing(cuda, golden_grids):
    """A batch of two instances of different size (systems mapped by sys_inst, sizes from the
    host table): the same solutions as the allocating entry point on two calls in a row, and
    the second call leaves the device's free memory and torch's allocation unchanged."""
    from pyeulerale_b200 import grid as G
    from pyeulerale_b200 import solver
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec

    rng = np.random.default_rng(31)
    grids = [golden_grids["naca0012_8x9"], G.naca_ogrid(13, 17, 0.08, 1.0, 15.0, 0.02)]
    specs = [InstanceSpec(grids[0], 0.5, 1.25), InstanceSpec(grids[1], 0.4, -1.0)]
    inst = InstanceSet(specs)
    states = [G.perturbed_states(s.M, s.N, s.mach, s.aoa_deg, 0.01, rng) for s in specs]
    dX = cuda.from_numpy(inst.pack_vertices()).cuda()
    dV = cuda.zeros_like(dX)
    dU = cuda.from_numpy(inst.pack_cells(states)).cuda()
    J = cuda.zeros(144 * inst.n_cells, dtype=cuda.float64, device="cuda")
    inst.call("eb_compute_odes_wrt_states", dX, dV, dU, J)
    sys_inst = [1, 0, 1]
    shifts = [2.0 + 1.0j, 1.5, 3.0j]
    sizes = [8 * specs[i].M * specs[i].N for i in sys_inst]
    rhs = cuda.from_numpy(rng.standard_normal(sum(sizes))).cuda()
    kw = dict(sys_inst=sys_inst, host_table=inst.host_table)
    ref, _ = solver.solve_shifted(inst.batch, J, rhs, shifts, **kw)
    x = cuda.full_like(rhs, np.nan)
    solver.solve_shifted_noalloc(inst.batch, J, rhs, shifts, x=x, **kw)  # first call: set-up
    cuda.cuda.synchronize()
    free0, alloc0 = cuda.cuda.mem_get_info()[0], cuda.cuda.memory_allocated()
    x.fill_(np.nan)
    got, info = solver.solve_shifted_noalloc(inst.batch, J, rhs, shifts, x=x, **kw)
    cuda.cuda.synchronize()
    assert cuda.cuda.mem_get_info()[0] == free0
    assert cuda.cuda.memory_allocated() == alloc0
    assert got.data_ptr() == x.data_ptr()
    assert info.max_rel_residual <= 1e-10
    assert rel_err(got.cpu().numpy(), ref.cpu().numpy()) <= 1e-10, info


def test_noalloc_rejects_oversized_systems(cuda):
    from pyeulerale_b200 import _lib, solver

    inst = _lib.make_instance(256, 256, 0.5, 0.0)
    b = _lib.single_batch(inst)
    J = cuda.zeros(8, dtype=cuda.float64, device="cuda")
    rhs = cuda.zeros(8 * 256 * 256, dtype=cuda.float64, device="cuda")
    with pytest.raises(_lib.EulerB200Error, match="48 MiB"):
        solver.solve_shifted_noalloc(b, J, rhs, [1.0], restart=60)
