"""Host-side logic and the C ABI surface (CPU only, no kernel launches)."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from pyeulerale_b200 import _lib, grid

ROOT = Path(__file__).resolve().parent.parent


def header_symbols() -> set[str]:
    text = (ROOT / "include" / "euler_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(eb_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_symbol():
    from pyeulerale_b200.build import build_library

    build_library()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    declared = header_symbols()
    assert len(declared) >= 30
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    bound = set(_lib.exported_symbols()) | {  # bound in pyeulerale_b200/solver.py
        "eb_gmres_solve", "eb_gmres_workspace_bytes", "eb_gmres_solve_noalloc",
        "eb_ringlu_factor", "eb_ringlu_solve", "eb_ringlu_workspace_bytes",
        "eb_ringlu_factor_many", "eb_ringlu_solve_many", "eb_ptc_run",
        "eb_ptc_workspace_bytes", "eb_gmres_solve_anchored", "eb_gmres_anchored_aux_bytes"}
    assert declared <= bound, declared - bound


@pytest.mark.parametrize("entry,n_arrays", [("eb_compute_odes", 4),
                                            ("eb_apply_odes_wrt_states_rev", 3),
                                            ("eb_apply_odes_wrt_vertices_fwd", 3),
                                            ("eb_compute_odes_wrt_states", 4)])
def test_misaligned_arrays_rejected_before_any_launch(entry, n_arrays):
    """Arrays are accessed as 16-byte vectors: an array 8 bytes off a 16-byte boundary is an
    argument error returned by the host-side checks (the fake addresses are never touched)."""
    from pyeulerale_b200.build import build_library

    build_library()
    batch = _lib.single_batch(_lib.make_instance(8, 9, 0.5, 1.25))
    good, bad = 0x7F0000000000, 0x7F0000000008
    args = [good] * n_arrays
    args[-1] = bad
    with pytest.raises(_lib.EulerB200Error, match="16-byte aligned") as err:
        _lib.call(entry, ctypes.byref(batch), *args, None)
    assert err.value.code == -1


@pytest.mark.parametrize("entry", ["eb_apply_odes_wrt_states_rev", "eb_apply_odes_wrt_states_fwd",
                                   "eb_apply_odes_wrt_vertices_rev", "eb_apply_odes_wrt_mach_fwd"])
def test_batch_without_max_dim_rejected_before_any_launch(entry):
    """The per-instance product kernels size their grid rows by max_dim: a batch of several
    instances without it is an argument error returned by the host-side checks (the fake table
    and array addresses are never touched)."""
    from pyeulerale_b200.build import build_library

    build_library()
    batch = _lib.single_batch(_lib.make_instance(8, 9, 0.5, 1.25))
    batch.n_inst, batch.d_table, batch.max_dim = 2, 0x7F0000000000, 0
    with pytest.raises(_lib.EulerB200Error, match="max_dim") as err:
        _lib.call(entry, ctypes.byref(batch), 0x7F0000001000, 0x7F0000002000, 0x7F0000003000,
                  None)
    assert err.value.code == -1


def test_struct_layouts_match_header():
    assert ctypes.sizeof(_lib.Instance) == 104
    assert _lib.Instance.wall_offset.offset == 24
    assert _lib.Instance.mach.offset == 32
    assert _lib.Batch.single.offset == 40
    assert _lib.Batch.max_dim.offset == 12


def test_plot3d_round_trip(tmp_path, golden_grids):
    X = golden_grids["naca0012_8x9"]
    grid.write_plot3d(tmp_path / "g.plot3d", X)
    Y = grid.read_plot3d(tmp_path / "g.plot3d")
    np.testing.assert_array_equal(X, Y)
    assert Y.flags.f_contiguous


def test_naca_ogrid_is_closed_and_sized():
    X = grid.naca_ogrid(33, 41, thickness=0.04, chord=10.0, far_radius=200.0,
                        first_spacing=0.1)
    assert X.shape == (2, 33, 41)
    np.testing.assert_array_equal(X[:, :, 0], X[:, :, -1])
    r = np.hypot(X[0, -1, :] - 5.0, X[1, -1, :])
    np.testing.assert_allclose(r, 200.0)
    first = np.hypot(*(X[:, 1, :] - X[:, 0, :]))
    assert np.all(first > 0.05) and np.all(first < 0.2)
    # trailing edge -> lower side first
    assert X[1, 0, X.shape[2] // 4] < 0 < X[1, 0, 3 * X.shape[2] // 4]


def test_free_stream_state_matches_formula():
    s = grid.free_stream_state(0.5, 0.0)
    assert s[0] == 1.0 and s[2] == 0.0
    np.testing.assert_allclose(s[3], 1 / 0.4 + 1.4 * 0.25 / 2)


def test_make_instance_angle_factor():
    inst = _lib.make_instance(8, 9, 0.5, 90.0)
    assert abs(inst.cos_aoa) < 1e-15 and inst.sin_aoa == 1.0
    b = _lib.single_batch(inst)
    assert (b.n_cells, b.n_verts, b.n_wall) == (72, 90, 9)


def test_dropin_requires_cuda(golden_grids):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from pyeulerale_b200 import SpatialDiscretization

    with pytest.raises(RuntimeError, match="CUDA"):
        SpatialDiscretization(golden_grids["naca0012_8x9"])


@pytest.mark.parametrize("field,value", [("check_every", 0), ("restart", 0),
                                         ("max_iterations", 0), ("tol", 0.0)])
def test_gmres_bad_options_rejected_before_any_launch(field, value):
    """GMRES options out of range (check_every = 0 would divide by zero on the host) are an
    argument error returned before any launch, for both GMRES entry points (the fake device
    addresses are never touched)."""
    from pyeulerale_b200 import solver
    from pyeulerale_b200.build import build_library

    build_library()
    lib = solver._bind()
    batch = _lib.single_batch(_lib.make_instance(8, 9, 0.5, 1.25))
    opts = solver.GmresOptions(1e-10, 30, 100, 10, 0)
    setattr(opts, field, value)
    infos = (solver.GmresInfo * 1)()
    shifts = np.array([1.0, 0.0])
    fake = 0x7F0000000000
    rc = lib.eb_gmres_solve(ctypes.byref(batch), None, fake, 1, None, shifts.ctypes.data, 0,
                            fake, fake, ctypes.byref(opts), fake, 1 << 30, infos, None)
    assert rc == _lib.EB_ERR_ARG
    assert "bad options" in lib.eb_last_error().decode()
    lib.eb_gmres_solve_noalloc.restype = ctypes.c_int
    lib.eb_gmres_solve_noalloc.argtypes = [
        ctypes.POINTER(_lib.Batch), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.POINTER(solver.GmresOptions), ctypes.POINTER(solver.GmresInfo), ctypes.c_void_p]
    rc = lib.eb_gmres_solve_noalloc(ctypes.byref(batch), None, fake, 1, None,
                                    shifts.ctypes.data, 0, fake, fake, ctypes.byref(opts),
                                    infos, None)
    assert rc == _lib.EB_ERR_ARG
    assert "bad options" in lib.eb_last_error().decode()


def test_anchor_shifts_groups_by_magnitude():
    """Anchors: consecutive groups of shifts ordered by magnitude, each anchored at the group's
    geometric-mean magnitude in its middle shift's direction; at most 8 systems per anchor."""
    from pyeulerale_b200.solver import anchor_shifts

    ks = np.logspace(-2, 1, 64)
    shifts = 1j * ks[::-1]  # any order
    anchors, sa = anchor_shifts(shifts, 4)
    assert len(anchors) == 16 and np.bincount(sa).tolist() == [4] * 16
    for a in range(16):
        g = shifts[sa == a]
        assert np.all(np.abs(g.real) == 0) and abs(anchors[a].real) == 0
        assert min(abs(g)) <= abs(anchors[a]) <= max(abs(g))
        np.testing.assert_allclose(abs(anchors[a]), np.exp(np.mean(np.log(abs(g)))), rtol=1e-14)
    anchors, sa = anchor_shifts([0.0, 1j, 2j], 2)
    assert sa.tolist() == [0, 0, 1] and anchors[0] == 0.5j and anchors[1] == 2j
    with pytest.raises(ValueError):
        anchor_shifts(shifts, 9)


def test_anchored_aux_bytes_validates_assignment():
    """eb_gmres_anchored_aux_bytes (host only) rejects anchors out of range and more than eight
    systems on one anchor, and grows with the systems per anchor."""
    from pyeulerale_b200.solver import _bind_anchored

    lib = _bind_anchored()
    def aux(sa, n_anchors):
        a = np.ascontiguousarray(sa, dtype=np.int32)
        return lib.eb_gmres_anchored_aux_bytes(32, 32, len(a), n_anchors, a.ctypes.data)
    assert aux([0, 0, 1, 1], 2) > 0
    assert aux([0] * 8, 1) > aux([0] * 4, 1) > 0
    assert aux([0] * 9, 1) == -1
    assert aux([0, 2], 2) == -1
    assert aux([-1, 0], 2) == -1
