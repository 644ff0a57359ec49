"""ctypes binding of the CUDA library ``libeuler_b200.so`` (C ABI in include/euler_b200.h).

The library is built in-tree by :func:`pyeulerale_b200.build.build_library`. There is no CPU
fallback: loading fails loudly when the shared library is missing, and every entry point
raises :class:`EulerB200Error` when it returns a negative status.
"""

from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libeuler_b200.so"

EB_OK = 0
EB_ERR_ARG = -1
EB_ERR_CUDA = -2
EB_ERR_NOCONV = -3
EB_ERR_NAN = -4

DIR_STATES, DIR_VERTICES, DIR_VELOCITIES = 0, 1, 2


class EulerB200Error(RuntimeError):
    """A library entry point returned an error status."""

    def __init__(self, name: str, code: int, text: str) -> None:
        super().__init__(f"{name} failed with status {code}: {text}")
        self.code = code


class Instance(ctypes.Structure):
    """``eb_instance``: one grid with its flow parameters (104 bytes)."""

    _fields_ = [
        ("M", ctypes.c_int32), ("N", ctypes.c_int32),
        ("cell_offset", ctypes.c_int64), ("vert_offset", ctypes.c_int64),
        ("wall_offset", ctypes.c_int64),
        ("mach", ctypes.c_double), ("cos_aoa", ctypes.c_double), ("sin_aoa", ctypes.c_double),
        ("k2", ctypes.c_double), ("k4", ctypes.c_double), ("c4", ctypes.c_double),
        ("chord", ctypes.c_double), ("xc", ctypes.c_double), ("zc", ctypes.c_double),
    ]


class Batch(ctypes.Structure):
    """``eb_batch``: a set of instances (single instance passed by value)."""

    _fields_ = [
        ("d_table", ctypes.c_void_p), ("n_inst", ctypes.c_int32), ("max_dim", ctypes.c_int32),
        ("n_cells", ctypes.c_int64), ("n_verts", ctypes.c_int64), ("n_wall", ctypes.c_int64),
        ("single", Instance),
    ]


assert ctypes.sizeof(Instance) == 104


def make_instance(M: int, N: int, mach: float, aoa_deg: float, k2: float = 1.0,
                  k4: float = 1.0 / 32, c4: float = 2.0, chord: float = 1.0,
                  center: tuple[float, float] = (0.0, 0.0), cell_offset: int = 0,
                  vert_offset: int = 0, wall_offset: int = 0) -> Instance:
    """Fills an ``eb_instance``; cos/sin of the angle use the reference's degree factor."""
    a = 0.0174532925199432957692369 * float(aoa_deg)  # deg_to_rad, f90:54
    return Instance(int(M), int(N), int(cell_offset), int(vert_offset), int(wall_offset),
                    float(mach), math.cos(a), math.sin(a), float(k2), float(k4), float(c4),
                    float(chord), float(center[0]), float(center[1]))


def single_batch(inst: Instance) -> Batch:
    b = Batch()
    b.d_table = None
    b.n_inst = 1
    b.max_dim = max(inst.M, inst.N)
    b.n_cells = inst.M * inst.N
    b.n_verts = (inst.M + 1) * (inst.N + 1)
    b.n_wall = inst.N
    b.single = inst
    return b


_SIGNATURES: dict[str, list] = {
    "eb_set_free_stream_state": ["b", "p", "s"],
    "eb_compute_odes": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_odes_untiled": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_forces": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_odes_wrt_mach": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_odes_wrt_states": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_odes_wrt_states_untiled": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_odes_wrt_vertices": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_odes_wrt_velocities": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_forces_wrt_states": ["b", "p", "p", "p", "s"],
    "eb_compute_forces_wrt_vertices": ["b", "p", "p", "p", "s"],
    "eb_apply_odes_wrt_mach_fwd": ["b", "p", "p", "p", "s"],
    "eb_apply_odes_wrt_mach_rev": ["b", "p", "p", "p", "s"],
    "eb_apply_odes_wrt_states_fwd": ["b", "p", "p", "p", "s"],
    "eb_apply_odes_wrt_states_rev": ["b", "p", "p", "p", "s"],
    "eb_apply_odes_wrt_vertices_fwd": ["b", "p", "p", "p", "s"],
    "eb_apply_odes_wrt_vertices_rev": ["b", "p", "p", "p", "s"],
    "eb_apply_forces_wrt_states_fwd": ["b", "p", "p", "p", "s"],
    "eb_apply_forces_wrt_states_rev": ["b", "p", "p", "p", "s"],
    "eb_apply_forces_wrt_vertices_fwd": ["b", "p", "p", "p", "s"],
    "eb_apply_forces_wrt_vertices_rev": ["b", "p", "p", "p", "s"],
    "eb_apply_odes_tangent": ["b", "p", "p", "p", "p", "p", "p", "p", "p", "p", "s"],
    "eb_apply_odes_adjoint": ["b", "p", "p", "p", "p", "i", "p", "p", "p", "p", "s"],
    "eb_convert_odes_wrt_states": ["b", "p", "p", "p", "p", "s"],
    "eb_compute_pressure_coefficients": ["b", "p", "p", "s"],
    "eb_apply_pressure_coefficients_wrt_states_fwd": ["b", "p", "p", "p", "s"],
    "eb_bsr_shifted_spmv": ["i64", "p", "p", "p", "d", "d", "p", "p", "s"],
    "eb_fp64_fma_probe": ["i64", "i", "p", "s"],
    "eb_fp64_mma_probe": ["i64", "i", "p", "s"],
    "eb_zgemm_strided_batched": ["i", "i", "i", "d", "p", "i", "i64", "p", "i", "i64", "d", "p",
                                 "i", "i64", "i", "i", "s"],
    "eb_odes_wrt_mach_dir": ["b", "p", "p", "p", "i", "p", "p", "p", "s"],
    "eb_odes_wrt_states_dir": ["b", "p", "p", "p", "i", "p", "p", "p", "s"],
    "eb_odes_wrt_vertices_dir": ["b", "p", "p", "p", "i", "p", "p", "p", "s"],
    "eb_forces_wrt_states_dir": ["b", "p", "p", "i", "p", "p", "p", "s"],
    "eb_forces_wrt_vertices_dir": ["b", "p", "p", "i", "p", "p", "p", "s"],
}

_CTYPE = {
    "b": ctypes.POINTER(Batch), "p": ctypes.c_void_p, "s": ctypes.c_void_p,
    "i": ctypes.c_int, "i64": ctypes.c_int64, "d": ctypes.c_double,
}


def exported_symbols() -> list[str]:
    """Entry points this binding expects the library to export (all of include/euler_b200.h)."""
    return sorted([*_SIGNATURES, "eb_last_error", "eb_version", "eb_autotune_report"])


_lib = None


def load() -> ctypes.CDLL:
    """Loads the in-tree CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH.name} is not built; run pyeulerale_b200.build.build_library() "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.eb_last_error.restype = ctypes.c_char_p
    lib.eb_last_error.argtypes = []
    lib.eb_version.restype = ctypes.c_char_p
    lib.eb_version.argtypes = []
    for name, args in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = ctypes.c_int
        fn.argtypes = [_CTYPE[a] for a in args]
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    """Calls an entry point and raises EulerB200Error on a negative status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != EB_OK:
        raise EulerB200Error(name, rc, lib.eb_last_error().decode())


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    return None if t is None else t.data_ptr()


def as_f64_view(a: np.ndarray) -> np.ndarray:
    """Fortran-order complex/real array as a flat float64 view (copying if needed)."""
    flat = np.asarray(a).ravel(order="F")
    return flat.view(np.float64) if np.iscomplexobj(flat) else flat.astype(np.float64, copy=False)


def autotune_report() -> str:
    """The launch-variant autotuner's choices so far (``eb_autotune_report``)."""
    lib = load()
    fn = lib.eb_autotune_report
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_char_p, ctypes.c_int]
    n = fn(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    fn(buf, n + 1)
    return buf.value.decode()
