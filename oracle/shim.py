"""f2py-compatible facade over the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The reference's Python class (``src/py_euler_ale/core.py`` of PyEulerALE) reaches its Fortran
module through ``py_euler_ale.euler_ale.spatial_discretization``, an f2py extension built with
``--lower`` (``meson.build:21-35``). This module offers an object with the same 20 procedures,
the same hidden-size calling convention (sizes are taken from the array shapes, as the
``!f2py intent(hide)`` lines of ``src/spatial_discretization.f90`` specify) and the same four
module variables as writable 0-d arrays (``core.py:258-263``), so that the reference's own
``core.py``, unit tests and example drivers run unchanged against the C++ oracle in
``oracle/sd_oracle.cpp``.

Nothing in the product package imports this file.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "libsdoracle.so"


class _Params(ctypes.Structure):
    _fields_ = [("aoa", ctypes.c_double), ("k2", ctypes.c_double),
                ("k4", ctypes.c_double), ("c4", ctypes.c_double)]


def build() -> Path:
    """Compiles the oracle library with ``make`` if it is missing or stale."""
    src = _HERE / "sd_oracle.cpp"
    if not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


_lib = None


def load_library() -> ctypes.CDLL:
    """Loads (building if needed) the oracle shared library."""
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(_LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        pp = ctypes.POINTER(_Params)
        i, d, L = ctypes.c_int, ctypes.c_double, ctypes.c_long
        sig = {
            "sdo_set_threads": (None, [i]),
            "sdo_max_threads": (i, []),
            "sdo_set_free_stream_state": (None, [pp, d, d, i, i, dp]),
            "sdo_compute_odes": (None, [pp, d, d, i, i, dp, dp, dp, dp]),
            "sdo_compute_odes_wrt_mach": (None, [pp, d, d, i, i, dp, dp, dp, dp]),
            "sdo_apply_odes_wrt_mach_fwd": (None, [i, i, dp, dp, dp]),
            "sdo_apply_odes_wrt_mach_rev": (None, [i, i, dp, dp, dp]),
            "sdo_compute_odes_wrt_states": (None, [pp, d, d, i, i, dp, dp, dp, dp]),
            "sdo_convert_odes_wrt_states": (L, [i, i, dp, dp, ip, ip, L]),
            "sdo_apply_odes_wrt_states_fwd": (None, [i, i, dp, dp, dp]),
            "sdo_apply_odes_wrt_states_rev": (None, [i, i, dp, dp, dp]),
            "sdo_compute_odes_wrt_vertices": (None, [pp, d, d, i, i, dp, dp, dp, dp]),
            "sdo_compute_odes_wrt_velocities": (None, [pp, d, d, i, i, dp, dp, dp, dp]),
            "sdo_apply_odes_wrt_vertices_fwd": (None, [i, i, dp, dp, dp]),
            "sdo_apply_odes_wrt_vertices_rev": (None, [i, i, dp, dp, dp]),
            "sdo_compute_forces": (None, [i, i, dp, dp, dp]),
            "sdo_compute_forces_wrt_states": (None, [i, i, dp, dp, dp]),
            "sdo_apply_forces_wrt_states_fwd": (None, [i, i, dp, dp, dp]),
            "sdo_apply_forces_wrt_states_rev": (None, [i, i, dp, dp, dp]),
            "sdo_compute_forces_wrt_vertices": (None, [i, i, dp, dp, dp]),
            "sdo_apply_forces_wrt_vertices_fwd": (None, [i, i, dp, dp, dp]),
            "sdo_apply_forces_wrt_vertices_rev": (None, [i, i, dp, dp, dp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        threads = int(os.environ.get("SDO_THREADS", "1"))
        lib.sdo_set_threads(threads)
        _lib = lib
    return _lib


def _in(a, dtype=np.complex128) -> np.ndarray:
    """intent(in): f2py copies any array-like into a Fortran-contiguous array of the type."""
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def _inout(a, dtype=np.complex128) -> np.ndarray:
    """intent(inout): f2py requires a Fortran-contiguous array of exactly the type."""
    if not isinstance(a, np.ndarray):
        raise ValueError("intent(inout) argument must be an array")
    if a.dtype != dtype:
        raise ValueError(f"intent(inout) array must have dtype {np.dtype(dtype).name}")
    if not (a.flags.f_contiguous or a.ndim <= 1 and a.flags.c_contiguous):
        raise ValueError("failed to initialize intent(inout) array -- input not fortran contiguous")
    return a


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


class SpatialDiscretizationModule:
    """Stand-in for the f2py module object ``euler_ale.spatial_discretization``."""

    def __init__(self) -> None:
        self._lib = load_library()
        # Module variables (f90:63-66); `aoa` has no initializer in the reference.
        self.aoa = np.zeros((), dtype=np.float64)
        self.jst_k2 = np.array(1.0)
        self.jst_k4 = np.array(1.0 / 32)
        self.jst_c4 = np.array(2.0)

    # -- helpers ---------------------------------------------------------------------------
    def _params(self) -> _Params:
        return _Params(float(self.aoa), float(self.jst_k2), float(self.jst_k4),
                       float(self.jst_c4))

    @staticmethod
    def _mn_states(states: np.ndarray) -> tuple[int, int]:
        return int(states.shape[1]), int(states.shape[2])

    def _field_call(self, name, mach, vertices, velocities, states, out, out_shape_fn,
                    out_dtype=np.float64):
        mach = complex(mach)
        X, V, U = _in(vertices), _in(velocities), _in(states)
        M, N = self._mn_states(U)
        out = _inout(out, out_dtype)
        if out.shape != out_shape_fn(M, N):
            raise ValueError(f"{name}: output has shape {out.shape}")
        p = self._params()
        getattr(self._lib, name)(ctypes.byref(p), mach.real, mach.imag, M, N,
                                 _ptr(X), _ptr(V), _ptr(U), _ptr(out))

    # -- procedures (f90:68-87) ------------------------------------------------------------
    def set_free_stream_state(self, mach, states) -> None:
        mach = complex(mach)
        U = _inout(states)
        M, N = self._mn_states(U)
        p = self._params()
        self._lib.sdo_set_free_stream_state(ctypes.byref(p), mach.real, mach.imag, M, N, _ptr(U))

    def compute_odes(self, mach, vertices, velocities, states, odes) -> None:
        self._field_call("sdo_compute_odes", mach, vertices, velocities, states, odes,
                         lambda M, N: (4, M, N), np.complex128)

    def compute_odes_wrt_mach(self, mach, vertices, velocities, states, jacs) -> None:
        self._field_call("sdo_compute_odes_wrt_mach", mach, vertices, velocities, states, jacs,
                         lambda M, N: (4, 1, M, N))

    def compute_odes_wrt_states(self, mach, vertices, velocities, states, jacs) -> None:
        self._field_call("sdo_compute_odes_wrt_states", mach, vertices, velocities, states,
                         jacs, lambda M, N: (4, 4, M, N, 9))

    def compute_odes_wrt_vertices(self, mach, vertices, velocities, states, jacs) -> None:
        self._field_call("sdo_compute_odes_wrt_vertices", mach, vertices, velocities, states,
                         jacs, lambda M, N: (4, 2, M, N, 4))

    def compute_odes_wrt_velocities(self, mach, vertices, velocities, states, jacs) -> None:
        self._field_call("sdo_compute_odes_wrt_velocities", mach, vertices, velocities, states,
                         jacs, lambda M, N: (4, 2, M, N, 4))

    def apply_odes_wrt_mach_fwd(self, jacs, d_mach, d_odes) -> None:
        J = _in(jacs, np.float64)
        dm = _in(d_mach).reshape(1)
        y = _inout(d_odes)
        self._lib.sdo_apply_odes_wrt_mach_fwd(y.shape[1], y.shape[2], _ptr(J), _ptr(dm), _ptr(y))

    def apply_odes_wrt_mach_rev(self, jacs, d_odes, d_mach) -> None:
        J = _in(jacs, np.float64)
        w = _in(d_odes)
        dm = _inout(d_mach)
        self._lib.sdo_apply_odes_wrt_mach_rev(w.shape[1], w.shape[2], _ptr(J), _ptr(w), _ptr(dm))

    def convert_odes_wrt_states(self, jacs, data, indices, index_pointers) -> None:
        J = _in(jacs, np.float64)
        M, N = int(J.shape[2]), int(J.shape[3])
        data = _inout(data, np.float64)
        indices = _inout(indices, np.int32)
        index_pointers = _inout(index_pointers, np.int32)
        got = self._lib.sdo_convert_odes_wrt_states(M, N, _ptr(J), _ptr(data), _iptr(indices),
                                                    _iptr(index_pointers), indices.shape[0])
        if got < 0:
            raise ValueError("convert_odes_wrt_states: output arrays too small")

    def apply_odes_wrt_states_fwd(self, jacs, d_states, d_odes) -> None:
        J = _in(jacs, np.float64)
        x = _in(d_states)
        y = _inout(d_odes)
        self._lib.sdo_apply_odes_wrt_states_fwd(y.shape[1], y.shape[2], _ptr(J), _ptr(x), _ptr(y))

    def apply_odes_wrt_states_rev(self, jacs, d_odes, d_states) -> None:
        J = _in(jacs, np.float64)
        w = _in(d_odes)
        y = _inout(d_states)
        self._lib.sdo_apply_odes_wrt_states_rev(w.shape[1], w.shape[2], _ptr(J), _ptr(w), _ptr(y))

    def apply_odes_wrt_vertices_fwd(self, jacs, d_vertices, d_odes) -> None:
        J = _in(jacs, np.float64)
        x = _in(d_vertices)
        y = _inout(d_odes)
        self._lib.sdo_apply_odes_wrt_vertices_fwd(y.shape[1], y.shape[2], _ptr(J), _ptr(x),
                                                  _ptr(y))

    def apply_odes_wrt_vertices_rev(self, jacs, d_odes, d_vertices) -> None:
        J = _in(jacs, np.float64)
        w = _in(d_odes)
        y = _inout(d_vertices)
        self._lib.sdo_apply_odes_wrt_vertices_rev(w.shape[1], w.shape[2], _ptr(J), _ptr(w),
                                                  _ptr(y))

    def compute_forces(self, vertices, states, forces) -> None:
        X, U = _in(vertices), _in(states)
        F = _inout(forces)
        M, N = self._mn_states(U)
        self._lib.sdo_compute_forces(M, N, _ptr(X), _ptr(U), _ptr(F))

    def compute_forces_wrt_states(self, vertices, states, jacs) -> None:
        X, U = _in(vertices), _in(states)
        J = _inout(jacs, np.float64)
        M, N = self._mn_states(U)
        self._lib.sdo_compute_forces_wrt_states(M, N, _ptr(X), _ptr(U), _ptr(J))

    def compute_forces_wrt_vertices(self, vertices, states, jacs) -> None:
        X, U = _in(vertices), _in(states)
        J = _inout(jacs, np.float64)
        M, N = self._mn_states(U)
        self._lib.sdo_compute_forces_wrt_vertices(M, N, _ptr(X), _ptr(U), _ptr(J))

    def apply_forces_wrt_states_fwd(self, jacs, d_states, d_forces) -> None:
        J = _in(jacs, np.float64)
        x = _in(d_states)
        y = _inout(d_forces)
        self._lib.sdo_apply_forces_wrt_states_fwd(x.shape[1], x.shape[2], _ptr(J), _ptr(x),
                                                  _ptr(y))

    def apply_forces_wrt_states_rev(self, jacs, d_forces, d_states) -> None:
        J = _in(jacs, np.float64)
        w = _in(d_forces)
        y = _inout(d_states)
        self._lib.sdo_apply_forces_wrt_states_rev(y.shape[1], y.shape[2], _ptr(J), _ptr(w),
                                                  _ptr(y))

    def apply_forces_wrt_vertices_fwd(self, jacs, d_vertices, d_forces) -> None:
        J = _in(jacs, np.float64)
        x = _in(d_vertices)
        y = _inout(d_forces)
        self._lib.sdo_apply_forces_wrt_vertices_fwd(x.shape[1] - 1, x.shape[2] - 1, _ptr(J),
                                                    _ptr(x), _ptr(y))

    def apply_forces_wrt_vertices_rev(self, jacs, d_forces, d_vertices) -> None:
        J = _in(jacs, np.float64)
        w = _in(d_forces)
        y = _inout(d_vertices)
        self._lib.sdo_apply_forces_wrt_vertices_rev(y.shape[1] - 1, y.shape[2] - 1, _ptr(J),
                                                    _ptr(w), _ptr(y))
