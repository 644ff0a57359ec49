"""The reference's native-module interface, backed by the CUDA library.

PyEulerALE's class reaches its Fortran code as ``py_euler_ale.euler_ale.spatial_discretization``
(an f2py extension, ``meson.build:21-35``, imported at ``src/py_euler_ale/core.py:17``). This
module offers an object with the same 20 procedures (f90:68-87), the same calling convention
(array sizes taken from the arrays, results written in place into the caller's Fortran-ordered
arrays, complex128 fields and float64 Jacobians) and the same four module variables as writable
0-d arrays (``aoa``, ``jst_k2``, ``jst_k4``, ``jst_c4``; f90:63-66). Binding it in place of the
Fortran extension runs the reference's own ``core.py`` on the B200.

Every call copies its host inputs to the device, launches the kernel through the C ABI and
copies the result back. The complex fields' imaginary parts are not used: the reference stores
states, vertices and velocities as complex only for its complex-step differentiation, and its
class only ever passes real values (``core.py:159-211``).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _inout(a, dtype=np.complex128) -> np.ndarray:
    if not isinstance(a, np.ndarray) or a.dtype != dtype:
        raise ValueError(f"intent(inout) argument must be a {np.dtype(dtype).name} array")
    if not (a.flags.f_contiguous or (a.ndim <= 1 and a.flags.c_contiguous)):
        raise ValueError("failed to initialize intent(inout) array -- input not fortran contiguous")
    return a


class SpatialDiscretizationModule:
    """Stand-in for ``euler_ale.spatial_discretization`` running on the GPU."""

    def __init__(self) -> None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("the B200 module needs a CUDA device; there is no CPU fallback")
        self._torch = torch
        _lib.load()
        self.aoa = np.zeros((), dtype=np.float64)
        self.jst_k2 = np.array(1.0)
        self.jst_k4 = np.array(1.0 / 32)
        self.jst_c4 = np.array(2.0)

    # ---- helpers ----------------------------------------------------------------------------
    def _batch(self, M: int, N: int, mach: complex = 0.5) -> _lib.Batch:
        inst = _lib.make_instance(M, N, complex(mach).real, float(self.aoa), float(self.jst_k2),
                                  float(self.jst_k4), float(self.jst_c4))
        return _lib.single_batch(inst)

    def _dev_real(self, a) -> "object":
        a = np.asarray(a)
        flat = np.ascontiguousarray(a.real.ravel(order="F"), dtype=np.float64)
        return self._torch.from_numpy(flat).cuda()

    def _dev_complex(self, a) -> "object":
        flat = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).ravel(order="F"))
        return self._torch.from_numpy(flat.view(np.float64)).cuda()

    def _empty(self, n: int):
        return self._torch.zeros(n, dtype=self._torch.float64, device="cuda")

    def _call(self, name, b, *args) -> None:
        conv = [a.data_ptr() if hasattr(a, "data_ptr") else a for a in args]
        _lib.call(name, ctypes.byref(b), *conv, None)

    @staticmethod
    def _store_real(out: np.ndarray, dev) -> None:
        out[...] = np.reshape(dev.cpu().numpy(), out.shape, order="F")

    @staticmethod
    def _store_complex(out: np.ndarray, dev) -> None:
        out[...] = np.reshape(dev.cpu().numpy().view(np.complex128), out.shape, order="F")

    def _fields(self, vertices, velocities, states):
        U = np.asarray(states)
        M, N = U.shape[1], U.shape[2]
        return M, N, self._dev_real(vertices), self._dev_real(velocities), self._dev_real(U)

    # ---- procedures ---------------------------------------------------------------------------
    def set_free_stream_state(self, mach, states) -> None:
        U = _inout(states)
        b = self._batch(U.shape[1], U.shape[2], mach)
        d = self._empty(U.size * 4)
        self._call("eb_set_free_stream_state", b, d)
        U[...] = np.reshape(d.cpu().numpy(), U.shape, order="F")

    def compute_odes(self, mach, vertices, velocities, states, odes) -> None:
        M, N, X, V, U = self._fields(vertices, velocities, states)
        R = self._empty(4 * M * N)
        self._call("eb_compute_odes", self._batch(M, N, mach), X, V, U, R)
        _inout(odes)[...] = np.reshape(R.cpu().numpy(), odes.shape, order="F")

    def _jacobian(self, name, size, mach, vertices, velocities, states, jacs) -> None:
        M, N, X, V, U = self._fields(vertices, velocities, states)
        J = self._empty(size(M, N))
        self._call(name, self._batch(M, N, mach), X, V, U, J)
        self._store_real(_inout(jacs, np.float64), J)

    def compute_odes_wrt_mach(self, mach, vertices, velocities, states, jacs) -> None:
        self._jacobian("eb_compute_odes_wrt_mach", lambda M, N: 4 * M * N, mach, vertices,
                       velocities, states, jacs)

    def compute_odes_wrt_states(self, mach, vertices, velocities, states, jacs) -> None:
        self._jacobian("eb_compute_odes_wrt_states", lambda M, N: 144 * M * N, mach, vertices,
                       velocities, states, jacs)

    def compute_odes_wrt_vertices(self, mach, vertices, velocities, states, jacs) -> None:
        self._jacobian("eb_compute_odes_wrt_vertices", lambda M, N: 32 * M * N, mach, vertices,
                       velocities, states, jacs)

    def compute_odes_wrt_velocities(self, mach, vertices, velocities, states, jacs) -> None:
        self._jacobian("eb_compute_odes_wrt_velocities", lambda M, N: 32 * M * N, mach,
                       vertices, velocities, states, jacs)

    def compute_forces(self, vertices, states, forces) -> None:
        U = np.asarray(states)
        M, N = U.shape[1], U.shape[2]
        F = self._empty(2 * N)
        self._call("eb_compute_forces", self._batch(M, N), self._dev_real(vertices),
                   self._dev_real(U), F, None)
        _inout(forces)[...] = np.reshape(F.cpu().numpy(), forces.shape, order="F")

    def compute_forces_wrt_states(self, vertices, states, jacs) -> None:
        U = np.asarray(states)
        M, N = U.shape[1], U.shape[2]
        J = self._empty(8 * N)
        self._call("eb_compute_forces_wrt_states", self._batch(M, N), self._dev_real(vertices),
                   self._dev_real(U), J)
        self._store_real(_inout(jacs, np.float64), J)

    def compute_forces_wrt_vertices(self, vertices, states, jacs) -> None:
        U = np.asarray(states)
        M, N = U.shape[1], U.shape[2]
        J = self._empty(8 * N)
        self._call("eb_compute_forces_wrt_vertices", self._batch(M, N),
                   self._dev_real(vertices), self._dev_real(U), J)
        self._store_real(_inout(jacs, np.float64), J)

    def _apply(self, name, M, N, jacs, vec, out) -> None:
        J = self._torch.from_numpy(np.ascontiguousarray(
            np.asarray(jacs, dtype=np.float64).ravel(order="F"))).cuda()
        x = self._dev_complex(vec)
        y = self._empty(2 * out.size)
        self._call(name, self._batch(M, N), J, x, y)
        self._store_complex(_inout(out), y)

    def apply_odes_wrt_mach_fwd(self, jacs, d_mach, d_odes) -> None:
        self._apply("eb_apply_odes_wrt_mach_fwd", d_odes.shape[1], d_odes.shape[2], jacs,
                    np.reshape(d_mach, (1,)), d_odes)

    def apply_odes_wrt_mach_rev(self, jacs, d_odes, d_mach) -> None:
        w = np.asarray(d_odes)
        self._apply("eb_apply_odes_wrt_mach_rev", w.shape[1], w.shape[2], jacs, w, d_mach)

    def apply_odes_wrt_states_fwd(self, jacs, d_states, d_odes) -> None:
        self._apply("eb_apply_odes_wrt_states_fwd", d_odes.shape[1], d_odes.shape[2], jacs,
                    d_states, d_odes)

    def apply_odes_wrt_states_rev(self, jacs, d_odes, d_states) -> None:
        self._apply("eb_apply_odes_wrt_states_rev", d_states.shape[1], d_states.shape[2], jacs,
                    d_odes, d_states)

    def apply_odes_wrt_vertices_fwd(self, jacs, d_vertices, d_odes) -> None:
        self._apply("eb_apply_odes_wrt_vertices_fwd", d_odes.shape[1], d_odes.shape[2], jacs,
                    d_vertices, d_odes)

    def apply_odes_wrt_vertices_rev(self, jacs, d_odes, d_vertices) -> None:
        w = np.asarray(d_odes)
        self._apply("eb_apply_odes_wrt_vertices_rev", w.shape[1], w.shape[2], jacs, w,
                    d_vertices)

    def apply_forces_wrt_states_fwd(self, jacs, d_states, d_forces) -> None:
        x = np.asarray(d_states)
        self._apply("eb_apply_forces_wrt_states_fwd", x.shape[1], x.shape[2], jacs, x, d_forces)

    def apply_forces_wrt_states_rev(self, jacs, d_forces, d_states) -> None:
        self._apply("eb_apply_forces_wrt_states_rev", d_states.shape[1], d_states.shape[2],
                    jacs, d_forces, d_states)

    def apply_forces_wrt_vertices_fwd(self, jacs, d_vertices, d_forces) -> None:
        x = np.asarray(d_vertices)
        self._apply("eb_apply_forces_wrt_vertices_fwd", x.shape[1] - 1, x.shape[2] - 1, jacs,
                    x, d_forces)

    def apply_forces_wrt_vertices_rev(self, jacs, d_forces, d_vertices) -> None:
        self._apply("eb_apply_forces_wrt_vertices_rev", d_vertices.shape[1] - 1,
                    d_vertices.shape[2] - 1, jacs, d_forces, d_vertices)

    def convert_odes_wrt_states(self, jacs, data, indices, index_pointers) -> None:
        J = np.asarray(jacs, dtype=np.float64)
        M, N = J.shape[2], J.shape[3]
        dJ = self._torch.from_numpy(np.ascontiguousarray(J.ravel(order="F"))).cuda()
        nnzb = (9 * M - 6) * N
        d_data = self._empty(16 * nnzb)
        d_idx = self._torch.zeros(nnzb, dtype=self._torch.int32, device="cuda")
        d_ptr = self._torch.zeros(M * N + 1, dtype=self._torch.int32, device="cuda")
        self._call("eb_convert_odes_wrt_states", self._batch(M, N), dJ, d_data, d_idx, d_ptr)
        self._store_real(_inout(data, np.float64), d_data)
        _inout(indices, np.int32)[...] = d_idx.cpu().numpy()
        _inout(index_pointers, np.int32)[...] = d_ptr.cpu().numpy()
