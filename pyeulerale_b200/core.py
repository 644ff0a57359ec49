"""Drop-in ``SpatialDiscretization`` backed by the B200 CUDA library.

Same constructor, properties and methods as the reference class
(PyEulerALE ``src/py_euler_ale/core.py:24-1488``), with the same in-place host-array contract:
``states``, ``vertices``, ``velocities``, ``odes`` and ``forces`` are real views of
Fortran-ordered complex128 host arrays that the user modifies in place, every ``compute_*`` /
``linearize`` call reads them, and results are written back to host arrays. The work runs on
the GPU through the C ABI (``include/euler_b200.h``):

* residual, forces and all Jacobians are forward-mode dual-number kernels (no complex step);
* Jacobian products are stencil gathers on the device-resident Jacobians;
* the resolvent ``(dR/dU - shift I)^-1`` is a direct block LU over the grid's radial rings on
  the device, refined to the solve tolerance (the reference factorises with SuperLU on every
  call); complex GMRES with a block-Jacobi preconditioner is the alternative solver;
* the 13 second-order routines are exact directional derivatives of the Jacobians (nested
  duals) instead of the reference's central differences of complex-step Jacobians, so they
  agree with the reference to its finite-difference truncation error.

The flow parameters (angle of attack, JST constants) are held per instance and passed with
every call, instead of the reference's module globals (core.py:258-263).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

from . import _lib
from ._lib import DIR_STATES, DIR_VELOCITIES, DIR_VERTICES, call, ptr
from .grid import HEAT_RATIO, NUM_DIM, NUM_VAR, read_plot3d


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("pyeulerale_b200 needs a CUDA device (B200, sm_100a); "
                           "there is no CPU fallback")
    return torch


class SpatialDiscretization:
    """Spatial discretization of the compressible 2D Euler equations around a moving airfoil.

    Central-scheme finite volumes with JST artificial dissipation on a moving structured
    O-grid, linearized for ``dU/dt = R(U, X, V)``, ``F = F(U, X)`` (reference class docstring,
    core.py:25-37), evaluated on a B200 in FP64.
    """

    def __init__(
        self,
        grid_file: str | Path | np.ndarray,
        angle_of_attack: float = 1.25,
        mach_number: float = 0.5,
        coefficient_length: float = 1.0,
        coefficient_center: tuple[float, float] = (0.0, 0.0),
        jst_k2: float = 1,
        jst_k4: float = 1 / 32,
        jst_c4: float = 2,
        *,
        solver: str = "direct",
        gmres_tol: float = 1e-10,
        gmres_restart: int = 60,
        gmres_maxiter: int = 3000,
    ) -> None:
        """Initialize the discretization (core.py:60-113).

        Args:
            grid_file: PLOT3D grid file (single block, closed 2D O-grid), or an array of
                vertex coordinates ``(2, radial_pts, angular_pts)``.
            angle_of_attack: Far-field angle of attack in degree.
            mach_number: Free-stream Mach number.
            coefficient_length: Characteristic length of the section coefficients.
            coefficient_center: Reference point of the section moment coefficient.
            jst_k2, jst_k4, jst_c4: JST artificial dissipation constants.
            solver: Resolvent method: ``"direct"`` (ring-block LU on the device, refined to
                ``gmres_tol``) or ``"gmres"`` (block-Jacobi-preconditioned GMRES).
            gmres_tol: Relative residual of the resolvent solves.
            gmres_restart, gmres_maxiter: GMRES restart length and iteration limit.
        """
        self._torch = _torch()
        _lib.load()
        self.mach_number = mach_number
        self.angle_of_attack = angle_of_attack
        self._coefficient_length = coefficient_length
        self._coefficient_center = coefficient_center
        self._k2, self._k4, self._c4 = jst_k2, jst_k4, jst_c4
        if solver not in ("direct", "gmres"):
            raise ValueError("solver must be 'direct' or 'gmres'")
        self._solver = solver
        self._gmres = dict(tol=gmres_tol, restart=gmres_restart, maxiter=gmres_maxiter)
        self._ringlu = None
        self._vertices = self._read_grid(grid_file)
        self._num_radial = self._vertices.shape[1] - 1
        self._num_angular = self._vertices.shape[2] - 1
        M, N = self._num_radial, self._num_angular
        if M < 4 or N < 5:
            raise ValueError("the grid needs at least 5 radial and 6 angular points")
        self._velocities = np.zeros_like(self._vertices)
        self._states = np.asfortranarray(np.empty(dtype=complex, shape=(NUM_VAR, M, N)))
        self._odes = np.asfortranarray(np.empty(dtype=complex, shape=(NUM_VAR, M, N)))
        self._forces = np.asfortranarray(np.empty(dtype=complex, shape=(NUM_DIM, N)))
        torch = self._torch
        dev = torch.device("cuda")
        f64 = dict(dtype=torch.float64, device=dev)
        nv, nc = (M + 1) * (N + 1), M * N
        self._dX = torch.zeros(2 * nv, **f64)
        self._dV = torch.zeros(2 * nv, **f64)
        self._dU = torch.zeros(4 * nc, **f64)
        self._dR = torch.zeros(4 * nc, **f64)
        self._dF = torch.zeros(2 * N, **f64)
        self._dJ_ma = torch.zeros(4 * nc, **f64)
        self._dJ_u = torch.zeros(144 * nc, **f64)
        self._dJ_x = torch.zeros(32 * nc, **f64)
        self._dJ_v = torch.zeros(32 * nc, **f64)
        self._dJF_u = torch.zeros(8 * N, **f64)
        self._dJF_x = torch.zeros(8 * N, **f64)
        self._mirrors: dict[str, np.ndarray] = {}
        self._lu_stale = True
        self.set_free_stream_state()

    # ---- properties (core.py:115-211) -------------------------------------------------------
    @property
    def mach_number(self) -> float:
        """Free-stream Mach number"""
        return self._mach.real

    @mach_number.setter
    def mach_number(self, mach_number: float) -> None:
        self._mach = complex(mach_number)

    @property
    def angle_of_attack(self) -> float:
        """Far-field angle of attack in degree"""
        return self._aoa

    @angle_of_attack.setter
    def angle_of_attack(self, angle_of_attack: float) -> None:
        self._aoa = angle_of_attack

    @property
    def coefficient_length(self) -> float:
        """Characteristic length for the section coefficients"""
        return self._coefficient_length

    @property
    def coefficient_center(self) -> tuple[float, float]:
        """Reference point for the section moment coefficient"""
        return self._coefficient_center

    @property
    def _dynamic_pressure(self) -> float:
        """Dynamic pressure"""
        return self.mach_number**2 * HEAT_RATIO / 2

    @property
    def num_radial(self) -> int:
        """Number of cells in radial direction."""
        return self._num_radial

    @property
    def num_angular(self) -> int:
        """Number of cells in angular direction."""
        return self._num_angular

    @property
    def vertices(self) -> np.ndarray:
        """Grid vertices ``(NUM_DIM, num_radial+1, num_angular+1)``."""
        return self._vertices.real

    @property
    def surface_points(self) -> np.ndarray:
        """Mid-points of consecutive airfoil-surface vertices ``(NUM_DIM, num_angular)``."""
        return np.mean([self._vertices[:, 0, :-1].real, self._vertices[:, 0, 1:].real], axis=0)

    @property
    def velocities(self) -> np.ndarray:
        """Grid vertex velocities ``(NUM_DIM, num_radial+1, num_angular+1)``."""
        return self._velocities.real

    @property
    def states(self) -> np.ndarray:
        """Cell averaged conserved variables ``(NUM_VAR, num_radial, num_angular)``."""
        return self._states.real

    @property
    def odes(self) -> np.ndarray:
        """States' rate of change ``(NUM_VAR, num_radial, num_angular)``."""
        return self._odes.real

    @property
    def forces(self) -> np.ndarray:
        """Section forces on the ``surface_points`` ``(NUM_DIM, num_angular)``."""
        return self._forces.real

    # ---- private Jacobian mirrors (reference layouts, core.py:101-112) ----------------------
    def _mirror(self, key: str, tensor, shape: tuple) -> np.ndarray:
        if key not in self._mirrors:
            host = tensor.cpu().numpy()
            self._mirrors[key] = np.asfortranarray(np.reshape(host, shape, order="F"))
        return self._mirrors[key]

    @property
    def _odes_wrt_mach(self) -> np.ndarray:
        return self._mirror("ma", self._dJ_ma, (NUM_VAR, 1, self.num_radial, self.num_angular))

    @property
    def _odes_wrt_states(self) -> np.ndarray:
        return self._mirror("u", self._dJ_u,
                            (NUM_VAR, NUM_VAR, self.num_radial, self.num_angular, 9))

    @property
    def _odes_wrt_vertices(self) -> np.ndarray:
        return self._mirror("x", self._dJ_x,
                            (NUM_VAR, NUM_DIM, self.num_radial, self.num_angular, 4))

    @property
    def _odes_wrt_velocities(self) -> np.ndarray:
        return self._mirror("v", self._dJ_v,
                            (NUM_VAR, NUM_DIM, self.num_radial, self.num_angular, 4))

    @property
    def _forces_wrt_states(self) -> np.ndarray:
        return self._mirror("fu", self._dJF_u, (NUM_DIM, NUM_VAR, self.num_angular))

    @property
    def _forces_wrt_vertices(self) -> np.ndarray:
        return self._mirror("fx", self._dJF_x, (NUM_DIM, NUM_DIM, self.num_angular, 2))

    # ---- helpers ------------------------------------------------------------------------------
    @staticmethod
    def _read_grid(grid_file) -> np.ndarray:
        """Reads the grid (core.py:213-227) into a Fortran-ordered complex array."""
        if isinstance(grid_file, np.ndarray):
            v = grid_file
        else:
            v = read_plot3d(grid_file)
        return np.asfortranarray(v, dtype=complex)

    @staticmethod
    def _check_array(array: np.ndarray, shape: tuple,
                     dtype: np.dtype = np.dtypes.Complex128DType()) -> None:
        """Same checks and errors as the reference (core.py:229-256)."""
        if array.shape != shape:
            msg = f"Incorrect shape. Got {array.shape}, expected {shape}"
        elif array.dtype != dtype:
            msg = f"Incorrect data type. Got {array.dtype.name}, expected {np.dtype(dtype).name}"
        elif not array.flags.f_contiguous:
            msg = "Array is not FORTRAN-contiguous"
        else:
            return
        raise RuntimeError(msg)

    def _batch(self) -> _lib.Batch:
        inst = _lib.make_instance(self.num_radial, self.num_angular, self.mach_number,
                                  self._aoa, self._k2, self._k4, self._c4,
                                  self._coefficient_length, self._coefficient_center)
        return _lib.single_batch(inst)

    def _h2d(self, dst, array: np.ndarray) -> None:
        torch = self._torch
        src = np.ascontiguousarray(np.asarray(array).ravel(order="F"))
        if np.iscomplexobj(src):
            src = src.view(np.float64)
        dst.copy_(torch.from_numpy(src.astype(np.float64, copy=False)))

    def _upload(self, velocities: bool = True) -> None:
        self._h2d(self._dX, self._vertices.real)
        if velocities:
            self._h2d(self._dV, self._velocities.real)
        self._h2d(self._dU, self._states.real)

    def _cvec(self, array: np.ndarray):
        """Complex host array -> interleaved device float64 vector."""
        torch = self._torch
        src = np.ascontiguousarray(np.asarray(array, dtype=complex).ravel(order="F"))
        return torch.from_numpy(src.view(np.float64)).to("cuda")

    @staticmethod
    def _store(out: np.ndarray, dev, shape: tuple) -> np.ndarray:
        host = dev.cpu().numpy().view(np.complex128)
        out[...] = np.reshape(host, shape, order="F")
        return out

    def _stream(self) -> int:
        return self._torch.cuda.current_stream().cuda_stream

    def _call(self, name: str, *args) -> None:
        b = self._batch()
        call(name, _lib.ctypes.byref(b), *args, self._stream())

    # ---- state, residual, forces ------------------------------------------------------------
    def set_free_stream_state(self) -> None:
        """Sets ``states`` to free-stream (core.py:265-268)."""
        self._call("eb_set_free_stream_state", ptr(self._dU))
        host = self._dU.cpu().numpy()
        self._states[...] = np.reshape(host, self._states.shape, order="F")

    def compute_odes(self) -> None:
        """Computes ``odes`` from ``states``, ``vertices`` and ``velocities`` (core.py:270-276)."""
        self._upload()
        self._call("eb_compute_odes", ptr(self._dX), ptr(self._dV), ptr(self._dU), ptr(self._dR))
        host = self._dR.cpu().numpy()
        self._odes[...] = np.reshape(host, self._odes.shape, order="F")

    def compute_forces(self) -> None:
        """Computes ``forces`` from ``states`` and ``vertices`` (core.py:601-608)."""
        self._upload(velocities=False)
        self._call("eb_compute_forces", ptr(self._dX), ptr(self._dU), ptr(self._dF), None)
        host = self._dF.cpu().numpy()
        self._forces[...] = np.reshape(host, self._forces.shape, order="F")

    def linearize(self) -> None:
        """Computes the Jacobians on the device (core.py:278-292)."""
        self._upload()
        X, V, U = ptr(self._dX), ptr(self._dV), ptr(self._dU)
        self._call("eb_compute_odes_wrt_mach", X, V, U, ptr(self._dJ_ma))
        self._call("eb_compute_odes_wrt_states", X, V, U, ptr(self._dJ_u))
        self._call("eb_compute_odes_wrt_vertices", X, V, U, ptr(self._dJ_x))
        self._call("eb_compute_odes_wrt_velocities", X, V, U, ptr(self._dJ_v))
        self._call("eb_compute_forces_wrt_states", X, U, ptr(self._dJF_u))
        self._call("eb_compute_forces_wrt_vertices", X, U, ptr(self._dJF_x))
        self._mirrors.clear()
        self._lu_stale = True

    # ---- Jacobian products (core.py:294-510, 610-716) ----------------------------------------
    def _apply(self, name, jac, src: np.ndarray, out: np.ndarray | None, out_shape: tuple,
               out_numel: int) -> np.ndarray:
        torch = self._torch
        x = self._cvec(src)
        y = torch.empty(2 * out_numel, dtype=torch.float64, device="cuda")
        self._call(name, ptr(jac), ptr(x), ptr(y))
        if out is None:
            out = np.asfortranarray(np.empty(out_shape, dtype=complex))
        return self._store(out, y, out_shape)

    def apply_odes_wrt_mach_fwd(self, d_mach: np.ndarray, d_odes: np.ndarray | None = None):
        """``dR/dMa . dMa`` (core.py:294-319)."""
        self._check_array(d_mach, (1,))
        if d_odes is not None:
            self._check_array(d_odes, self._odes.shape)
        return self._apply("eb_apply_odes_wrt_mach_fwd", self._dJ_ma, d_mach, d_odes,
                           self._odes.shape, self._odes.size)

    def apply_odes_wrt_mach_rev(self, d_odes: np.ndarray, d_mach: np.ndarray | None = None):
        """``dR/dMa^T . dR`` (core.py:321-346)."""
        self._check_array(d_odes, self._odes.shape)
        if d_mach is not None:
            self._check_array(d_mach, (1,))
        return self._apply("eb_apply_odes_wrt_mach_rev", self._dJ_ma, d_odes, d_mach, (1,), 1)

    def apply_odes_wrt_states_fwd(self, d_states: np.ndarray, d_odes: np.ndarray | None = None):
        """``dR/dU . dU`` (core.py:348-373)."""
        self._check_array(d_states, self._states.shape)
        if d_odes is not None:
            self._check_array(d_odes, self._odes.shape)
        return self._apply("eb_apply_odes_wrt_states_fwd", self._dJ_u, d_states, d_odes,
                           self._odes.shape, self._odes.size)

    def apply_odes_wrt_states_rev(self, d_odes: np.ndarray, d_states: np.ndarray | None = None):
        """``dR/dU^T . dR`` (core.py:375-400)."""
        self._check_array(d_odes, self._odes.shape)
        if d_states is not None:
            self._check_array(d_states, self._states.shape)
        return self._apply("eb_apply_odes_wrt_states_rev", self._dJ_u, d_odes, d_states,
                           self._states.shape, self._states.size)

    def apply_odes_wrt_vertices_fwd(self, d_vertices: np.ndarray,
                                    d_odes: np.ndarray | None = None):
        """``dR/dX . dX`` (core.py:402-427)."""
        self._check_array(d_vertices, self._vertices.shape)
        if d_odes is not None:
            self._check_array(d_odes, self._odes.shape)
        return self._apply("eb_apply_odes_wrt_vertices_fwd", self._dJ_x, d_vertices, d_odes,
                           self._odes.shape, self._odes.size)

    def apply_odes_wrt_vertices_rev(self, d_odes: np.ndarray,
                                    d_vertices: np.ndarray | None = None):
        """``dR/dX^T . dR`` (core.py:429-454)."""
        self._check_array(d_odes, self._odes.shape)
        if d_vertices is not None:
            self._check_array(d_vertices, self._vertices.shape)
        return self._apply("eb_apply_odes_wrt_vertices_rev", self._dJ_x, d_odes, d_vertices,
                           self._vertices.shape, self._vertices.size)

    def apply_odes_wrt_velocities_fwd(self, d_velocities: np.ndarray,
                                      d_odes: np.ndarray | None = None):
        """``dR/dV . dV`` (core.py:456-482)."""
        self._check_array(d_velocities, self._velocities.shape)
        if d_odes is not None:
            self._check_array(d_odes, self._odes.shape)
        return self._apply("eb_apply_odes_wrt_vertices_fwd", self._dJ_v, d_velocities, d_odes,
                           self._odes.shape, self._odes.size)

    def apply_odes_wrt_velocities_rev(self, d_odes: np.ndarray,
                                      d_velocities: np.ndarray | None = None):
        """``dR/dV^T . dR`` (core.py:484-510)."""
        self._check_array(d_odes, self._odes.shape)
        if d_velocities is not None:
            self._check_array(d_velocities, self._velocities.shape)
        return self._apply("eb_apply_odes_wrt_vertices_rev", self._dJ_v, d_odes, d_velocities,
                           self._velocities.shape, self._velocities.size)

    def apply_forces_wrt_states_fwd(self, d_states: np.ndarray,
                                    d_forces: np.ndarray | None = None):
        """``dF/dU . dU`` (core.py:610-635)."""
        self._check_array(d_states, self._states.shape)
        if d_forces is not None:
            self._check_array(d_forces, self._forces.shape)
        return self._apply("eb_apply_forces_wrt_states_fwd", self._dJF_u, d_states, d_forces,
                           self._forces.shape, self._forces.size)

    def apply_forces_wrt_states_rev(self, d_forces: np.ndarray,
                                    d_states: np.ndarray | None = None):
        """``dF/dU^T . dF`` (core.py:637-662)."""
        self._check_array(d_forces, self._forces.shape)
        if d_states is not None:
            self._check_array(d_states, self._states.shape)
        return self._apply("eb_apply_forces_wrt_states_rev", self._dJF_u, d_forces, d_states,
                           self._states.shape, self._states.size)

    def apply_forces_wrt_vertices_fwd(self, d_vertices: np.ndarray,
                                      d_forces: np.ndarray | None = None):
        """``dF/dX . dX`` (core.py:664-689)."""
        self._check_array(d_vertices, self._vertices.shape)
        if d_forces is not None:
            self._check_array(d_forces, self._forces.shape)
        return self._apply("eb_apply_forces_wrt_vertices_fwd", self._dJF_x, d_vertices,
                           d_forces, self._forces.shape, self._forces.size)

    def apply_forces_wrt_vertices_rev(self, d_forces: np.ndarray,
                                      d_vertices: np.ndarray | None = None):
        """``dF/dX^T . dF`` (core.py:691-716)."""
        self._check_array(d_forces, self._forces.shape)
        if d_vertices is not None:
            self._check_array(d_vertices, self._vertices.shape)
        return self._apply("eb_apply_forces_wrt_vertices_rev", self._dJF_x, d_forces,
                           d_vertices, self._vertices.shape, self._vertices.size)

    # ---- resolvent (core.py:512-599) ---------------------------------------------------------
    def _solve(self, rhs: np.ndarray, shift: complex, adjoint: bool) -> np.ndarray:
        from . import solver

        b = self._cvec(rhs)
        if self._solver == "gmres":
            x, info = solver.solve_shifted(self._batch(), self._dJ_u, b, [complex(shift)],
                                           adjoint=adjoint, **self._gmres)
            self.last_solve_info = info
        else:
            if self._ringlu is None:
                self._ringlu = solver.RingLU(self._batch(), tol=self._gmres["tol"])
            lu = self._ringlu
            lu.batch = self._batch()
            # The factors stay valid while the Jacobian and the shift are unchanged.
            if lu.J is None or lu.shift != complex(shift) or self._lu_stale:
                lu.factor(self._dJ_u, shift)
                self._lu_stale = False
            x, rel = lu.solve(b, adjoint=adjoint)
            self.last_solve_info = {"method": "direct", "rel_residual": rel}
        return x.cpu().numpy().view(np.complex128)

    def solve_odes_wrt_states_fwd(self, d_odes: np.ndarray, shift: float | complex = 0.,
                                  d_states: np.ndarray | None = None) -> np.ndarray:
        """``(dR/dU - shift Id)^-1 . dR`` on the device (core.py:533-565)."""
        self._check_array(d_odes, self._odes.shape, dtype=d_odes.dtype)
        result_dtype = np.promote_types(type(shift), d_odes.dtype)
        if d_states is None:
            d_states = np.empty_like(d_odes, result_dtype)
        else:
            self._check_array(d_states, self._states.shape, result_dtype)
        x = self._solve(d_odes, shift, adjoint=False)
        sol = np.reshape(x, self._states.shape, order="F")
        d_states[...] = sol if np.iscomplexobj(d_states) else sol.real
        return d_states

    def solve_odes_wrt_states_adj(self, d_states: np.ndarray, shift: float | complex = 0.,
                                  d_odes: np.ndarray | None = None) -> np.ndarray:
        """``(dR/dU - shift Id)^-H . dU`` on the device (core.py:567-599)."""
        self._check_array(d_states, self._odes.shape, dtype=d_states.dtype)
        result_dtype = np.promote_types(type(shift), d_states.dtype)
        if d_odes is None:
            d_odes = np.empty_like(d_states, result_dtype)
        else:
            self._check_array(d_odes, self._odes.shape, result_dtype)
        x = self._solve(d_states, shift, adjoint=True)
        sol = np.reshape(x, self._odes.shape, order="F")
        d_odes[...] = sol if np.iscomplexobj(d_odes) else sol.real
        return d_odes

    # ---- second-order gradients (core.py:718-1275) -------------------------------------------
    def _second_order(self, builder: str, dir_kind: int, direction: np.ndarray, apply_rev: str,
                      jac_numel: int, cotangent: np.ndarray, out_shape: tuple) -> np.ndarray:
        """[d/de J_A(B + e Re d)]^T conj(w) + i [d/de J_A(B + e Im d)]^T conj(w)."""
        torch = self._torch
        self._upload()
        d = self._cvec(direction)
        J_re = torch.empty(jac_numel, dtype=torch.float64, device="cuda")
        J_im = torch.empty_like(J_re)
        X, V, U = ptr(self._dX), ptr(self._dV), ptr(self._dU)
        if builder.startswith("eb_forces"):
            self._call(builder, X, U, dir_kind, ptr(d), ptr(J_re), ptr(J_im))
        else:
            self._call(builder, X, V, U, dir_kind, ptr(d), ptr(J_re), ptr(J_im))
        w = self._cvec(np.conj(cotangent))
        numel = int(np.prod(out_shape))
        y_re = torch.empty(2 * numel, dtype=torch.float64, device="cuda")
        y_im = torch.empty_like(y_re)
        self._call(apply_rev, ptr(J_re), ptr(w), ptr(y_re))
        self._call(apply_rev, ptr(J_im), ptr(w), ptr(y_im))
        a = y_re.cpu().numpy().view(np.complex128)
        b = y_im.cpu().numpy().view(np.complex128)
        return np.asfortranarray(np.reshape(a + 1j * b, out_shape, order="F"))

    def _grad_out(self, out, shape, result):
        if out is not None:
            self._check_array(out, shape)
            out[...] = result
            return out
        return result

    def _nc(self) -> int:
        return self.num_radial * self.num_angular

    def compute_odes_wrt_states_inner_product_wrt_mach(self, d_odes, d_states, mach_gradient=None):
        """``grad_Ma <dR, dR/dU . dU>`` (core.py:718-759)."""
        self._check_array(d_states, self._states.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_mach_dir", DIR_STATES, d_states,
                               "eb_apply_odes_wrt_mach_rev", 4 * self._nc(), d_odes, (1,))
        return self._grad_out(mach_gradient, (1,), g)

    def compute_odes_wrt_states_inner_product_wrt_states(self, d_odes, d_states,
                                                         states_gradient=None):
        """``grad_U <dR, dR/dU . dU>`` (core.py:761-802)."""
        self._check_array(d_states, self._states.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_states_dir", DIR_STATES, d_states,
                               "eb_apply_odes_wrt_states_rev", 144 * self._nc(), d_odes,
                               self._states.shape)
        return self._grad_out(states_gradient, self._states.shape, g)

    def compute_odes_wrt_states_inner_product_wrt_vertices(self, d_odes, d_states,
                                                           vertices_gradient=None):
        """``grad_X <dR, dR/dU . dU>`` (core.py:804-845)."""
        self._check_array(d_states, self._states.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_vertices_dir", DIR_STATES, d_states,
                               "eb_apply_odes_wrt_vertices_rev", 32 * self._nc(), d_odes,
                               self._vertices.shape)
        return self._grad_out(vertices_gradient, self._vertices.shape, g)

    def compute_odes_wrt_vertices_inner_product_wrt_mach(self, d_odes, d_vertices,
                                                         mach_gradient=None):
        """``grad_Ma <dR, dR/dX . dX>`` (core.py:847-888)."""
        self._check_array(d_vertices, self._vertices.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_mach_dir", DIR_VERTICES, d_vertices,
                               "eb_apply_odes_wrt_mach_rev", 4 * self._nc(), d_odes, (1,))
        return self._grad_out(mach_gradient, (1,), g)

    def compute_odes_wrt_vertices_inner_product_wrt_states(self, d_odes, d_vertices,
                                                           states_gradient=None):
        """``grad_U <dR, dR/dX . dX>`` (core.py:890-931)."""
        self._check_array(d_vertices, self._vertices.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_states_dir", DIR_VERTICES, d_vertices,
                               "eb_apply_odes_wrt_states_rev", 144 * self._nc(), d_odes,
                               self._states.shape)
        return self._grad_out(states_gradient, self._states.shape, g)

    def compute_odes_wrt_vertices_inner_product_wrt_vertices(self, d_odes, d_vertices,
                                                             vertices_gradient=None):
        """``grad_X <dR, dR/dX . dX>`` (core.py:933-974)."""
        self._check_array(d_vertices, self._vertices.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_vertices_dir", DIR_VERTICES, d_vertices,
                               "eb_apply_odes_wrt_vertices_rev", 32 * self._nc(), d_odes,
                               self._vertices.shape)
        return self._grad_out(vertices_gradient, self._vertices.shape, g)

    def compute_odes_wrt_velocities_inner_product_wrt_mach(self, d_odes, d_velocities,
                                                           mach_gradient=None):
        """``grad_Ma <dR, dR/dV . dV>`` (core.py:976-1017)."""
        self._check_array(d_velocities, self._vertices.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_mach_dir", DIR_VELOCITIES, d_velocities,
                               "eb_apply_odes_wrt_mach_rev", 4 * self._nc(), d_odes, (1,))
        return self._grad_out(mach_gradient, (1,), g)

    def compute_odes_wrt_velocities_inner_product_wrt_states(self, d_odes, d_velocities,
                                                             states_gradient=None):
        """``grad_U <dR, dR/dV . dV>`` (core.py:1019-1060)."""
        self._check_array(d_velocities, self._vertices.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_states_dir", DIR_VELOCITIES, d_velocities,
                               "eb_apply_odes_wrt_states_rev", 144 * self._nc(), d_odes,
                               self._states.shape)
        return self._grad_out(states_gradient, self._states.shape, g)

    def compute_odes_wrt_velocities_inner_product_wrt_vertices(self, d_odes, d_velocities,
                                                               vertices_gradient=None):
        """``grad_X <dR, dR/dV . dV>`` (core.py:1062-1103)."""
        self._check_array(d_velocities, self._vertices.shape)
        self._check_array(d_odes, self._odes.shape)
        g = self._second_order("eb_odes_wrt_vertices_dir", DIR_VELOCITIES, d_velocities,
                               "eb_apply_odes_wrt_vertices_rev", 32 * self._nc(), d_odes,
                               self._vertices.shape)
        return self._grad_out(vertices_gradient, self._vertices.shape, g)

    def compute_forces_wrt_states_inner_product_wrt_states(self, d_forces, d_states,
                                                           states_gradient=None):
        """``grad_U <dF, dF/dU . dU>`` (core.py:1105-1146)."""
        self._check_array(d_states, self._states.shape)
        self._check_array(d_forces, self._forces.shape)
        g = self._second_order("eb_forces_wrt_states_dir", DIR_STATES, d_states,
                               "eb_apply_forces_wrt_states_rev", 8 * self.num_angular,
                               d_forces, self._states.shape)
        return self._grad_out(states_gradient, self._states.shape, g)

    def compute_forces_wrt_states_inner_product_wrt_vertices(self, d_forces, d_states,
                                                             vertices_gradient=None):
        """``grad_X <dF, dF/dU . dU>`` (core.py:1148-1189)."""
        self._check_array(d_states, self._states.shape)
        self._check_array(d_forces, self._forces.shape)
        g = self._second_order("eb_forces_wrt_vertices_dir", DIR_STATES, d_states,
                               "eb_apply_forces_wrt_vertices_rev", 8 * self.num_angular,
                               d_forces, self._vertices.shape)
        return self._grad_out(vertices_gradient, self._vertices.shape, g)

    def compute_forces_wrt_vertices_inner_product_wrt_states(self, d_forces, d_vertices,
                                                             states_gradient=None):
        """``grad_U <dF, dF/dX . dX>`` (core.py:1191-1232)."""
        self._check_array(d_vertices, self._vertices.shape)
        self._check_array(d_forces, self._forces.shape)
        g = self._second_order("eb_forces_wrt_states_dir", DIR_VERTICES, d_vertices,
                               "eb_apply_forces_wrt_states_rev", 8 * self.num_angular,
                               d_forces, self._states.shape)
        return self._grad_out(states_gradient, self._states.shape, g)

    def compute_forces_wrt_vertices_inner_product_wrt_vertices(self, d_forces, d_vertices,
                                                               vertices_gradient=None):
        """``grad_X <dF, dF/dX . dX>`` (core.py:1234-1275)."""
        self._check_array(d_vertices, self._vertices.shape)
        self._check_array(d_forces, self._forces.shape)
        g = self._second_order("eb_forces_wrt_vertices_dir", DIR_VERTICES, d_vertices,
                               "eb_apply_forces_wrt_vertices_rev", 8 * self.num_angular,
                               d_forces, self._vertices.shape)
        return self._grad_out(vertices_gradient, self._vertices.shape, g)

    # ---- coefficients (core.py:1277-1488; host NumPy, as in the reference) ------------------
    def compute_drag_coefficient(self) -> float:
        """Section drag coefficient from ``forces`` (core.py:1277-1287, no chord division)."""
        forces_x, _ = self.forces
        return np.sum(forces_x) / self._dynamic_pressure

    def compute_drag_coefficient_wrt_forces(self, forces_gradient=None) -> np.ndarray:
        """``grad_F c_d`` (core.py:1289-1312)."""
        if forces_gradient is not None:
            self._check_array(forces_gradient, self._forces.shape)
        else:
            forces_gradient = np.empty_like(self._forces)
        forces_gradient[0, :] = 1. / (self._dynamic_pressure * self.coefficient_length)
        forces_gradient[1, :] = 0.
        return forces_gradient

    def compute_lift_coefficient(self) -> float:
        """Section lift coefficient from ``forces`` (core.py:1314-1324)."""
        _, forces_z = self.forces
        return np.sum(forces_z) / (self._dynamic_pressure * self.coefficient_length)

    def compute_lift_coefficient_wrt_forces(self, forces_gradient=None) -> np.ndarray:
        """``grad_F c_l`` (core.py:1326-1349)."""
        if forces_gradient is not None:
            self._check_array(forces_gradient, self._forces.shape)
        else:
            forces_gradient = np.empty_like(self._forces)
        forces_gradient[0, :] = 0.
        forces_gradient[1, :] = 1. / (self._dynamic_pressure * self.coefficient_length)
        return forces_gradient

    def compute_moment_coefficient(self) -> float:
        """Section moment coefficient from ``forces`` and ``vertices`` (core.py:1351-1364)."""
        points_x, points_z = self.surface_points - np.reshape(self.coefficient_center, (2, 1))
        forces_x, forces_z = self.forces
        return np.sum(points_z * forces_x - points_x * forces_z) / (
            self._dynamic_pressure * self.coefficient_length**2)

    def compute_moment_coefficient_wrt_forces(self, forces_gradient=None) -> np.ndarray:
        """``grad_F c_m`` (core.py:1366-1390)."""
        if forces_gradient is not None:
            self._check_array(forces_gradient, self._forces.shape)
        else:
            forces_gradient = np.empty_like(self._forces)
        points_x, points_z = self.surface_points - np.reshape(self.coefficient_center, (2, 1))
        q = self._dynamic_pressure * self.coefficient_length**2
        forces_gradient[0, :] = points_z / q
        forces_gradient[1, :] = -points_x / q
        return forces_gradient

    def compute_moment_coefficient_wrt_vertices(self, vertices_gradient=None) -> np.ndarray:
        """``grad_X c_m`` at fixed ``forces`` (core.py:1392-1421)."""
        if vertices_gradient is not None:
            self._check_array(vertices_gradient, self._vertices.shape)
        else:
            vertices_gradient = np.empty_like(self._vertices)
        forces_x, forces_z = self._forces
        q = self._dynamic_pressure * self.coefficient_length**2
        points_gradient = np.stack([-forces_z / q, forces_x / q])
        vertices_gradient[:] = 0.
        vertices_gradient[:, 0, :-1] += points_gradient / 2.
        vertices_gradient[:, 0, 1:] += points_gradient / 2.
        return vertices_gradient

    def compute_pressure_coefficients(self, pressure_coefficients=None) -> np.ndarray:
        """Pressure coefficients of all cells, on the device (core.py:1423-1449)."""
        shape = (self.num_radial, self.num_angular)
        if pressure_coefficients is not None:
            self._check_array(pressure_coefficients, shape=shape,
                              dtype=np.dtypes.Float64DType())
        else:
            pressure_coefficients = np.asfortranarray(np.empty(dtype=float, shape=shape))
        torch = self._torch
        self._upload(velocities=False)
        cp = torch.empty(self._nc(), dtype=torch.float64, device="cuda")
        self._call("eb_compute_pressure_coefficients", ptr(self._dU), ptr(cp))
        pressure_coefficients[:] = np.reshape(cp.cpu().numpy(), shape, order="F")
        return pressure_coefficients

    def apply_pressure_coefficients_wrt_states_fwd(self, d_states,
                                                   d_pressure_coefficients=None) -> np.ndarray:
        """``dcp/dU . dU`` on the device (core.py:1451-1488)."""
        self._check_array(d_states, self._states.shape)
        shape = (self.num_radial, self.num_angular)
        if d_pressure_coefficients is not None:
            self._check_array(d_pressure_coefficients, shape=shape)
        else:
            d_pressure_coefficients = np.asfortranarray(np.empty(dtype=complex, shape=shape))
        torch = self._torch
        self._upload(velocities=False)
        dcp = torch.empty(2 * self._nc(), dtype=torch.float64, device="cuda")
        self._call("eb_apply_pressure_coefficients_wrt_states_fwd", ptr(self._dU),
                   ptr(self._cvec(d_states)), ptr(dcp))
        return self._store(d_pressure_coefficients, dcp, shape)
