"""Python side of the device resolvent (``eb_gmres_solve`` in csrc/gmres.cu).

``solve_shifted`` solves ``(dR/dU - s I) x = b`` (or the Hermitian-adjoint system) for any
number of (instance, shift, right-hand side) systems in one native call. All vectors are
torch complex128-compatible float64 device tensors in the interleaved layout of the C ABI.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class GmresOptions(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("restart", ctypes.c_int32),
                ("max_iterations", ctypes.c_int32), ("check_every", ctypes.c_int32),
                ("use_initial_guess", ctypes.c_int32)]


class GmresInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("cycles", ctypes.c_int32),
                ("converged", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("rel_residual", ctypes.c_double)]


_bound = False


def _bind() -> ctypes.CDLL:
    global _bound
    lib = _lib.load()
    if not _bound:
        lib.eb_gmres_workspace_bytes.restype = ctypes.c_int64
        lib.eb_gmres_workspace_bytes.argtypes = [
            ctypes.POINTER(_lib.Batch), ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_int]
        lib.eb_gmres_solve.restype = ctypes.c_int
        lib.eb_gmres_solve.argtypes = [
            ctypes.POINTER(_lib.Batch), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.POINTER(GmresOptions), ctypes.c_void_p, ctypes.c_int64,
            ctypes.POINTER(GmresInfo), ctypes.c_void_p]
        _bound = True
    return lib


class SolveInfo(list):
    """Per-system GMRES statistics (iterations, cycles, converged, rel_residual)."""

    @property
    def iterations(self) -> list[int]:
        return [i["iterations"] for i in self]

    @property
    def max_rel_residual(self) -> float:
        return max(i["rel_residual"] for i in self)


def solve_shifted(batch: _lib.Batch, J, rhs, shifts, *, adjoint: bool = False,
                  tol: float = 1e-10, restart: int = 60, maxiter: int = 3000,
                  check_every: int = 10, x0=None, sys_inst=None, host_table=None,
                  workspace=None, raise_on_failure: bool = True):
    """Solves the shifted systems; returns ``(x, SolveInfo)``.

    Args:
        batch: the instances (``_lib.Batch``).
        J: device d(odes)/d(states) of the batch (float64, 144 per cell).
        rhs: device float64 tensor, system-major interleaved complex right-hand sides.
        shifts: one complex shift per system.
        adjoint: solve with ``(A - s I)^H`` (the reference's ``solve_odes_wrt_states_adj``).
        sys_inst: instance index of each system (default: all on instance 0).
        host_table: host ``_lib.Instance`` array for batches of several instances.
    """
    import torch

    lib = _bind()
    n_sys = len(shifts)
    sh = np.zeros(2 * n_sys)
    sh[0::2] = np.real(shifts)
    sh[1::2] = np.imag(shifts)
    inst = None if sys_inst is None else np.ascontiguousarray(sys_inst, dtype=np.int32)
    tab_ptr = None if host_table is None else ctypes.addressof(host_table)
    inst_ptr = None if inst is None else inst.ctypes.data
    bref = ctypes.byref(batch)
    need = lib.eb_gmres_workspace_bytes(bref, tab_ptr, n_sys, inst_ptr, int(restart))
    if need < 0:
        raise ValueError("invalid GMRES systems")
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(int(need), dtype=torch.uint8, device=rhs.device)
    x = torch.zeros_like(rhs) if x0 is None else x0
    opts = GmresOptions(float(tol), int(restart), int(maxiter), int(check_every),
                        0 if x0 is None else 1)
    infos = (GmresInfo * n_sys)()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.eb_gmres_solve(bref, tab_ptr, J.data_ptr(), n_sys, inst_ptr, sh.ctypes.data,
                            1 if adjoint else 0, rhs.data_ptr(), x.data_ptr(),
                            ctypes.byref(opts), workspace.data_ptr(), int(workspace.numel()),
                            infos, stream)
    info = SolveInfo({"iterations": i.iterations, "cycles": i.cycles,
                      "converged": bool(i.converged), "rel_residual": i.rel_residual}
                     for i in infos)
    if rc != _lib.EB_OK and raise_on_failure:
        raise _lib.EulerB200Error("eb_gmres_solve", rc, lib.eb_last_error().decode()
                                  + f" (rel. residuals {[i['rel_residual'] for i in info]})")
    return x, info


def _bind_anchored() -> ctypes.CDLL:
    lib = _bind()
    if not getattr(lib, "_anchored_bound", False):
        P = ctypes.c_void_p
        lib.eb_gmres_anchored_aux_bytes.restype = ctypes.c_int64
        lib.eb_gmres_anchored_aux_bytes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int, P]
        lib.eb_gmres_solve_anchored.restype = ctypes.c_int
        lib.eb_gmres_solve_anchored.argtypes = [
            ctypes.POINTER(_lib.Batch), P, ctypes.c_int, P, P, P, ctypes.POINTER(GmresOptions),
            ctypes.c_int, P, P, ctypes.c_int64, P, ctypes.c_int64, P, ctypes.c_int64,
            ctypes.POINTER(GmresInfo), P]
        lib._anchored_bound = True
    return lib


def solve_anchored(batch: _lib.Batch, J, rhs, shifts, anchors: "RingLUMany", sys_anchor, *,
                   tol: float = 1e-10, restart: int = 40, maxiter: int = 240,
                   check_every: int = 5, raise_on_failure: bool = True):
    """GMRES on ``(J - s I) x = b`` for many shifts of one instance, each right-preconditioned by
    the ring-LU factors of its anchor (``eb_gmres_solve_anchored``); returns ``(x, SolveInfo)``.

    ``anchors`` holds the anchors' factorisations (``RingLUMany.factor(J, anchor_shifts)``),
    ``sys_anchor[s]`` the anchor of system ``s`` (at most 8 systems per anchor). ``rhs``: device
    float64 tensor of the systems' interleaved complex right-hand sides, system-major.
    """
    import torch

    lib = _bind_anchored()
    n_sys = len(shifts)
    sh = np.zeros(2 * n_sys)
    sh[0::2] = np.real(shifts)
    sh[1::2] = np.imag(shifts)
    sa = np.ascontiguousarray(sys_anchor, dtype=np.int32)
    bref = ctypes.byref(batch)
    M, N = batch.single.M, batch.single.N
    need = lib.eb_gmres_workspace_bytes(bref, None, n_sys, None, int(restart))
    aux_need = lib.eb_gmres_anchored_aux_bytes(M, N, n_sys, anchors.capacity, sa.ctypes.data)
    if need < 0 or aux_need < 0:
        raise ValueError("invalid anchored GMRES systems")
    workspace = torch.empty(int(need), dtype=torch.uint8, device=rhs.device)
    aux = torch.empty(int(aux_need), dtype=torch.uint8, device=rhs.device)
    x = torch.zeros_like(rhs)
    opts = GmresOptions(float(tol), int(restart), int(maxiter), int(check_every), 0)
    infos = (GmresInfo * n_sys)()
    rc = lib.eb_gmres_solve_anchored(
        bref, J.data_ptr(), n_sys, sh.ctypes.data, rhs.data_ptr(), x.data_ptr(),
        ctypes.byref(opts), anchors.capacity, sa.ctypes.data, anchors.workspace.data_ptr(),
        anchors.stride, workspace.data_ptr(), int(workspace.numel()), aux.data_ptr(),
        int(aux.numel()), infos, torch.cuda.current_stream().cuda_stream)
    info = SolveInfo({"iterations": i.iterations, "cycles": i.cycles,
                      "converged": bool(i.converged), "rel_residual": i.rel_residual}
                     for i in infos)
    if rc != _lib.EB_OK and (raise_on_failure or rc != _lib.EB_ERR_NOCONV):
        raise _lib.EulerB200Error("eb_gmres_solve_anchored", rc, lib.eb_last_error().decode()
                                  + f" (rel. residuals {[i['rel_residual'] for i in info]})")
    return x, info


def anchor_shifts(shifts, per_anchor: int = 4):
    """Anchors for ``solve_anchored``: the shifts ordered by magnitude in consecutive groups of
    ``per_anchor``; a group's anchor has the geometric mean of its magnitudes (the arithmetic mean
    if one is zero) and its middle shift's direction. Returns ``(anchors, sys_anchor)``."""
    s = np.asarray(shifts, dtype=complex)
    if not 1 <= per_anchor <= 8:
        raise ValueError("per_anchor must be in 1..8")
    order = np.argsort(np.abs(s), kind="stable")
    n_a = -(-len(s) // per_anchor)
    anchors = np.empty(n_a, dtype=complex)
    sys_anchor = np.empty(len(s), dtype=np.int32)
    for a in range(n_a):
        idx = order[a * per_anchor:(a + 1) * per_anchor]
        g = s[idx]
        mid = g[len(g) // 2]
        mags = np.abs(g)
        if np.all(mags > 0):
            anchors[a] = np.exp(np.mean(np.log(mags))) * mid / abs(mid)
        else:
            anchors[a] = np.mean(g)
        sys_anchor[idx] = a
    return anchors, sys_anchor


def _bind_ringlu() -> ctypes.CDLL:
    lib = _lib.load()
    if not getattr(lib, "_ringlu_bound", False):
        P = ctypes.c_void_p
        lib.eb_ringlu_workspace_bytes.restype = ctypes.c_int64
        lib.eb_ringlu_workspace_bytes.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.eb_ringlu_factor.restype = ctypes.c_int
        lib.eb_ringlu_factor.argtypes = [ctypes.POINTER(_lib.Batch), P, ctypes.c_double,
                                         ctypes.c_double, P, ctypes.c_int64, P]
        lib.eb_ringlu_solve.restype = ctypes.c_int
        lib.eb_ringlu_solve.argtypes = [
            ctypes.POINTER(_lib.Batch), P, ctypes.c_double, ctypes.c_double, ctypes.c_int, P,
            ctypes.c_int64, P, P, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
            P]
        lib.eb_ringlu_factor_many.restype = ctypes.c_int
        lib.eb_ringlu_factor_many.argtypes = [ctypes.POINTER(_lib.Batch), P, ctypes.c_int, P, P,
                                              ctypes.c_int64, P]  # workspace base, stride
        lib.eb_ringlu_solve_many.restype = ctypes.c_int
        lib.eb_ringlu_solve_many.argtypes = [
            ctypes.POINTER(_lib.Batch), P, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int64, P, P,
            ctypes.c_double, ctypes.c_int, P, P]
        lib._ringlu_bound = True
    return lib


def ringlu_workspace_bytes(M: int, N: int) -> int:
    """Device bytes of one ring-LU factorisation of an M x N cell grid (-1: unsupported)."""
    return int(_bind_ringlu().eb_ringlu_workspace_bytes(int(M), int(N)))


class RingLU:
    """Direct resolvent of one instance: ring-block LU factors of ``J - shift I`` on the device.

    ``factor(J, shift)`` builds the factors (``eb_ringlu_factor``); ``solve(rhs, adjoint)``
    returns ``(J - shift I)^-1 rhs`` or ``(J - shift I)^-H rhs`` refined to ``tol``
    (``eb_ringlu_solve``). One factorisation serves both solve directions.
    """

    def __init__(self, batch: _lib.Batch, tol: float = 1e-10, max_refine: int = 4) -> None:
        import torch

        self._torch = torch
        self.batch = batch
        self.tol = tol
        self.max_refine = max_refine
        lib = _bind_ringlu()
        self._lib = lib
        need = lib.eb_ringlu_workspace_bytes(batch.single.M, batch.single.N)
        if need < 0:
            raise ValueError("ring LU needs a single instance with M >= 4, N >= 5")
        self.workspace = torch.empty(int(need), dtype=torch.uint8, device="cuda")
        self.J = None
        self.shift = None

    def factor(self, J, shift: complex) -> None:
        shift = complex(shift)
        stream = self._torch.cuda.current_stream().cuda_stream
        rc = self._lib.eb_ringlu_factor(ctypes.byref(self.batch), J.data_ptr(), shift.real,
                                        shift.imag, self.workspace.data_ptr(),
                                        self.workspace.numel(), stream)
        if rc != _lib.EB_OK:
            raise _lib.EulerB200Error("eb_ringlu_factor", rc, self._lib.eb_last_error().decode())
        self.J, self.shift = J, shift

    def solve(self, rhs, adjoint: bool = False, out=None):
        """Solves with the current factors; returns ``(x, rel_residual)``."""
        if self.J is None:
            raise RuntimeError("factor() first")
        x = self._torch.empty_like(rhs) if out is None else out
        rel = ctypes.c_double(0.0)
        stream = self._torch.cuda.current_stream().cuda_stream
        rc = self._lib.eb_ringlu_solve(ctypes.byref(self.batch), self.J.data_ptr(),
                                       self.shift.real, self.shift.imag, 1 if adjoint else 0,
                                       self.workspace.data_ptr(), self.workspace.numel(),
                                       rhs.data_ptr(), x.data_ptr(), self.tol, self.max_refine,
                                       ctypes.byref(rel), stream)
        if rc != _lib.EB_OK:
            raise _lib.EulerB200Error("eb_ringlu_solve", rc,
                                      self._lib.eb_last_error().decode() + f" (rel {rel.value})")
        return x, rel.value


class RingLUMany:
    """Ring-LU factors of ``J - s I`` for several shifts ``s`` of one instance at once.

    ``factor(J, shifts)`` runs ``eb_ringlu_factor_many``: every elimination step is one launch
    over all shifts (batched Gauss-Jordan ring inversions and strided-batched GEMMs).
    ``solve(rhs, adjoint)`` solves one right-hand side per shift through
    ``eb_ringlu_solve_many`` the same way. ``capacity`` fixes the number of shift workspaces
    (each ``ringlu_workspace_bytes(M, N)`` bytes, in one device allocation).
    """

    def __init__(self, batch: _lib.Batch, capacity: int, tol: float = 1e-10,
                 max_refine: int = 4, workspace=None) -> None:
        import torch

        self._torch = torch
        self._lib = _bind_ringlu()
        self.batch, self.tol, self.max_refine = batch, tol, max_refine
        need = self._lib.eb_ringlu_workspace_bytes(batch.single.M, batch.single.N)
        if need < 0:
            raise ValueError("ring LU needs a single instance with M >= 4, N >= 5")
        self.stride = (int(need) + 255) // 256 * 256
        self.capacity = int(capacity)
        if workspace is None:
            workspace = torch.empty(self.stride * self.capacity, dtype=torch.uint8, device="cuda")
        elif workspace.numel() < self.stride * self.capacity or workspace.data_ptr() % 256:
            raise ValueError("workspace too small or not 256-byte aligned")
        self.workspace = workspace
        self.J = None
        self.shifts: list[complex] = []

    def _shift_array(self) -> np.ndarray:
        sh = np.zeros(2 * len(self.shifts))
        sh[0::2] = np.real(self.shifts)
        sh[1::2] = np.imag(self.shifts)
        return sh

    def factor(self, J, shifts) -> None:
        """Factors J - s I for every shift s; ``J`` is one device Jacobian for all shifts or a
        sequence of one per shift (instances of the same grid size)."""
        shifts = [complex(v) for v in np.atleast_1d(shifts)]
        n = len(shifts)
        if not 1 <= n <= self.capacity:
            raise ValueError(f"{n} shifts for {self.capacity} workspaces")
        Js = list(J) if isinstance(J, (list, tuple)) else [J] * n
        if len(Js) != n:
            raise ValueError(f"{len(Js)} Jacobians for {n} shifts")
        self.J, self.shifts = None, shifts
        sh = self._shift_array()
        jp = (ctypes.c_void_p * n)(*[j.data_ptr() for j in Js])
        rc = self._lib.eb_ringlu_factor_many(ctypes.byref(self.batch), jp, n,
                                             sh.ctypes.data, self.workspace.data_ptr(),
                                             self.stride,
                                             self._torch.cuda.current_stream().cuda_stream)
        if rc != _lib.EB_OK:
            raise _lib.EulerB200Error("eb_ringlu_factor_many", rc,
                                      self._lib.eb_last_error().decode())
        self.J = Js

    def solve_one(self, k: int, rhs, adjoint: bool = False):
        """Solves the system of shift ``k`` alone (``eb_ringlu_solve`` on its workspace) for one
        device right-hand side; returns ``(x, rel_residual)``."""
        if self.J is None or not 0 <= k < len(self.shifts):
            raise ValueError("no factors for that shift")
        torch = self._torch
        x = torch.empty_like(rhs)
        rel = ctypes.c_double()
        s = self.shifts[k]
        rc = self._lib.eb_ringlu_solve(ctypes.byref(self.batch), self.J[k].data_ptr(), s.real,
                                       s.imag, 1 if adjoint else 0,
                                       self.workspace.data_ptr() + k * self.stride, self.stride,
                                       rhs.data_ptr(), x.data_ptr(), self.tol, self.max_refine,
                                       ctypes.byref(rel),
                                       torch.cuda.current_stream().cuda_stream)
        if rc != _lib.EB_OK:
            raise _lib.EulerB200Error("eb_ringlu_solve", rc, self._lib.eb_last_error().decode())
        return x, rel.value

    def solve(self, rhs, adjoint: bool = False, out=None):
        """Solves system ``s`` for ``rhs[s]`` (a sequence of, or a stacked, device tensor);
        returns ``(x, rel_residuals)`` with ``x`` stacked like ``rhs``."""
        if self.J is None:
            raise RuntimeError("factor() first")
        n = len(self.shifts)
        if len(rhs) != n:
            raise ValueError(f"{len(rhs)} right-hand sides for {n} shifts")
        torch = self._torch
        x = (torch.empty_like(rhs) if isinstance(rhs, torch.Tensor)
             else [torch.empty_like(r) for r in rhs]) if out is None else out
        sh = self._shift_array()
        rp = (ctypes.c_void_p * n)(*[rhs[k].data_ptr() for k in range(n)])
        xp = (ctypes.c_void_p * n)(*[x[k].data_ptr() for k in range(n)])
        rel = (ctypes.c_double * n)()
        jp = (ctypes.c_void_p * n)(*[j.data_ptr() for j in self.J])
        rc = self._lib.eb_ringlu_solve_many(ctypes.byref(self.batch), jp, n,
                                            sh.ctypes.data, 1 if adjoint else 0,
                                            self.workspace.data_ptr(), self.stride, rp, xp,
                                            self.tol, self.max_refine, rel,
                                            torch.cuda.current_stream().cuda_stream)
        if rc != _lib.EB_OK:
            raise _lib.EulerB200Error("eb_ringlu_solve_many", rc,
                                      self._lib.eb_last_error().decode() + f" (rel {list(rel)})")
        return x, list(rel)


def solve_shifted_noalloc(batch: _lib.Batch, J, rhs, shifts, *, adjoint: bool = False,
                          tol: float = 1e-10, restart: int = 60, maxiter: int = 3000,
                          check_every: int = 10, x=None, sys_inst=None, host_table=None):
    """``solve_shifted`` through ``eb_gmres_solve_noalloc``: no device workspace is allocated.

    For callers that cannot allocate device memory (their memory belongs to another runtime's
    pool, or their loop may not allocate once running): the solver's workspace is the
    library's fixed 48 MiB device array. ``x`` may be given to avoid allocating the solution
    vector too. Calls that overlap on the GPU share that array and race.
    """
    import torch

    lib = _lib.load()
    if not getattr(lib, "_noalloc_bound", False):
        lib.eb_gmres_solve_noalloc.restype = ctypes.c_int
        lib.eb_gmres_solve_noalloc.argtypes = [
            ctypes.POINTER(_lib.Batch), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.POINTER(GmresOptions), ctypes.POINTER(GmresInfo), ctypes.c_void_p]
        lib._noalloc_bound = True
    n_sys = len(shifts)
    sh = np.zeros(2 * n_sys)
    sh[0::2] = np.real(shifts)
    sh[1::2] = np.imag(shifts)
    inst = None if sys_inst is None else np.ascontiguousarray(sys_inst, dtype=np.int32)
    x = torch.empty_like(rhs) if x is None else x
    opts = GmresOptions(float(tol), int(restart), int(maxiter), int(check_every), 0)
    infos = (GmresInfo * n_sys)()
    rc = lib.eb_gmres_solve_noalloc(
        ctypes.byref(batch), None if host_table is None else ctypes.addressof(host_table),
        J.data_ptr(), n_sys, None if inst is None else inst.ctypes.data, sh.ctypes.data,
        1 if adjoint else 0, rhs.data_ptr(), x.data_ptr(), ctypes.byref(opts), infos,
        torch.cuda.current_stream().cuda_stream)
    if rc != _lib.EB_OK:
        raise _lib.EulerB200Error("eb_gmres_solve_noalloc", rc, lib.eb_last_error().decode())
    return x, SolveInfo({"iterations": i.iterations, "cycles": i.cycles,
                         "converged": bool(i.converged), "rel_residual": i.rel_residual}
                        for i in infos)


def _bind_ptc() -> ctypes.CDLL:
    lib = _lib.load()
    if not getattr(lib, "_ptc_bound", False):
        P = ctypes.c_void_p
        lib.eb_ptc_workspace_bytes.restype = ctypes.c_int64
        lib.eb_ptc_workspace_bytes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.eb_ptc_run.restype = ctypes.c_int
        lib.eb_ptc_run.argtypes = [ctypes.POINTER(_lib.Batch), P, P, P, P, P, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, P, ctypes.c_int64,
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                   P]
        lib._ptc_bound = True
    return lib


def ptc_run(batch: _lib.Batch, X, V, U, R, J, ser: float = 0.1, rtol: float = 1e-9,
            max_steps: int = 100, workspace=None):
    """The PTC/SER steady-state loop of one instance on the device (``eb_ptc_run``).

    ``X``, ``V``, ``U`` (updated in place), ``R`` and ``J`` (receiving the final residual and
    states Jacobian) are device float64 tensors in the reference layouts. Returns
    ``(norms, rel_norms, status)``: per step max|R| and max|R| / max|R_0|, and the C ABI status
    (``EB_OK``, or ``EB_ERR_NAN`` when the residual became non-finite or a ring block singular).
    """
    import torch

    lib = _bind_ptc()
    need = lib.eb_ptc_workspace_bytes(batch.single.M, batch.single.N, int(max_steps))
    if need < 0:
        raise ValueError("PTC needs a single instance with M >= 4, N >= 5")
    if workspace is None or workspace.numel() < need or workspace.data_ptr() % 256:
        workspace = torch.empty(int(need), dtype=torch.uint8, device=U.device)
    hist = (ctypes.c_double * (2 * int(max_steps)))()
    n = ctypes.c_int(0)
    V_ptr = None if V is None else V.data_ptr()
    rc = lib.eb_ptc_run(ctypes.byref(batch), X.data_ptr(), V_ptr, U.data_ptr(), R.data_ptr(),
                        J.data_ptr(), float(ser), float(rtol), int(max_steps),
                        workspace.data_ptr(), int(workspace.numel()), hist, ctypes.byref(n),
                        torch.cuda.current_stream().cuda_stream)
    if rc not in (_lib.EB_OK, _lib.EB_ERR_NAN):
        raise _lib.EulerB200Error("eb_ptc_run", rc, lib.eb_last_error().decode())
    vals = list(hist)[:2 * n.value]
    return vals[0::2], vals[1::2], rc
