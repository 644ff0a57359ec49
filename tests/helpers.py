"""Test helpers: seeded cases, and the same quantities from the CUDA library and the oracle."""

from __future__ import annotations

import ctypes

import numpy as np

from pyeulerale_b200 import grid as G


def make_case(name: str, golden_grids: dict, seed: int = 0) -> dict:
    """Seeded input sets: vertices, velocities, states (real, Fortran order) + flow."""
    rng = np.random.default_rng(seed)
    if name == "ref8x9":
        X = golden_grids["naca0012_8x9"]
        M, N = X.shape[1] - 1, X.shape[2] - 1
        U = G.perturbed_states(M, N, 0.5, 1.25, 0.005, rng)
        return dict(X=X, V=np.zeros_like(X), U=U, mach=0.5, aoa=1.25)
    if name == "naca0012_33":  # 33x33 O-grid, chord 1, far field 20 chords, 1 % noise
        X = G.naca_ogrid(33, 33, thickness=0.12, chord=1.0, far_radius=20.0, first_spacing=0.01)
        U = G.perturbed_states(32, 32, 0.5, 1.25, 0.01, rng)
        return dict(X=X, V=np.zeros_like(X), U=U, mach=0.5, aoa=1.25)
    if name == "naca0012_33_moving":  # same grid with a smooth vertex velocity field
        X = G.naca_ogrid(33, 33, thickness=0.12, chord=1.0, far_radius=20.0, first_spacing=0.01)
        U = G.perturbed_states(32, 32, 0.6, 2.0, 0.01, rng)
        V = G.smooth_velocities(X, rng)
        return dict(X=X, V=V, U=U, mach=0.6, aoa=2.0)
    if name == "min4x5":  # the smallest grid the reference handles: M = 4, N = 5
        X = G.naca_ogrid(5, 6, thickness=0.12, chord=1.0, far_radius=10.0, first_spacing=0.05)
        U = G.perturbed_states(4, 5, 0.5, 1.25, 0.01, rng)
        V = G.smooth_velocities(X, rng)
        return dict(X=X, V=V, U=U, mach=0.5, aoa=1.25)
    if name == "naca0004_129":
        X = golden_grids["naca0004_129x129"]
        U = G.perturbed_states(128, 128, 0.5, 0.0, 0.01, rng)
        return dict(X=X, V=np.zeros_like(X), U=U, mach=0.5, aoa=0.0)
    if name == "naca0004_33_sym":
        # every fourth vertex of the shipped 129x129 grid: its leading- and trailing-edge lines
        # lie exactly on z = 0, and at alpha = 0 the states have j2 = 0 exactly, so the faces
        # on those lines carry exactly zero normal velocity (abs_c's derivative sign at zero)
        X = np.asfortranarray(golden_grids["naca0004_129x129"][:, ::4, ::4])
        U = G.perturbed_states(32, 32, 0.5, 0.0, 0.01, rng)
        return dict(X=X, V=np.zeros_like(X), U=U, mach=0.5, aoa=0.0)
    raise KeyError(name)


def oracle_eval(oracle, case: dict) -> dict:
    """Residual, forces and complex-step Jacobians of the oracle (reference layouts)."""
    X = np.asfortranarray(case["X"], dtype=complex)
    V = np.asfortranarray(case["V"], dtype=complex)
    U = np.asfortranarray(case["U"], dtype=complex)
    M, N = U.shape[1], U.shape[2]
    oracle.aoa[...] = case["aoa"]
    mach = case["mach"]
    out = {}
    R = np.asfortranarray(np.zeros((4, M, N), dtype=complex))
    oracle.compute_odes(mach, X, V, U, R)
    out["R"] = R.real.copy()
    F = np.asfortranarray(np.zeros((2, N), dtype=complex))
    oracle.compute_forces(X, U, F)
    out["F"] = F.real.copy()
    shapes = {"J_ma": (4, 1, M, N), "J_u": (4, 4, M, N, 9), "J_x": (4, 2, M, N, 4),
              "J_v": (4, 2, M, N, 4), "JF_u": (2, 4, N), "JF_x": (2, 2, N, 2)}
    J = {k: np.asfortranarray(np.zeros(s)) for k, s in shapes.items()}
    oracle.compute_odes_wrt_mach(mach, X, V, U, J["J_ma"])
    oracle.compute_odes_wrt_states(mach, X, V, U, J["J_u"])
    oracle.compute_odes_wrt_vertices(mach, X, V, U, J["J_x"])
    oracle.compute_odes_wrt_velocities(mach, X, V, U, J["J_v"])
    oracle.compute_forces_wrt_states(X, U, J["JF_u"])
    oracle.compute_forces_wrt_vertices(X, U, J["JF_x"])
    out.update(J)
    return out


class Gpu:
    """Device copies of one case and thin wrappers of the C ABI entry points."""

    def __init__(self, torch, case: dict) -> None:
        from pyeulerale_b200 import _lib

        self.torch, self.lib = torch, _lib
        U = case["U"]
        self.M, self.N = U.shape[1], U.shape[2]
        self.inst = _lib.make_instance(self.M, self.N, case["mach"], case["aoa"])
        self.batch = _lib.single_batch(self.inst)
        self.X = self.dev(case["X"])
        self.V = self.dev(case["V"])
        self.U = self.dev(U)

    def dev(self, a: np.ndarray):
        flat = np.ascontiguousarray(np.asarray(a).ravel(order="F"))
        if np.iscomplexobj(flat):
            flat = flat.view(np.float64)
        return self.torch.from_numpy(flat.astype(np.float64)).cuda()

    def empty(self, n: int):
        return self.torch.zeros(n, dtype=self.torch.float64, device="cuda")

    def call(self, name: str, *args) -> None:
        self.lib.call(name, ctypes.byref(self.batch), *[
            a.data_ptr() if hasattr(a, "data_ptr") else a for a in args], None)

    @staticmethod
    def host(t, shape, complex_: bool = False) -> np.ndarray:
        a = t.cpu().numpy()
        if complex_:
            a = a.view(np.complex128)
        return np.asfortranarray(np.reshape(a, shape, order="F"))

    def evaluate(self) -> dict:
        M, N = self.M, self.N
        nc = M * N
        R, F = self.empty(4 * nc), self.empty(2 * N)
        self.call("eb_compute_odes", self.X, self.V, self.U, R)
        self.call("eb_compute_forces", self.X, self.U, F, None)
        J = {"J_ma": self.empty(4 * nc), "J_u": self.empty(144 * nc), "J_x": self.empty(32 * nc),
             "J_v": self.empty(32 * nc), "JF_u": self.empty(8 * N), "JF_x": self.empty(8 * N)}
        self.call("eb_compute_odes_wrt_mach", self.X, self.V, self.U, J["J_ma"])
        self.call("eb_compute_odes_wrt_states", self.X, self.V, self.U, J["J_u"])
        self.call("eb_compute_odes_wrt_vertices", self.X, self.V, self.U, J["J_x"])
        self.call("eb_compute_odes_wrt_velocities", self.X, self.V, self.U, J["J_v"])
        self.call("eb_compute_forces_wrt_states", self.X, self.U, J["JF_u"])
        self.call("eb_compute_forces_wrt_vertices", self.X, self.U, J["JF_x"])
        self.torch.cuda.synchronize()
        shapes = {"J_ma": (4, 1, M, N), "J_u": (4, 4, M, N, 9), "J_x": (4, 2, M, N, 4),
                  "J_v": (4, 2, M, N, 4), "JF_u": (2, 4, N), "JF_x": (2, 2, N, 2)}
        out = {"R": self.host(R, (4, M, N)), "F": self.host(F, (2, N))}
        out.update({k: self.host(v, shapes[k]) for k, v in J.items()})
        out["_dev"] = J
        return out


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """Norm-wise (max-norm) relative difference |a - b|_inf / |b|_inf."""
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))


def crandn(rng, shape) -> np.ndarray:
    a = np.empty(shape, order="F", dtype=complex)
    a[:] = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return a
