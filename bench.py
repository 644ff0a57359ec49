#!/usr/bin/env python
"""Throughput of the B200 spatial discretization on the 129x129 NACA-0004 workload.

Workload (seeded synthetic inputs; the reference publishes no benchmark dataset): the
129x129 NACA-0004 O-grid of chord 10 with a far field at radius 200 (first spacing 0.1),
Ma 0.5, alpha 0, moment centre (2.5, 0); states = free stream x (1 + 1 % Gaussian noise),
a smooth seeded grid-velocity field. A batch of B instances (default 256 per GPU, 4.2 M cells,
~400 MB of residual inputs + outputs, well above the 126 MB L2) is packed into one instance
table.

One timed "step" is one residual evaluation R(Ma, U, X, V) of the whole batch (one launch).
The JSON line reports cell-residual evaluations per second (``value``), and beside it the VJP
rate (full set of reverse products per instance: d/dU, d/dX, d/dV, d/dMa), the linearisation
rates (the d(odes)/d(states) Jacobian, the matrix-free tangent, the forward products, the
shifted BSR SpMV), the 13 second-order inner-product gradients and the resolvent rate: the
pitch frequency response (64 shifts) plus the adjoint lift gradient of the PTC steady state of
one instance, solved to 1e-10 relative residual, with the shifts factored together (batched)
and one at a time through the drop-in class (plain).

``--impl reference`` times the CPU restatement of the reference (complex arithmetic, all host
threads) on a bounded sample of the same workload. Under torchrun every rank processes its own
B instances (weak scaling; instances are independent, no data-path collective).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-residual evals/s; VJP/s; batched resolvent solves/s vs plain at 1e-10 rel"
UNIT = "cell-residual evals/s"
BYTES_PER_CELL_RESIDUAL = 96          # U 32 + X 16 + V 16 + R 32 (FP64)
BYTES_PER_CELL_VJP = 1152 + 256 + 256 + 32 + 4 * 64 + 64 + 2 * 32 + 8
# matrix-free VJP set: U, X, V and complex w in; complex d_states, d_vertices, d_velocities out
BYTES_PER_CELL_ADJOINT = 32 + 16 + 16 + 64 + 64 + 32 + 32
BYTES_PER_CELL_JAC_STATES = 32 + 16 + 16 + 1152   # U, X, V in; nine 4x4 blocks out
# U, X, V, complex dU, dX, dV in; complex dR out
BYTES_PER_CELL_TANGENT = 32 + 16 + 16 + 64 + 32 + 32 + 64
# per product: Jacobian + complex direction in, complex d_odes out (states 1152 + 64 + 64,
# vertices and velocities 256 + 32 + 64 each, Mach 32 + 64)
BYTES_PER_CELL_JVP = 1280 + 2 * 352 + 96
LINEAR_SPMV_INSTANCES = 16          # BSR matrices cycled by the SpMV timing (~343 MB)
SPMV_STREAMS = 4                    # streams the captured SpMVs are spread over
GRID = dict(radial_pts=129, angular_pts=129, thickness=0.04, chord=10.0, far_radius=200.0,
            first_spacing=0.1)
FLOW = dict(mach=0.5, aoa_deg=0.0, center=(2.5, 0.0))
PROFILE_SUMMARY = ROOT / "profiles" / "residual_tiled_naca0004_129x129.md"


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--instances", type=int, default=256, help="instances per GPU")
    p.add_argument("--shifts", type=int, default=4,
                   help="frequency-response shifts timed one at a time (plain path)")
    p.add_argument("--batched-shifts", type=int, default=64,
                   help="frequency-response shifts timed through the batched driver")
    p.add_argument("--parts",
                   default="residual,vjp,linear,second_order,adjoint257,resolvent,uneven",
                   help="comma-separated parts to run besides the residual "
                        "(vjp, linear, second_order, adjoint257, resolvent, uneven)")
    p.add_argument("--uneven-instances", type=int, default=48)
    p.add_argument("--uneven-sizes", default="65,129,257,513x257",
                   help="O-grid point counts the uneven instances draw from: n (n x n) or "
                        "RxA (R radial x A angular points)")
    p.add_argument("--uneven-iter", type=int, default=30, help="PTC iteration cap")
    p.add_argument("--uneven-plain", type=int, default=1,
                   help="instances of each size timed one at a time for the comparison")
    p.add_argument("--workspace-gb", type=float, default=80.0,
                   help="device memory for batched factorisations")
    p.add_argument("--profile-region", choices=["none", "residual", "batched", "anchored"],
                   default="none",
                   help="bracket one region with cudaProfilerStart/Stop (for "
                        "ncu --profile-from-start off): the timed residual launches or the "
                        "batched frequency response")
    p.add_argument("--per-anchor", type=int, default=3,
                   help="frequency-response shifts per factorised anchor (anchored method)")
    p.add_argument("--shift-group", type=int, default=32,
                   help="shifts factored concurrently (one workspace of ~2.7 GB each)")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline budget")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--dry-run", action="store_true",
                   help="rank plumbing only (gloo on the CPU, no GPU work): every rank joins, "
                        "times an empty region, and rank 0 prints the JSON line")
    return p.parse_args()


def launch_ranks(args) -> int | None:
    """Starts one rank per GPU when ``--gpus N`` (N > 1) is given outside a torchrun launch.

    Re-executes this script under ``torch.distributed.run`` (one node, N processes, rendezvous
    on 127.0.0.1) and returns its exit code; returns None when this process already is a rank
    (WORLD_SIZE set) or when one GPU is asked for.
    """
    if args.gpus <= 1 or "WORLD_SIZE" in os.environ:
        return None
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def run_dry(args) -> None:
    """The multi-rank skeleton of the B200 arm without a GPU: gloo process group, barrier,
    max over ranks of a timed empty region, one JSON line from rank 0."""
    import datetime

    import torch.distributed as dist

    from pyeulerale_b200.batch import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but {world} ranks were started")
    t0 = time.perf_counter()
    if world > 1:
        dist.barrier()
    t = max_over_ranks(time.perf_counter() - t0)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": None, "unit": UNIT, "n_gpus": world,
                          "dry_run": True, "max_rank_seconds": t,
                          "config": {"instances_per_gpu": args.instances,
                                     "parallelism": f"replicas x{world}"}}), flush=True)


# ---- workload -------------------------------------------------------------------------------

def workload(n_inst: int, seed: int):
    from pyeulerale_b200 import grid

    X = grid.naca_ogrid(GRID["radial_pts"], GRID["angular_pts"], GRID["thickness"],
                        GRID["chord"], GRID["far_radius"], GRID["first_spacing"])
    M, N = X.shape[1] - 1, X.shape[2] - 1
    rng = np.random.default_rng(seed)
    Us = [grid.perturbed_states(M, N, FLOW["mach"], FLOW["aoa_deg"], 0.01, rng)
          for _ in range(n_inst)]
    V = grid.smooth_velocities(X, rng, amplitude=0.01)
    return X, V, Us


# ---- clocks ---------------------------------------------------------------------------------

class ClockSampler:
    """SM clock and throttle-reason sampling (NVML, every 5 ms) during the timed region."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, device_index: int) -> None:
        self.device_index = device_index
        self.samples: list[tuple[int, int]] = []
        self._stop = None
        self._thread = None
        self.max_mhz = None

    def __enter__(self):
        import threading

        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception:  # NVML unavailable: report unsampled
            return self
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    mhz = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((mhz, reasons))
                except Exception:
                    pass
                self._stop.wait(0.005)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        time.sleep(0.05)
        return self

    def __exit__(self, *exc):
        if self._thread:
            self._stop.set()
            self._thread.join(timeout=5)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        mhz = [m for m, _ in self.samples]
        loaded = [m for m in mhz if m > 0.5 * max(mhz)]
        reasons = sorted({name for _, r in self.samples for name, bit in self.REASONS.items()
                          if r & bit})
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples)}


# ---- CPU baseline (the oracle) --------------------------------------------------------------

def cpu_model() -> str:
    """The host CPU's model name and logical core count (Linux /proc/cpuinfo)."""
    try:
        names = [ln.split(":", 1)[1].strip() for ln in open("/proc/cpuinfo")
                 if ln.startswith("model name")]
        return f"{names[0]} ({len(names)} logical cores)" if names else "unknown"
    except OSError:
        return "unknown"


def cpu_residual_rate(X, V, Us, threads: int, budget_s: float) -> tuple[float, str]:
    """Cells/s of the complex-arithmetic oracle residual on a bounded sample."""
    from oracle.shim import SpatialDiscretizationModule, load_library

    lib = load_library()
    lib.sdo_set_threads(threads)
    ora = SpatialDiscretizationModule()
    ora.aoa[...] = FLOW["aoa_deg"]
    Xc = np.asfortranarray(X, dtype=complex)
    Vc = np.asfortranarray(V, dtype=complex)
    M, N = Us[0].shape[1], Us[0].shape[2]
    R = np.asfortranarray(np.zeros((4, M, N), dtype=complex))
    Uc = [np.asfortranarray(u, dtype=complex) for u in Us]
    ora.compute_odes(FLOW["mach"], Xc, Vc, Uc[0], R)  # warm-up
    cells, t0, k = 0, time.perf_counter(), 0
    while time.perf_counter() - t0 < budget_s:
        ora.compute_odes(FLOW["mach"], Xc, Vc, Uc[k % len(Uc)], R)
        cells += M * N
        k += 1
    dt = time.perf_counter() - t0
    lib.sdo_set_threads(1)
    return cells / dt, f"{k} residual evaluations of one {M}x{N} instance in {dt:.1f} s"


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.shim import load_library

    threads = load_library().sdo_max_threads()
    X, V, Us = workload(4, seed=0)
    per_step = max(0.2, min(1.0, 60.0 / max(args.steps, 1)))

    # warm-up steps, then timed steps (each a bounded sample of the workload)
    for _ in range(args.warmup):
        cpu_residual_rate(X, V, Us, threads, 0.2)
    rates = []
    sample = ""
    for _ in range(args.steps):
        r, sample = cpu_residual_rate(X, V, Us, threads, per_step)
        rates.append(r)
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * 128 * 128 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded NACA-0004 O-grid)",
        "config": {"workload": "residual of the 129x129 NACA-0004 O-grid (128x128 cells), "
                               "Ma 0.5, alpha 0, complex arithmetic as the reference",
                   "cells_per_instance": 128 * 128},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "cpu": cpu_model(),
                         "sample": f"per step: {sample}; C++ restatement of "
                                   "src/spatial_discretization.f90 (oracle/sd_oracle.cpp)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_resolvent_rate(X, V, U, mach: float, shift: complex) -> dict:
    """Shifted solves/s of the reference's own resolvent method on the host: the Jacobian from
    the oracle, then per shift the CSR assembly and SuperLU (scipy.sparse.linalg.spsolve), as
    SpatialDiscretization._assemble_csr / solve_odes_wrt_states_fwd do (core.py:512-565).
    One shift is the bounded sample (SuperLU is single-threaded)."""
    from scipy.sparse import bsr_array
    from scipy.sparse.linalg import spsolve

    from oracle.shim import SpatialDiscretizationModule

    M, N = U.shape[1], U.shape[2]
    disc = SpatialDiscretizationModule()
    disc.aoa[...] = FLOW["aoa_deg"]
    t0 = time.perf_counter()
    J = np.zeros((4, 4, M, N, 9), order="F")
    disc.compute_odes_wrt_states(mach, np.asarray(X, complex), np.asarray(V, complex),
                                 np.asarray(U, complex), J)
    nnzb = (9 * M - 6) * N
    data = np.empty((4, 4, nnzb), order="F")
    idx = np.empty(nnzb, dtype=np.intc)
    ptr = np.empty(M * N + 1, dtype=np.intc)
    disc.convert_odes_wrt_states(J, data, idx, ptr)
    t_lin = time.perf_counter() - t0
    b = np.array([1.0, 1j]) @ np.random.default_rng(5).standard_normal((2, 4 * M * N))
    t0 = time.perf_counter()
    A = bsr_array((np.moveaxis(data, -1, 0), idx - 1, ptr - 1), dtype=complex).tocsr()
    A.setdiag(A.diagonal() - shift)
    x = spsolve(A, b)
    t_solve = time.perf_counter() - t0
    rel = float(np.linalg.norm(A @ x - b) / np.linalg.norm(b))
    return {"value": 1.0 / t_solve, "unit": "shifted solves/s", "cores": 1, "kind": "port",
            "cpu": cpu_model(),
            "sample": f"one solve at shift {shift:.4g} of the {M}x{N}-cell steady-state "
                      f"Jacobian in {t_solve:.1f} s (relative residual {rel:.1e}); the Jacobian "
                      f"and its BSR form (oracle, complex step) took {t_lin:.1f} s once",
            "method": "CSR assembly + SuperLU (scipy.sparse.linalg.spsolve) per shift, as "
                      "core.py:512-565"}


def cpu_linear_rates(X, V, U, mach: float) -> dict:
    """The reference's own linearisation procedures on the host, in its single thread (the
    oracle restatement of src/spatial_discretization.f90): the complex-step d(odes)/d(states)
    Jacobian (f90:666-750), the four forward and the four reverse products with the stored
    Jacobians (f90:604-650, 825-918, 1005-1072) of one 128x128 instance, its BSR conversion
    (f90:765-814), and the matrix-vector product of the CSR matrix that _assemble_csr builds
    (core.py:512-531) under scipy."""
    from scipy.sparse import bsr_array

    from oracle.shim import SpatialDiscretizationModule

    M, N = U.shape[1], U.shape[2]
    disc = SpatialDiscretizationModule()
    disc.aoa[...] = FLOW["aoa_deg"]
    Xc, Vc, Uc = (np.asfortranarray(np.asarray(a, dtype=complex)) for a in (X, V, U))
    J_u = np.zeros((4, 4, M, N, 9), order="F")
    J_x = np.zeros((4, 2, M, N, 4), order="F")
    J_v = np.zeros((4, 2, M, N, 4), order="F")
    J_m = np.zeros((4, 1, M, N), order="F")

    def per_call(fn, budget=0.5):
        fn()
        n, t0 = 0, time.perf_counter()
        while True:
            fn()
            n += 1
            t = time.perf_counter() - t0
            if t >= budget:
                return t / n

    t_jac = per_call(lambda: disc.compute_odes_wrt_states(mach, Xc, Vc, Uc, J_u), 1.0)
    disc.compute_odes_wrt_vertices(mach, Xc, Vc, Uc, J_x)
    disc.compute_odes_wrt_velocities(mach, Xc, Vc, Uc, J_v)
    disc.compute_odes_wrt_mach(mach, Xc, Vc, Uc, J_m)
    rng = np.random.default_rng(9)

    def crand(shape):
        return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))

    cells, verts = (4, M, N), (2, M + 1, N + 1)
    w, gU, gX, gV, gM = crand(cells), crand(cells), crand(verts), crand(verts), crand((1,))

    def vjp():
        disc.apply_odes_wrt_states_rev(J_u, w, gU)
        disc.apply_odes_wrt_vertices_rev(J_x, w, gX)
        disc.apply_odes_wrt_vertices_rev(J_v, w, gV)
        disc.apply_odes_wrt_mach_rev(J_m, w, gM)

    dU, dXv, dVv, dm = crand(cells), crand(verts), crand(verts), crand((1,))
    jR = [crand(cells) for _ in range(4)]

    def jvp():
        disc.apply_odes_wrt_states_fwd(J_u, dU, jR[0])
        disc.apply_odes_wrt_vertices_fwd(J_x, dXv, jR[1])
        disc.apply_odes_wrt_vertices_fwd(J_v, dVv, jR[2])
        disc.apply_odes_wrt_mach_fwd(J_m, dm, jR[3])

    t_vjp, t_jvp = per_call(vjp), per_call(jvp)
    nnzb = (9 * M - 6) * N
    data = np.empty((4, 4, nnzb), order="F")
    idx = np.empty(nnzb, dtype=np.intc)
    ptr = np.empty(M * N + 1, dtype=np.intc)
    t_conv = per_call(lambda: disc.convert_odes_wrt_states(J_u, data, idx, ptr))
    A = bsr_array((np.moveaxis(data, -1, 0), idx - 1, ptr - 1), dtype=complex).tocsr()
    x = crand(4 * M * N)
    t_spmv = per_call(lambda: A @ x)
    return {"jacobian_states": {"value": M * N / t_jac, "unit": "cells/s"},
            "vjp": {"value": 1.0 / t_vjp, "unit": "VJP/s (four reverse products, one instance)"},
            "jvp": {"value": 1.0 / t_jvp, "unit": "JVP/s (four forward products, one instance)"},
            "bsr_conversion": {"value": 1.0 / t_conv,
                               "unit": "conversions/s (the oracle's O(nnz) restatement; the "
                                       "reference's Fortran loop is O((MN)^2), f90:765-814)"},
            "bsr_spmv": {"value": 1.0 / t_spmv, "unit": "SpMV/s (scipy CSR, complex x)"},
            "cores": 1, "kind": "port", "cpu": cpu_model(),
            "sample": f"one {M}x{N}-cell instance, each procedure repeated for >= 0.5 s"}


def cpu_second_order_rate(X, V, U, mach: float) -> dict:
    """The reference's second-order method on the host for one routine,
    compute_odes_wrt_states_inner_product_wrt_states (core.py:761-802): central differences of
    complex-step Jacobians, four d(odes)/d(states) builds (real and imaginary part of the
    direction, plus and minus the step) and four reverse products, with the oracle restatement
    of the Fortran procedures."""
    from oracle.shim import SpatialDiscretizationModule

    M, N = U.shape[1], U.shape[2]
    disc = SpatialDiscretizationModule()
    disc.aoa[...] = FLOW["aoa_deg"]
    Xc, Vc, Uc = (np.asfortranarray(np.asarray(a, dtype=complex)) for a in (X, V, U))
    rng = np.random.default_rng(13)
    d_states = np.asfortranarray(rng.standard_normal((4, M, N)) + 1j * rng.standard_normal((4, M, N)))
    d_odes = np.asfortranarray(rng.standard_normal((4, M, N)) + 1j * rng.standard_normal((4, M, N)))
    t0 = time.perf_counter()
    grad = np.zeros((4, M, N), dtype=complex, order="F")
    vjp = np.zeros((4, M, N), dtype=complex, order="F")
    Jp = np.zeros((4, 4, M, N, 9), order="F")
    step = 1e-6 * (1.0 + np.linalg.norm(Uc)) ** 0.5 / np.linalg.norm(d_states)
    for sign in (1.0, -1.0):
        for part, factor in ((np.real, 1.0), (np.imag, 1j)):
            disc.compute_odes_wrt_states(mach, Xc, Vc, Uc + sign * step * part(d_states), Jp)
            disc.apply_odes_wrt_states_rev(Jp, d_odes.conj(), vjp)
            grad += sign * factor * vjp
    grad = grad / 2.0 / step
    t = time.perf_counter() - t0
    return {"value": 1.0 / t, "unit": "routine calls/s (one 128x128 instance)", "cores": 1,
            "kind": "port", "cpu": cpu_model(),
            "sample": f"compute_odes_wrt_states_inner_product_wrt_states once in {t:.2f} s "
                      "(four complex-step Jacobian builds and reverse products, core.py:761-802)"}


# ---- B200 arm -------------------------------------------------------------------------------

def time_zgemm(K: int, batch: int, stream, sp, reps: int = 10) -> dict:
    """The ring LU's dense product at its factorisation shape (K x K x K complex, batch shifts):
    the library's two GEMM variants (eb_zgemm_strided_batched) and, for comparison only, the
    BLAS product torch.matmul issues on the same shape."""
    import torch
    from pyeulerale_b200 import _lib

    g = torch.Generator(device="cuda").manual_seed(3)
    A, B, C = (torch.randn(batch, K, K, dtype=torch.complex128, device="cuda", generator=g)
               for _ in range(3))
    flops = 8.0 * K ** 3 * batch
    out = {"shape": f"{K}x{K}x{K} complex, batch {batch}", "flops_per_call": flops}

    def timed(fn):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    for v, name in ((0, "register_staged"), (1, "cp_async"), (2, "cp_async_64x32")):
        def call(v=v):
            _lib.call("eb_zgemm_strided_batched", K, K, K, -1.0, A.data_ptr(), K, K * K,
                      B.data_ptr(), K, K * K, 1.0, C.data_ptr(), K, K * K, batch, v, sp)
        t = timed(call)
        out[name] = {"ms": t * 1e3, "tflops": flops / t / 1e12}
    with torch.cuda.stream(stream):
        t = timed(lambda: torch.matmul(A, B, out=C))
    out["blas_torch_matmul"] = {"ms": t * 1e3, "tflops": flops / t / 1e12,
                                "note": "library comparison only; not on the product path"}
    return out


def read_traffic() -> float | None:
    """DRAM bytes per residual launch from the committed ncu summary, scaled per cell."""
    if not PROFILE_SUMMARY.exists():
        return None
    for line in PROFILE_SUMMARY.read_text().splitlines():
        if line.startswith("dram_bytes_per_cell:"):
            return float(line.split(":")[1])
    return None


def run_b200(args) -> None:
    import torch
    import torch.distributed as dist

    from pyeulerale_b200 import _lib
    from pyeulerale_b200.batch import InstanceSet, InstanceSpec, max_over_ranks

    parts = set(args.parts.split(","))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but {world} ranks were started")
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    _lib.load()
    B = args.instances
    X, V, Us = workload(B, seed=1000 + rank)
    specs = [InstanceSpec(X, FLOW["mach"], FLOW["aoa_deg"], GRID["chord"], FLOW["center"])
             for _ in range(B)]
    inst = InstanceSet(specs)
    cells = inst.n_cells
    f64 = dict(dtype=torch.float64, device="cuda")
    hX = torch.from_numpy(inst.pack_vertices()).pin_memory()
    hV = torch.from_numpy(inst.pack_vertices([V] * B)).pin_memory()
    hU = torch.from_numpy(inst.pack_cells(Us)).pin_memory()
    hR = torch.empty(4 * cells, dtype=torch.float64).pin_memory()
    dX, dV, dU = hX.cuda(), hV.cuda(), hU.cuda()
    dR = torch.empty(4 * cells, **f64)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def residual():
        inst.call("eb_compute_odes", dX, dV, dU, dR, stream=sp)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # residual: warm-up, then K timed launches
    for _ in range(args.warmup):
        residual()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        if args.profile_region == "residual":
            torch.cuda.profiler.start()
        ev0.record(stream)
        for _ in range(args.steps):
            residual()
        ev1.record(stream)
        barrier()
        if args.profile_region == "residual":
            torch.cuda.profiler.stop()
    t_res = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    clk = clocks.summary()
    value = world * cells * args.steps / t_res
    per_launch = t_res / args.steps
    achieved = BYTES_PER_CELL_RESIDUAL * cells / per_launch / 1e9
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) \
        if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_source = ("MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks else
                   "no MEASURED_PEAKS.json on this machine: the pool's earlier measured copy "
                   "bandwidth 6650 GB/s (of fallback)")
    traffic_cell = read_traffic()

    # FP64 throughput (the FP64 roofline denominator): the library's DFMA probe on every SM
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    sink = torch.zeros(1, **f64)
    fma_iters = 100_000

    def fma_probe():
        _lib.call("eb_fp64_fma_probe", fma_iters, sms, sink.data_ptr(), sp)

    for _ in range(3):
        fma_probe()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(5):
        fma_probe()
    f1.record(stream)
    barrier()
    t_fma = f0.elapsed_time(f1) / 1e3 / 5
    fp64_peak_tflops = 2.0 * 8 * sms * 256 * 8 * fma_iters / t_fma / 1e12
    # FP64 tensor-core throughput (the dense products' denominator): the library's DMMA probe
    mma_iters = 20_000
    for _ in range(3):
        _lib.call("eb_fp64_mma_probe", mma_iters, sms, sink.data_ptr(), sp)
    f0.record(stream)
    for _ in range(5):
        _lib.call("eb_fp64_mma_probe", mma_iters, sms, sink.data_ptr(), sp)
    f1.record(stream)
    barrier()
    t_mma = f0.elapsed_time(f1) / 1e3 / 5
    fp64_mma_tflops = 512.0 * 8 * (4 * sms * 256 // 32) * mma_iters / t_mma / 1e12

    # end to end through the C ABI with host buffers: every step copies its inputs (X, V, U)
    # from pinned host memory and its result R back. Serial: one stream, copies and launch in
    # sequence. Pipelined (the reported e2e): pyeulerale_b200.pipeline.ResidualPipeline, step
    # k+1's inputs, step k's residual and step k-1's result in flight together.
    from pyeulerale_b200.pipeline import ResidualPipeline

    e2e_steps = max(3, args.steps // 5)
    for _ in range(max(1, args.warmup // 2)):
        dX.copy_(hX, non_blocking=True)
        dV.copy_(hV, non_blocking=True)
        dU.copy_(hU, non_blocking=True)
        residual()
        hR.copy_(dR, non_blocking=True)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        dX.copy_(hX, non_blocking=True)
        dV.copy_(hV, non_blocking=True)
        dU.copy_(hU, non_blocking=True)
        residual()
        hR.copy_(dR, non_blocking=True)
    e1.record(stream)
    barrier()
    t_serial = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    del dX, dV, dU, dR  # the pipeline holds its own device buffers
    pipe = ResidualPipeline(inst, depth=2)
    for _ in range(max(2, args.warmup // 2)):
        pipe.submit(hX, hV, hU, hR)
    pipe.synchronize()
    barrier()
    e0.record(pipe.s_in)
    for _ in range(e2e_steps):
        pipe.submit(hX, hV, hU, hR)
    e1.record(pipe.s_out)
    pipe.synchronize()
    barrier()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    h2d = (hX.numel() + hV.numel() + hU.numel()) * 8
    d2h = hR.numel() * 8
    e2e_value = world * cells * e2e_steps / t_e2e
    e2e_serial = world * cells * e2e_steps / t_serial
    dX, dV, dU = pipe.bufs[0]["X"], pipe.bufs[0]["V"], pipe.bufs[0]["U"]

    # VJP set (d/dU, d/dX, d/dV, d/dMa of <w, R> per instance, complex w as the reference's
    # reverse products take): the matrix-free adjoint kernel from (U, X, V, w), all work timed;
    # beside it the reverse products with stored Jacobians, alone and with the Jacobian builds
    vjp = None
    if "vjp" in parts:
        w = torch.randn(8 * cells, **f64)
        gU = torch.empty(8 * cells, **f64)
        gX = torch.empty(4 * inst.n_verts, **f64)
        gV = torch.empty(4 * inst.n_verts, **f64)
        gM = torch.empty(2 * B, **f64)

        def timed(fn, n):
            for _ in range(args.warmup):
                fn()
            barrier()
            v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            v0.record(stream)
            for _ in range(n):
                fn()
            v1.record(stream)
            barrier()
            return max_over_ranks(v0.elapsed_time(v1) / 1e3) / n

        def adjoint():
            inst.call("eb_apply_odes_adjoint", dX, dV, dU, w, 1, gU, gX, gV, gM, stream=sp)

        t_adj = timed(adjoint, max(5, args.steps // 4))
        J_u = torch.empty(144 * cells, **f64)
        J_x = torch.empty(32 * cells, **f64)
        J_v = torch.empty(32 * cells, **f64)
        J_m = torch.empty(4 * cells, **f64)

        def build():
            inst.call("eb_compute_odes_wrt_states", dX, dV, dU, J_u, stream=sp)
            inst.call("eb_compute_odes_wrt_vertices", dX, dV, dU, J_x, stream=sp)
            inst.call("eb_compute_odes_wrt_velocities", dX, dV, dU, J_v, stream=sp)
            inst.call("eb_compute_odes_wrt_mach", dX, dV, dU, J_m, stream=sp)

        def products():
            inst.call("eb_apply_odes_wrt_states_rev", J_u, w, gU, stream=sp)
            inst.call("eb_apply_odes_wrt_vertices_rev", J_x, w, gX, stream=sp)
            inst.call("eb_apply_odes_wrt_vertices_rev", J_v, w, gV, stream=sp)
            inst.call("eb_apply_odes_wrt_mach_rev", J_m, w, gM, stream=sp)

        t_build = timed(build, 3)
        t_prod = timed(products, max(5, args.steps // 2))
        vjp = {"value": world * B / t_adj,
               "unit": "VJP/s (dR/dU, dR/dX, dR/dV, dR/dMa of <w, R> per instance, from U, X, "
                       "V and complex w, all work timed)",
               "kernel": "k_residual_adjoint + k_mach_adjoint (eb_apply_odes_adjoint)",
               "achieved_gbs": BYTES_PER_CELL_ADJOINT * cells / t_adj / 1e9,
               "bytes_per_cell": BYTES_PER_CELL_ADJOINT,
               "cells_per_s": world * cells / t_adj,
               "stored_blocks": {
                   "value": world * B / t_prod,
                   "unit": "VJP/s, reverse products with the Jacobians already built",
                   "achieved_gbs": BYTES_PER_CELL_VJP * cells / t_prod / 1e9,
                   "launches_per_vjp_batch": 4},
               "stored_blocks_with_build": {
                   "value": world * B / (t_build + t_prod),
                   "unit": "VJP/s, Jacobian builds (states, vertices, velocities, Mach) + "
                           "reverse products"}}
        del J_u, J_x, J_v, J_m, gU, gX, gV, gM, w

    # linearisation: the 4x4-block Jacobian d(odes)/d(states) of every instance, the
    # matrix-free forward tangent (complex dU, dX, dV, dMa in one stencil pass) of every
    # instance, and the shifted BSR SpMV (A - s I) x cycled over the BSR forms of
    # LINEAR_SPMV_INSTANCES instances (more bytes than L2 holds, so every pass reads HBM)
    linear = cpu_lin = None
    if "linear" in parts:
        def per_call(fn, n):
            for _ in range(args.warmup):
                fn()
            barrier()
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(n):
                fn()
            z.record(stream)
            barrier()
            return max_over_ranks(a.elapsed_time(z) / 1e3) / n

        J_u = torch.empty(144 * cells, **f64)
        t_jac = per_call(lambda: inst.call("eb_compute_odes_wrt_states", dX, dV, dU, J_u,
                                           stream=sp), 5)
        t_jac_plain = per_call(lambda: inst.call("eb_compute_odes_wrt_states_untiled", dX, dV,
                                                 dU, J_u, stream=sp), 2)
        inst.call("eb_compute_odes_wrt_states", dX, dV, dU, J_u, stream=sp)
        gen = torch.Generator(device="cuda").manual_seed(77 + rank)
        tU = torch.randn(8 * cells, generator=gen, **f64)
        tX = torch.randn(4 * inst.n_verts, generator=gen, **f64)
        tV = torch.randn(4 * inst.n_verts, generator=gen, **f64)
        tM = torch.randn(2 * B, generator=gen, **f64)
        tR = torch.empty(8 * cells, **f64)
        t_tan = per_call(lambda: inst.call("eb_apply_odes_tangent", dX, dV, dU, tU, tX, tV, tM,
                                           tR, None, stream=sp), max(5, args.steps // 4))
        # JVP set: the four forward products with stored Jacobians, each into its own d_odes
        J_x = torch.empty(32 * cells, **f64)
        J_v = torch.empty(32 * cells, **f64)
        J_m = torch.empty(4 * cells, **f64)
        inst.call("eb_compute_odes_wrt_vertices", dX, dV, dU, J_x, stream=sp)
        inst.call("eb_compute_odes_wrt_velocities", dX, dV, dU, J_v, stream=sp)
        inst.call("eb_compute_odes_wrt_mach", dX, dV, dU, J_m, stream=sp)
        jR = [torch.empty(8 * cells, **f64) for _ in range(4)]

        def jvp():
            inst.call("eb_apply_odes_wrt_states_fwd", J_u, tU, jR[0], stream=sp)
            inst.call("eb_apply_odes_wrt_vertices_fwd", J_x, tX, jR[1], stream=sp)
            inst.call("eb_apply_odes_wrt_vertices_fwd", J_v, tV, jR[2], stream=sp)
            inst.call("eb_apply_odes_wrt_mach_fwd", J_m, tM, jR[3], stream=sp)

        t_jvp = per_call(jvp, max(5, args.steps // 4))
        del J_x, J_v, J_m, jR
        M1, N1 = specs[0].M, specs[0].N
        rows, nnzb = M1 * N1, (9 * M1 - 6) * N1
        one = InstanceSet(specs[:1])
        n_mat = min(LINEAR_SPMV_INSTANCES, B)
        mats = []
        for i in range(n_mat):
            data = torch.empty(16 * nnzb, **f64)
            idx = torch.empty(nnzb, dtype=torch.int32, device="cuda")
            ptr = torch.empty(rows + 1, dtype=torch.int32, device="cuda")
            one.call("eb_convert_odes_wrt_states", J_u[144 * inst.cell_offsets[i]:], data, idx,
                     ptr, stream=sp)
            mats.append((data, idx, ptr))
        data0, idx0, ptr0 = mats[0]
        t_conv = per_call(lambda: one.call("eb_convert_odes_wrt_states", J_u, data0, idx0, ptr0,
                                           stream=sp), max(5, args.steps // 4))
        sx = torch.randn(8 * rows * n_mat, generator=gen, **f64)
        sy = torch.empty(8 * rows * n_mat, **f64)

        def spmv_all(st):
            for i, (data, idx, ptr) in enumerate(mats):
                _lib.call("eb_bsr_shifted_spmv", rows, data.data_ptr(), idx.data_ptr(),
                          ptr.data_ptr(), 0.0, 1.5, sx[8 * rows * i:].data_ptr(),
                          sy[8 * rows * i:].data_ptr(), st)

        # one SpMV moves ~21 MB (~4 us of HBM time), less than the host needs to issue a call
        # and about one launch's ramp and tail: the n_mat independent calls are captured once
        # in a CUDA graph, spread over SPMV_STREAMS streams so that their launches overlap,
        # and the graph is replayed
        spmv_all(sp)
        barrier()
        spmv_graph = torch.cuda.CUDAGraph()
        side = [torch.cuda.Stream() for _ in range(SPMV_STREAMS)]
        with torch.cuda.graph(spmv_graph):
            cap = torch.cuda.current_stream()
            for k, s in enumerate(side):
                s.wait_stream(cap)
                with torch.cuda.stream(s):
                    for i in range(k, n_mat, SPMV_STREAMS):
                        data, idx, ptr = mats[i]
                        _lib.call("eb_bsr_shifted_spmv", rows, data.data_ptr(),
                                  idx.data_ptr(), ptr.data_ptr(), 0.0, 1.5,
                                  sx[8 * rows * i:].data_ptr(), sy[8 * rows * i:].data_ptr(),
                                  s.cuda_stream)
            for s in side:
                cap.wait_stream(s)
        t_spmv = per_call(spmv_graph.replay, max(5, args.steps // 4)) / n_mat
        spmv_bytes = nnzb * (128 + 4) + (rows + 1) * 4 + rows * (64 + 64)
        linear = {
            "jacobian_states": {"value": world * cells / t_jac, "unit": "cells/s",
                                "achieved_gbs": BYTES_PER_CELL_JAC_STATES * cells / t_jac / 1e9,
                                "bytes_per_cell": BYTES_PER_CELL_JAC_STATES,
                                "kernel": "k_jac_states_tiled",
                                "untiled": {"value": world * cells / t_jac_plain,
                                            "kernel": "k_jac_states (one thread per cell)"}},
            "tangent": {"value": world * cells / t_tan, "unit": "cells/s",
                        "achieved_gbs": BYTES_PER_CELL_TANGENT * cells / t_tan / 1e9,
                        "bytes_per_cell": BYTES_PER_CELL_TANGENT,
                        "direction": "complex dU, dX, dV, dMa together"},
            "jvp": {"value": world * B / t_jvp,
                    "unit": "JVP/s (dR/dU, dR/dX, dR/dV, dR/dMa forward products per instance)",
                    "achieved_gbs": BYTES_PER_CELL_JVP * cells / t_jvp / 1e9,
                    "bytes_per_cell": BYTES_PER_CELL_JVP, "launches_per_jvp_batch": 4},
            "bsr_conversion": {"value": world / t_conv,
                               "unit": "conversions/s (one 128x128 instance: 146,688 blocks, "
                                       "1-based indices as the reference emits them)",
                               "achieved_gbs": (1152 * rows + nnzb * (128 + 4)
                                                + (rows + 1) * 4) / t_conv / 1e9},
            "bsr_spmv": {"value": world / t_spmv, "unit": "SpMV/s (one 128x128 instance)",
                         "achieved_gbs": spmv_bytes / t_spmv / 1e9,
                         "bytes_per_spmv": spmv_bytes, "nnzb": nnzb,
                         "matrices_cycled": n_mat,
                         "issue": f"the {n_mat} calls captured in one CUDA graph on "
                                  f"{SPMV_STREAMS} streams, replayed"},
            "peak_gbs": peak}
        if rank == 0 and not args.no_cpu_baseline:
            cpu_lin = cpu_linear_rates(X, V, Us[0], FLOW["mach"])
            linear["cpu_reference_method"] = cpu_lin
            for key in ("jacobian_states", "jvp", "bsr_conversion", "bsr_spmv"):
                linear[key]["vs_cpu_reference_method"] = \
                    linear[key]["value"] / cpu_lin[key]["value"]
        del J_u, tU, tX, tV, tR, mats, sx, sy, spmv_graph, side

    # second order: the 13 inner-product gradients of the drop-in class (core.py:718-1275) on
    # one 128x128 instance, host arrays in and out as the reference's API has them (each call
    # builds one directional Jacobian on the device in nested duals and applies its reverse
    # product); beside it the reference's finite-difference method for one of them on the host
    second = None
    if "second_order" in parts:
        from pyeulerale_b200 import SpatialDiscretization

        sd2 = SpatialDiscretization(X, mach_number=FLOW["mach"], angle_of_attack=FLOW["aoa_deg"],
                                    coefficient_length=GRID["chord"],
                                    coefficient_center=FLOW["center"])
        sd2.states[...] = Us[0]
        M2, N2 = sd2.num_radial, sd2.num_angular
        srng = np.random.default_rng(31 + rank)

        def crand(shape):
            return np.asfortranarray(srng.standard_normal(shape)
                                     + 1j * srng.standard_normal(shape))

        w, dS = crand((4, M2, N2)), crand((4, M2, N2))
        dXs, dVs, dF = crand((2, M2 + 1, N2 + 1)), crand((2, M2 + 1, N2 + 1)), crand((2, N2))
        routines = [
            lambda: sd2.compute_odes_wrt_states_inner_product_wrt_mach(w, dS),
            lambda: sd2.compute_odes_wrt_states_inner_product_wrt_states(w, dS),
            lambda: sd2.compute_odes_wrt_states_inner_product_wrt_vertices(w, dS),
            lambda: sd2.compute_odes_wrt_vertices_inner_product_wrt_mach(w, dXs),
            lambda: sd2.compute_odes_wrt_vertices_inner_product_wrt_states(w, dXs),
            lambda: sd2.compute_odes_wrt_vertices_inner_product_wrt_vertices(w, dXs),
            lambda: sd2.compute_odes_wrt_velocities_inner_product_wrt_mach(w, dVs),
            lambda: sd2.compute_odes_wrt_velocities_inner_product_wrt_states(w, dVs),
            lambda: sd2.compute_odes_wrt_velocities_inner_product_wrt_vertices(w, dVs),
            lambda: sd2.compute_forces_wrt_states_inner_product_wrt_states(dF, dS),
            lambda: sd2.compute_forces_wrt_states_inner_product_wrt_vertices(dF, dS),
            lambda: sd2.compute_forces_wrt_vertices_inner_product_wrt_states(dF, dXs),
            lambda: sd2.compute_forces_wrt_vertices_inner_product_wrt_vertices(dF, dXs),
        ]
        for fn in routines:
            fn()
        barrier()
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            for fn in routines:
                fn()
        barrier()
        t_so = max_over_ranks(time.perf_counter() - t0)
        second = {"value": world * reps * len(routines) / t_so,
                  "unit": "second-order routine calls/s (drop-in class, host arrays, one "
                          "128x128 instance per call)",
                  "routines": len(routines), "calls": reps * len(routines), "seconds": t_so}
        if rank == 0 and not args.no_cpu_baseline:
            second["cpu_reference_method"] = cpu_second_order_rate(X, V, Us[0], FLOW["mach"])
            second["vs_cpu_reference_method"] = \
                (second["value"] / world) / second["cpu_reference_method"]["value"]
        del sd2

    # the adjoint workload at full size: NACA-0012 257x257 O-grid (chord 1, far field 20
    # chords), Ma 0.6, alpha 2 deg, the PTC state (to rel 1e-4: past 2.8e-5 the reference's PTC
    # law leaves the basin on this transonic case) plus a seeded 1e-3 perturbation and a smooth
    # grid-velocity field; each operation per call: the matrix-free VJP of R on the device, and
    # through the drop-in class (host arrays, the reference's API) the stored-Jacobian VJPs of
    # R and F, a second-order gradient and the adjoint lift gradient
    adj257 = None
    if "adjoint257" in parts:
        from pyeulerale_b200 import SpatialDiscretization, drivers
        from pyeulerale_b200 import grid as G

        X7 = G.naca_ogrid(257, 257, thickness=0.12, chord=1.0, far_radius=20.0,
                          first_spacing=0.01)
        s7 = SpatialDiscretization(X7, mach_number=0.6, angle_of_attack=2.0,
                                   coefficient_length=1.0, coefficient_center=(0.25, 0.0))
        t0 = time.perf_counter()
        hist7 = drivers.ptc(s7, rtol=1e-4, max_iter=20)
        t_ptc7 = time.perf_counter() - t0
        arng = np.random.default_rng(257)
        s7.states[:] = s7.states * (1.0 + 1e-3 * arng.standard_normal(s7.states.shape))
        s7.velocities[:] = G.smooth_velocities(X7, arng)
        s7.compute_odes()
        s7.compute_forces()
        t0 = time.perf_counter()
        s7.linearize()
        t_lin7 = time.perf_counter() - t0
        M7, N7 = s7.num_radial, s7.num_angular

        def unit(shape):
            a = arng.standard_normal(shape) + 1j * arng.standard_normal(shape)
            return np.asfortranarray(a / np.linalg.norm(a))

        w7, wf7, d7 = unit((4, M7, N7)), unit((2, N7)), unit((4, M7, N7))
        dw7 = torch.from_numpy(np.ascontiguousarray(w7.ravel(order="F")).view(np.float64)).cuda()
        g7 = [torch.empty(n, **f64) for n in (8 * M7 * N7, 4 * (M7 + 1) * (N7 + 1),
                                              4 * (M7 + 1) * (N7 + 1), 2)]

        def matrix_free():
            s7._call("eb_apply_odes_adjoint", s7._dX.data_ptr(), s7._dV.data_ptr(),
                     s7._dU.data_ptr(), dw7.data_ptr(), 1, *[g.data_ptr() for g in g7])
            torch.cuda.synchronize()

        ops = {
            "vjp_matrix_free": matrix_free,
            "vjp_states": lambda: s7.apply_odes_wrt_states_rev(w7),
            "vjp_vertices": lambda: s7.apply_odes_wrt_vertices_rev(w7),
            "vjp_velocities": lambda: s7.apply_odes_wrt_velocities_rev(w7),
            "vjp_mach": lambda: s7.apply_odes_wrt_mach_rev(w7),
            "forces_vjp_states": lambda: s7.apply_forces_wrt_states_rev(wf7),
            "forces_vjp_vertices": lambda: s7.apply_forces_wrt_vertices_rev(wf7),
            "second_order_states_states":
                lambda: s7.compute_odes_wrt_states_inner_product_wrt_states(w7, d7),
            "adjoint_lift_gradient": lambda: drivers.adjoint_lift_gradient(s7),
        }
        times, first = {}, {}
        for name, fn in ops.items():
            barrier()
            t0 = time.perf_counter()
            fn()
            barrier()
            first[name] = max_over_ranks(time.perf_counter() - t0)
            n = 2 if name == "adjoint_lift_gradient" else 5
            t0 = time.perf_counter()
            for _ in range(n):
                fn()
            barrier()
            times[name] = max_over_ranks(time.perf_counter() - t0) / n
        adj257 = {"value": 1.0 / times["vjp_matrix_free"],
                  "unit": "matrix-free VJPs/s (dR/dU, dR/dX, dR/dV, dR/dMa of <w, R>, one "
                          "257x257 instance, device arrays)",
                  "workload": "NACA-0012 257x257 O-grid, Ma 0.6, alpha 2 deg, PTC state + 1e-3 "
                              "perturbation, smooth grid velocities",
                  "ms_per_call": {k: v * 1e3 for k, v in times.items()},
                  "ms_first_call": {k: v * 1e3 for k, v in first.items()},
                  "note": "per call through the drop-in class with host arrays in and out, "
                          "except vjp_matrix_free (device arrays); the adjoint lift gradient's "
                          "first call factors the Jacobian at shift 0 (ring LU), later calls "
                          "reuse the factors (the drop-in keeps them while the Jacobian and "
                          "the shift are unchanged)",
                  "ptc": {"iterations": hist7.iterations, "final_rel_residual":
                          hist7.rel_norms[-1], "seconds": t_ptc7},
                  "linearize_seconds": t_lin7}
        del s7, g7, dw7

    # resolvent: the frequency response of the steady state (PTC from free stream), 64 shifts
    # s = i k V / (c / 2), k log-spaced on [0.01, 10], plus the adjoint lift gradient; batched
    # (anchored GMRES, the headline; and the direct ring LU of every shift, shift_group shifts
    # per factorisation call) against one shift at a time through the drop-in class
    res = None
    if "resolvent" in parts:
        from pyeulerale_b200 import SpatialDiscretization, drivers

        sd = SpatialDiscretization(X, mach_number=FLOW["mach"], angle_of_attack=FLOW["aoa_deg"],
                                   coefficient_length=GRID["chord"],
                                   coefficient_center=FLOW["center"])
        sd_rings, sd_cols = sd.num_radial, sd.num_angular
        t0 = time.perf_counter()
        hist = drivers.ptc(sd, rtol=1e-10, max_iter=200)
        t_ptc = time.perf_counter() - t0
        ks = np.logspace(-2, 1, max(args.batched_shifts, 1))
        ks_plain = ks[np.linspace(0, len(ks) - 1, max(min(args.shifts, len(ks)), 1)).astype(int)]
        drivers.frequency_response(sd, GRID["chord"], FLOW["center"][0], ks_plain[:1])  # warm-up
        barrier()
        t0 = time.perf_counter()
        cl_p, cm_p = drivers.frequency_response(sd, GRID["chord"], FLOW["center"][0], ks_plain)
        grad_p = drivers.adjoint_lift_gradient(sd)
        barrier()
        t_plain = max_over_ranks(time.perf_counter() - t0)
        group = max(1, min(args.shift_group, len(ks)))
        drivers.frequency_response_batched(sd, GRID["chord"], FLOW["center"][0], ks[:group],
                                           group=group)  # warm-up
        barrier()
        t0 = time.perf_counter()
        if args.profile_region == "batched":
            torch.cuda.profiler.start()
        cl_b, cm_b = drivers.frequency_response_batched(sd, GRID["chord"], FLOW["center"][0], ks,
                                                        group=group)
        if args.profile_region == "batched":
            torch.cuda.profiler.stop()
        grad_b = drivers.adjoint_lift_gradient(sd)
        barrier()
        t_batched = max_over_ranks(time.perf_counter() - t0)
        sel = np.searchsorted(ks, ks_plain)

        def agree_with_plain(cl, cm):
            return max(float(np.max(np.abs(cl[sel] - cl_p)) / np.max(np.abs(cl_p))),
                       float(np.max(np.abs(cm[sel] - cm_p)) / np.max(np.abs(cm_p))))

        # anchored: GMRES on every shift, preconditioned by the ring-LU factors of one anchor
        # per per_anchor shifts (the unconverged, if any, solved directly)
        drivers.frequency_response_batched(sd, GRID["chord"], FLOW["center"][0],
                                           ks[:2 * args.per_anchor], method="anchored",
                                           per_anchor=args.per_anchor)  # warm-up
        stats = {}
        barrier()
        t0 = time.perf_counter()
        if args.profile_region == "anchored":
            torch.cuda.profiler.start()
        cl_a, cm_a, grad_a = drivers.frequency_response_batched(
            sd, GRID["chord"], FLOW["center"][0], ks, method="anchored",
            per_anchor=args.per_anchor, stats=stats, lift_gradient=True)
        if args.profile_region == "anchored":
            torch.cuda.profiler.stop()
        barrier()
        t_anch = max_over_ranks(time.perf_counter() - t0)
        plain_rate = world * len(ks_plain) / t_plain
        batched_rate = world * len(ks) / t_batched
        anchored_rate = world * len(ks) / t_anch
        its = stats.get("iterations", [])
        res = {"value": anchored_rate,
               "unit": "transfer-function shifts/s (solve to 1e-10 relative residual + forces)",
               "workload": f"{len(ks)}-shift pitch frequency response of the PTC steady state "
                           "of the 129x129 NACA-0004 grid plus the adjoint lift gradient",
               "shifts": len(ks), "seconds": t_anch,
               "method": f"GMRES(40) per shift, right-preconditioned by the ring-LU factors of "
                         f"its anchor ({stats.get('anchors')} anchors, {args.per_anchor} shifts "
                         "each, factored in one batched call together with shift 0 for the "
                         "adjoint lift gradient); every shift to 1e-12 relative residual (so "
                         "that the transfer function agrees with the direct solves, themselves "
                         "at 1e-10)",
               "iterations": {"min": min(its, default=0), "median": float(np.median(its)) if its
                              else 0, "max": max(its, default=0), "sum": int(sum(its))},
               "direct_fallback_shifts": stats.get("direct"),
               "plain": {"value": plain_rate, "shifts": len(ks_plain), "seconds": t_plain},
               "batched_vs_plain": anchored_rate / plain_rate,
               "max_rel_diff_batched_vs_plain": agree_with_plain(cl_a, cm_a),
               "max_rel_diff_anchored_vs_direct": max(
                   float(np.max(np.abs(cl_a - cl_b)) / np.max(np.abs(cl_b))),
                   float(np.max(np.abs(cm_a - cm_b)) / np.max(np.abs(cm_b)))),
               "adjoint_gradient_rel_diff": float(np.max(np.abs(grad_a - grad_p))
                                                  / np.max(np.abs(grad_p))),
               "direct": {
                   "value": batched_rate, "shift_group": group, "seconds": t_batched,
                   "batched_vs_plain": batched_rate / plain_rate,
                   "achieved_tflops": len(ks) * sd_rings * 4 * (4 * sd_cols) ** 3 * 8
                   / t_batched / 1e12,
                   "flops": "4 (4N)^3 complex multiply-adds (8 flops) per ring and shift: the "
                            "Gauss-Jordan inversion and the three Schur / L products of the "
                            "factorisation, over the whole batched time",
                   "max_rel_diff_batched_vs_plain": agree_with_plain(cl_b, cm_b),
                   "method": "ring-block LU of every shift (batched Gauss-Jordan ring "
                             "inversions + strided-batched ZGEMM), refined to 1e-10"},
               "ptc": {"iterations": hist.iterations, "final_rel_residual": hist.rel_norms[-1],
                       "seconds": t_ptc}}
        res["dense_products"] = time_zgemm(4 * sd_cols, min(group, 16), stream, sp)
        if rank == 0 and not args.no_cpu_baseline:
            res["cpu_reference_method"] = cpu_resolvent_rate(
                sd.vertices, sd.velocities, sd.states, FLOW["mach"],
                1j * ks[0] * FLOW["mach"] * 1.4 ** 0.5 / (GRID["chord"] / 2))
            res["batched_vs_cpu_reference_method"] = \
                batched_rate / res["cpu_reference_method"]["value"]
        del sd

    # uneven instances: steady states (PTC) and adjoint lift gradients of many grids of
    # different sizes, thicknesses, Mach numbers and angles, batched (one launch per kernel over
    # all instances, equal-size instances factored together) against one instance at a time
    uneven = None
    if "uneven" in parts:
        from pyeulerale_b200 import SpatialDiscretization, drivers
        from pyeulerale_b200 import grid as G

        urng = np.random.default_rng(4 + rank)
        size_names = args.uneven_sizes.split(",")

        def points(name):
            r, _, a = name.partition("x")
            return int(r), int(a or r)

        uspecs, uclass = [], []
        for _ in range(args.uneven_instances):
            name = size_names[int(urng.integers(len(size_names)))]
            tt = int(urng.choice([4, 6, 8, 10, 12]))
            rp, ap = points(name)
            Xg = G.naca_ogrid(rp, ap, thickness=tt / 100, chord=1.0, far_radius=20.0,
                              first_spacing=0.01)
            uspecs.append(InstanceSpec(Xg, float(urng.uniform(0.3, 0.6)),
                                       float(urng.uniform(-2.0, 3.0)), 1.0, (0.25, 0.0)))
            uclass.append(name)
        uinst = InstanceSet(uspecs)
        ws_bytes = int(args.workspace_gb * (1 << 30))
        barrier()
        t0 = time.perf_counter()
        ures = drivers.ptc_batched(uinst, rtol=1e-10, max_iter=args.uneven_iter,
                                   workspace_bytes=ws_bytes)
        drivers.adjoint_lift_gradients_batched(uinst, ures, workspace_bytes=ws_bytes)
        barrier()
        t_ub = max_over_ranks(time.perf_counter() - t0)
        conv = sum(1 for h in ures.rel_norms if h and h[-1] <= 1e-10)
        iters = max(len(h) for h in ures.rel_norms)
        del ures
        torch.cuda.empty_cache()
        # plain: the first `uneven_plain` instances of each size one at a time through the
        # drop-in class; the plain time of the whole set is each size's mean time x its count
        per_size = {}
        for name in size_names:
            members = [k for k, c in enumerate(uclass) if c == name][:args.uneven_plain]
            if not members:
                continue
            barrier()
            t0 = time.perf_counter()
            for k in members:
                sp = uspecs[k]
                sd = SpatialDiscretization(sp.vertices, mach_number=sp.mach,
                                           angle_of_attack=sp.aoa_deg,
                                           coefficient_length=sp.chord,
                                           coefficient_center=sp.center)
                hist = drivers.ptc(sd, rtol=1e-10, max_iter=args.uneven_iter)
                if np.isfinite(hist.rel_norms[-1]):
                    try:
                        drivers.adjoint_lift_gradient(sd)
                    except _lib.EulerB200Error:
                        pass  # a singular adjoint system, as in the batched path
                del sd
                torch.cuda.empty_cache()
            barrier()
            dt = max_over_ranks(time.perf_counter() - t0)
            per_size[name] = {"count": uclass.count(name), "timed": len(members),
                              "seconds_per_instance": dt / len(members)}
        t_up = sum(v["count"] * v["seconds_per_instance"] for v in per_size.values())
        n_set = sum(v["count"] for v in per_size.values())
        uneven = {"value": world * len(uspecs) / t_ub,
                  "unit": "instances/s (PTC to 1e-10 + adjoint lift gradient)",
                  "workload": f"{len(uspecs)} NACA-00tt O-grids drawn from the sizes "
                              f"{size_names} (tt in 4..12, Ma in [0.3, 0.6], alpha in [-2, 3] "
                              "deg), per GPU",
                  "sizes": [int(s) if s.isdigit() else s for s in size_names],
                  "counts": {s: uclass.count(s) for s in size_names},
                  "seconds": t_ub, "converged": conv, "iterations_max": iters,
                  "plain": {"value": world * n_set / t_up, "per_size": per_size,
                            "seconds_estimated": t_up,
                            "method": "drop-in class, one instance at a time (PTC + adjoint); "
                                      "the set's plain time = per-size time x count"},
                  "batched_vs_plain": (len(uspecs) / t_ub) / (n_set / t_up)}
        del uinst

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        rate, sample = cpu_residual_rate(X, V, Us[:4], 1, args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port", "cpu": cpu_model(),
               "sample": f"{sample}; single-threaded like the reference; C++ restatement "
                         "of src/spatial_discretization.f90 in complex arithmetic"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * per_launch, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded NACA-0004 O-grid, perturbed free stream, smooth grid "
                "velocities)",
        "config": {"workload": f"residual of {B} instances of the 129x129 NACA-0004 O-grid "
                               "(128x128 cells each) per GPU, one launch per step",
                   "instances_per_gpu": B, "cells_per_gpu": cells,
                   "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": None if traffic_cell is None else traffic_cell * cells,
                     "traffic_source": None if traffic_cell is None else
                     f"ncu capture summarised in profiles/{PROFILE_SUMMARY.name} (DRAM bytes "
                     "per cell of the same kernel, scaled to this launch's cells), not "
                     "measured in this run",
                     "algorithmic_bytes_per_launch": BYTES_PER_CELL_RESIDUAL * cells,
                     "peak_source": peak_source},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                "path": "pyeulerale_b200.pipeline.ResidualPipeline (copies and launches of "
                        "consecutive steps overlapped on three streams)",
                "serial": {"value": e2e_serial,
                           "path": "one stream: H2D of X, V, U, eb_compute_odes, D2H of R"}},
        "gpu_launches": args.steps,
        "clocks": clk,
        "vjp": None if vjp is None else {
            **vjp, "roofline_frac": vjp["achieved_gbs"] / peak,
            "cpu_reference_method": None if cpu_lin is None else cpu_lin["vjp"],
            "vs_cpu_reference_method": None if cpu_lin is None
            else vjp["value"] / cpu_lin["vjp"]["value"]},
        "linear": linear,
        "autotune": _lib.autotune_report().splitlines(),
        "fp64_peak": {"tflops": fp64_peak_tflops, "sms": sms,
                      "probe": "eb_fp64_fma_probe: 8 CTAs x 256 threads per SM, 8 independent "
                               f"DFMA chains of {fma_iters} per thread, CUDA events",
                      "mma_tflops": fp64_mma_tflops,
                      "mma_probe": "eb_fp64_mma_probe: 4 CTAs x 8 warps per SM, 8 independent "
                                   f"m8n8k4 FP64 accumulators of {mma_iters} MMAs per warp"},
        "second_order": second,
        "adjoint257": adj257,
        "resolvent": res,
        "uneven": uneven,
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    rc = launch_ranks(args)
    if rc is not None:
        sys.exit(rc)
    if args.dry_run:
        run_dry(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
