"""Packed instance tables: many grids (of uneven sizes, Mach numbers and angles) in one launch.

An ``InstanceSet`` packs the per-instance arrays back to back (cells, vertices, wall faces) and
owns the device copy of the ``eb_instance`` table, so every kernel of the C ABI processes all
instances in a single launch. ``shard`` splits a list of instances across ranks (contiguous
blocks; the instances are independent, so no data-path collective is needed).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class InstanceSpec:
    """One grid with its flow parameters."""

    vertices: np.ndarray              # (2, M+1, N+1)
    mach: float
    aoa_deg: float
    chord: float = 1.0
    center: tuple[float, float] = (0.0, 0.0)
    k2: float = 1.0
    k4: float = 1.0 / 32
    c4: float = 2.0

    @property
    def M(self) -> int:
        return self.vertices.shape[1] - 1

    @property
    def N(self) -> int:
        return self.vertices.shape[2] - 1


class InstanceSet:
    """Packed instances with their host and device instance tables."""

    def __init__(self, specs: list[InstanceSpec]) -> None:
        import torch

        self.specs = specs
        n = len(specs)
        self.host_table = (_lib.Instance * n)()
        c = v = w = 0
        self.cell_offsets, self.vert_offsets, self.wall_offsets = [], [], []
        for i, s in enumerate(specs):
            if s.M < 4 or s.N < 5:
                raise ValueError(f"instance {i}: grid needs M >= 4 and N >= 5 cells")
            self.host_table[i] = _lib.make_instance(s.M, s.N, s.mach, s.aoa_deg, s.k2, s.k4,
                                                    s.c4, s.chord, s.center, c, v, w)
            self.cell_offsets.append(c)
            self.vert_offsets.append(v)
            self.wall_offsets.append(w)
            c += s.M * s.N
            v += (s.M + 1) * (s.N + 1)
            w += s.N
        self.n_cells, self.n_verts, self.n_wall = c, v, w
        raw = np.frombuffer(bytes(self.host_table), dtype=np.uint8).copy()
        self.device_table = torch.from_numpy(raw).cuda()
        b = _lib.Batch()
        if n == 1:
            b.d_table = None
            b.single = self.host_table[0]
        else:
            b.d_table = self.device_table.data_ptr()
        b.n_inst = n
        b.max_dim = max(max(s.M, s.N) for s in specs)
        b.n_cells, b.n_verts, b.n_wall = c, v, w
        self.batch = b

    def __len__(self) -> int:
        return len(self.specs)

    def set_mach(self, mach) -> None:
        """Sets the free-stream Mach number of every instance (host and device tables)."""
        import torch

        values = [float(v) for v in (mach.tolist() if hasattr(mach, "tolist") else mach)]
        if len(values) != len(self.specs):
            raise ValueError(f"{len(values)} Mach numbers for {len(self.specs)} instances")
        if all(v == self.host_table[i].mach for i, v in enumerate(values)):
            return
        for i, v in enumerate(values):
            self.specs[i].mach = v
            self.host_table[i].mach = v
        raw = np.frombuffer(bytes(self.host_table), dtype=np.uint8).copy()
        self.device_table.copy_(torch.from_numpy(raw))
        if len(self.specs) == 1:
            self.batch.single = self.host_table[0]

    def pack_vertices(self, arrays: list[np.ndarray] | None = None) -> np.ndarray:
        """Packed (2, ...) vertex-like arrays (default: the grids) as a flat float64 array."""
        arrays = arrays if arrays is not None else [s.vertices for s in self.specs]
        return np.concatenate([np.asarray(a, dtype=np.float64).ravel(order="F")
                               for a in arrays])

    def pack_cells(self, arrays: list[np.ndarray]) -> np.ndarray:
        """Packed (4, M, N) per-cell arrays as a flat array (complex stays complex)."""
        return np.concatenate([np.asarray(a).ravel(order="F") for a in arrays])

    def unpack_cells(self, flat: np.ndarray, per_cell: int = 4) -> list[np.ndarray]:
        out = []
        for s, off in zip(self.specs, self.cell_offsets):
            n = per_cell * s.M * s.N
            out.append(np.reshape(flat[per_cell * off: per_cell * off + n],
                                  (per_cell, s.M, s.N), order="F"))
        return out

    def call(self, name: str, *args, stream=None) -> None:
        """Calls a batch entry point of the C ABI with device tensors / pointers."""
        conv = [a.data_ptr() if hasattr(a, "data_ptr") else a for a in args]
        _lib.call(name, ctypes.byref(self.batch), *conv, stream)


def shard(items: list, rank: int, world: int) -> list:
    """Contiguous block of `items` owned by `rank` (sizes differ by at most one)."""
    n = len(items)
    lo = (n * rank) // world
    hi = (n * (rank + 1)) // world
    return items[lo:hi]


def gather(local: list) -> list:
    """Every rank's ``local`` list concatenated in rank order, on every rank.

    The instances are independent, so the only exchange is this host-side gather of the small
    per-instance outputs (coefficients, norms); with one process it returns ``local``.
    """
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(local)
    parts: list = [None] * dist.get_world_size()
    dist.all_gather_object(parts, list(local))
    return [x for part in parts for x in part]


def max_over_ranks(seconds: float) -> float:
    """The slowest rank's time (a job's time is the last rank's), on every rank."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return seconds
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([seconds], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
