"""Streaming residual evaluation of host-resident inputs (serving many steps through the GPU).

``ResidualPipeline`` evaluates R(Ma, U, X, V) for a packed ``InstanceSet`` step after step with
inputs and outputs in pinned host memory. Each step's host-to-device copies, its residual
launch and its device-to-host copy run on three streams over ``depth`` device buffer sets, so
in steady state the copy of step k+1's inputs, the residual of step k and the copy of step
k-1's result proceed at the same time (the two copy directions use separate copy engines).
A step costs the slowest of the three instead of their sum.
"""

from __future__ import annotations

from .batch import InstanceSet


class ResidualPipeline:
    def __init__(self, instances: InstanceSet, depth: int = 2) -> None:
        import torch

        self._torch = torch
        self.inst = instances
        self.depth = max(2, int(depth))
        f64 = dict(dtype=torch.float64, device="cuda")
        nv, nc = 2 * instances.n_verts, 4 * instances.n_cells
        self.bufs = [dict(X=torch.empty(nv, **f64), V=torch.empty(nv, **f64),
                          U=torch.empty(nc, **f64), R=torch.empty(nc, **f64))
                     for _ in range(self.depth)]
        self.s_in, self.s_run, self.s_out = (torch.cuda.Stream() for _ in range(3))
        self.copied = [torch.cuda.Event() for _ in range(self.depth)]   # inputs on the device
        self.computed = [torch.cuda.Event() for _ in range(self.depth)]  # R on the device
        self.drained = [torch.cuda.Event() for _ in range(self.depth)]   # R back on the host
        self.k = 0

    def submit(self, hX, hV, hU, hR) -> None:
        """Queues one step: inputs from pinned host tensors hX, hV, hU (packed vertices,
        velocities and states), the residual into pinned host tensor hR. Returns at once; the
        host tensors must stay unchanged (hR unread) until ``synchronize``."""
        torch = self._torch
        i = self.k % self.depth
        b = self.bufs[i]
        if self.k >= self.depth:  # buffer i is reused: its previous result must be copied out
            self.s_in.wait_event(self.drained[i])
        with torch.cuda.stream(self.s_in):
            b["X"].copy_(hX, non_blocking=True)
            b["V"].copy_(hV, non_blocking=True)
            b["U"].copy_(hU, non_blocking=True)
            self.copied[i].record(self.s_in)
        self.s_run.wait_event(self.copied[i])
        self.inst.call("eb_compute_odes", b["X"], b["V"], b["U"], b["R"],
                       stream=self.s_run.cuda_stream)
        self.computed[i].record(self.s_run)
        self.s_out.wait_event(self.computed[i])
        with torch.cuda.stream(self.s_out):
            hR.copy_(b["R"], non_blocking=True)
            self.drained[i].record(self.s_out)
        self.k += 1

    def synchronize(self) -> None:
        for s in (self.s_in, self.s_run, self.s_out):
            s.synchronize()
