"""PyTorch autograd for the residual and the wall forces of packed instances.

``residual(U, X, V, mach, instances)`` and ``forces(U, X, instances)`` return R(Ma, U, X, V)
(``eb_compute_odes``) and F(U, X) (``eb_compute_forces``) as differentiable float64 tensors in the
packed layouts of ``InstanceSet`` (reference layouts per instance, back to back). The
residual's backward pass is the matrix-free adjoint kernel (``eb_apply_odes_adjoint``): d/dU,
d/dX, d/dV and d/dMa of <w, R> in one reverse pass over the faces that recomputes the face
quantities from the saved U, X, V and gathers every output element without atomics (the
reference's counterparts are the stored-Jacobian reverse products, core.py:375-510 and
294-346). The forces' backward pass uses the wall-force Jacobians and their reverse products
(``eb_apply_forces_wrt_*_rev``, core.py:637-716), rebuilt inside it from the saved inputs.
Only the gradients of inputs that require them are formed. ``mach`` is a CPU float64 tensor
with one Mach number per instance; its gradient is the per-instance d<w, R>/dMa.
"""

from __future__ import annotations

import torch

from .batch import InstanceSet


def _complex(x: torch.Tensor) -> torch.Tensor:
    """Real float64 vector -> interleaved complex vector with zero imaginary part."""
    out = torch.zeros(2 * x.numel(), dtype=torch.float64, device=x.device)
    out[0::2] = x.reshape(-1)
    return out


def _empty(n: int, device) -> torch.Tensor:
    return torch.empty(n, dtype=torch.float64, device=device)


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class _Residual(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U, X, V, mach, inst: InstanceSet):
        inst.set_mach(mach)
        R = _empty(4 * inst.n_cells, U.device)
        inst.call("eb_compute_odes", X, V, U, R, stream=_stream())
        ctx.save_for_backward(U, X, V)
        ctx.inst = inst
        return R

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, gR):
        U, X, V = ctx.saved_tensors
        inst: InstanceSet = ctx.inst
        dev, nc, nv, st = U.device, inst.n_cells, inst.n_verts, _stream()
        need = ctx.needs_input_grad
        out = [_empty(n, dev) if need[k] else None
               for k, n in enumerate((4 * nc, 2 * nv, 2 * nv, len(inst)))]
        if any(o is not None for o in out):
            inst.call("eb_apply_odes_adjoint", X, V, U, gR.contiguous(), 0, *out, stream=st)
        grads = [*out, None]
        if grads[3] is not None:
            grads[3] = grads[3].to("cpu")
        return tuple(grads)


class _Forces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U, X, inst: InstanceSet):
        F = _empty(2 * inst.n_wall, U.device)
        inst.call("eb_compute_forces", X, U, F, None, stream=_stream())
        ctx.save_for_backward(U, X)
        ctx.inst = inst
        return F

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, gF):
        U, X = ctx.saved_tensors
        inst: InstanceSet = ctx.inst
        dev, st = U.device, _stream()
        w = _complex(gF.contiguous())
        grads = [None, None, None]
        if ctx.needs_input_grad[0]:
            J = _empty(8 * inst.n_wall, dev)
            inst.call("eb_compute_forces_wrt_states", X, U, J, stream=st)
            y = _empty(8 * inst.n_cells, dev)
            inst.call("eb_apply_forces_wrt_states_rev", J, w, y, stream=st)
            grads[0] = y[0::2].contiguous()
        if ctx.needs_input_grad[1]:
            J = _empty(8 * inst.n_wall, dev)
            inst.call("eb_compute_forces_wrt_vertices", X, U, J, stream=st)
            y = _empty(4 * inst.n_verts, dev)
            inst.call("eb_apply_forces_wrt_vertices_rev", J, w, y, stream=st)
            grads[1] = y[0::2].contiguous()
        return tuple(grads)


def residual(U: torch.Tensor, X: torch.Tensor, V: torch.Tensor, mach: torch.Tensor,
             instances: InstanceSet) -> torch.Tensor:
    """Differentiable packed residual R(Ma, U, X, V) (float64 device tensors, CPU ``mach``)."""
    return _Residual.apply(U, X, V, mach, instances)


def forces(U: torch.Tensor, X: torch.Tensor, instances: InstanceSet) -> torch.Tensor:
    """Differentiable packed wall forces F(U, X)."""
    return _Forces.apply(U, X, instances)
