"""Differentiable dual contouring: the extracted vertices as a function of the grid values.

The forward pass is the ordinary extraction (``dcb_extract_device``); the backward pass is the
hand-written adjoint ``dcb_backward``, which differentiates every vertex through its FP64 QEF
solve with the topology held fixed (active cells, Hermite edges and the rank of each solve).
Faces are integer outputs and carry no gradient. The reference's backends are forward-only;
this sits beside the reference-shaped API of ``backend.py``.
"""
import torch

from .backend import B200DualContouringBackend, DenseSdfGridDevice


class DualContourFunction(torch.autograd.Function):
    """``V, F = DualContourFunction.apply(values, backend, dims, spacing, origin)``."""

    @staticmethod
    def forward(ctx, values, backend, dims, spacing, origin):
        vals = values.detach().contiguous()
        V, F, _ = backend.extract_tensor(vals, dims, spacing, origin)
        ctx.backend = backend
        ctx.grid = (tuple(dims), tuple(spacing), tuple(origin))
        ctx.generation = backend._generation
        ctx.save_for_backward(vals)
        ctx.mark_non_differentiable(F)
        return V, F

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, grad_V, grad_F):
        (vals,) = ctx.saved_tensors
        be = ctx.backend
        dims, spacing, origin = ctx.grid
        if grad_V is None:
            return None, None, None, None, None
        if be._generation != ctx.generation:
            # another extraction ran on this backend since: rebuild this one's cell list
            be.extract_tensor_ptr(DenseSdfGridDevice(*dims, *spacing, *origin, d_values=vals))
        dgrid = be.backward_tensor(vals, dims, spacing, origin, grad_V)
        return dgrid.view(vals.shape), None, None, None, None


_default_backends = {}


def dual_contour(values, dims, spacing, origin, backend=None):
    """Differentiable extraction of a CUDA float32 grid (nx*ny*nz values, x fastest):
    returns ``(V (nv,3) float32, F (nf,4 or 3) int32)``; ``V`` carries the gradient back to
    ``values``."""
    if backend is None:
        dev = values.device.index if values.device.index is not None else torch.cuda.current_device()
        backend = _default_backends.get(dev)
        if backend is None:
            backend = _default_backends[dev] = B200DualContouringBackend(dev)
    return DualContourFunction.apply(values, backend, dims, spacing, origin)
