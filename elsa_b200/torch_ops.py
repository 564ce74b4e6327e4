"""torch autograd integration: projectors as differentiable layers.

``project(x, op)`` computes op(x) with the native forward kernel and back-propagates with the
native matched adjoint (the adjoint is the exact transpose of the forward, so gradients are exact
up to float rounding). ``x`` is a CUDA float32 tensor whose last dimension holds the volume
(x fastest); leading dimensions are a batch. ``op`` is an ``elsa_b200.Projector`` or a
``elsa_b200.pyelsa`` operator. With JosephsMethodCUDA's ``fast`` adjoint (not the transpose) the
gradients are only approximate; a warning says so once per operator.
"""
import warnings

import torch

__all__ = ["project", "backproject", "Projection"]


def _native(op):
    return getattr(op, "native", op)


def _run(op, inp, adjoint):
    op = _native(op)
    n_in = op.range_size if adjoint else op.domain_size
    n_out = op.domain_size if adjoint else op.range_size
    if inp.shape[-1] != n_in:
        raise ValueError("last dimension %d does not match the operator (%d)"
                         % (inp.shape[-1], n_in))
    if not inp.is_cuda or inp.dtype != torch.float32:
        raise TypeError("projector inputs are CUDA float32 tensors")
    flat = inp.contiguous().reshape(-1, n_in)
    out = torch.empty(flat.shape[0], n_out, dtype=torch.float32, device=inp.device)
    stream = torch.cuda.current_stream(inp.device).cuda_stream
    # the whole batch in one call (one launch per kernel for the 3D Joseph operator)
    if adjoint:
        op.apply_adjoint_batch_ptr(flat.data_ptr(), n_in, out.data_ptr(), n_out,
                                   flat.shape[0], stream)
    else:
        op.apply_batch_ptr(flat.data_ptr(), n_in, out.data_ptr(), n_out, flat.shape[0], stream)
    return out.reshape(*inp.shape[:-1], n_out)


class _Project(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, op, adjoint):
        ctx.op, ctx.adjoint = op, adjoint
        native = _native(op)
        if not getattr(native, "matched", True) and not getattr(native, "_warned", False):
            native._warned = True
            warnings.warn("this operator's adjoint is JosephsMethodCUDA's fast backprojection, "
                          "not the transpose of the forward: gradients are approximate",
                          RuntimeWarning, stacklevel=3)
        return _run(op, x, adjoint)

    @staticmethod
    def backward(ctx, grad):
        return _run(ctx.op, grad, not ctx.adjoint), None, None


def project(x, op):
    """A x, differentiable (backward applies A^T)."""
    return _Project.apply(x, op, False)


def backproject(y, op):
    """A^T y, differentiable (backward applies A)."""
    return _Project.apply(y, op, True)


class Projection(torch.nn.Module):
    """nn.Module wrapper of a projector (forward = A, or A^T with adjoint=True)."""

    def __init__(self, op, adjoint=False):
        super().__init__()
        self.op, self.adjoint = op, adjoint

    def forward(self, x):
        return backproject(x, self.op) if self.adjoint else project(x, self.op)
