"""torch.autograd wrapper of the engine's multi-RHS product Y = A(v) X and its hand-written
adjoint (gs_spmm / gs_spmm_adjoint).

The sparsity structure is fixed when the operator is built; the values v (CSR order) and the
right-hand sides X are differentiable inputs:

    op = SparseOperator(row, col, v0, ncols, vtype="f32")
    Y = spmm(v, X, op)              # v: [nnz] in CSR order, X: [ncols, k]
    loss.backward()                 # v.grad = vbar, X.grad = A^T Ybar

Values may also live in the operator's "slots" order (op.slot_values(); the adjoint
layout's slot order, padding slots included and kept at zero gradient): there the
deterministic adjoint writes vbar in place instead of scattering it to CSR order, which is
the fast layout for training the values.

No kernel here is PyTorch's: the forward runs the K1 multi-RHS kernel and the backward the
transposed-K1 kernel (or the atomic one), both in libgpuspmv_b200.so.
"""
from __future__ import annotations

import torch

from . import engine as E


class SparseOperator:
    """A K1 matrix prepared for products and adjoints (values replaceable per call)."""

    def __init__(self, row, col, val, ncols=None, vtype="f64", device="cuda", stream=None):
        self.mat = E.Matrix(row, col, val, ncols=ncols, fmt="K1", vtype=vtype, device=device,
                            stream=stream, adjoint=True)
        self.nrows, self.ncols, self.nnz = self.mat.nrows, self.mat.ncols, self.mat.nnz
        self.dtype = E.TORCH_DTYPES[self.mat.vtype]

    def ensure_values(self, values: torch.Tensor, order: str = "csr"):
        """Store `values` unless they are already the stored ones (same tensor, same version)."""
        key = (values.data_ptr(), values._version, order)
        if self.mat._values_key != key:
            self.mat.set_values(values, order)
            self.mat._values_key = key

    def slot_values(self, values_csr: torch.Tensor) -> torch.Tensor:
        """CSR-order values -> a new tensor in the operator's slot order."""
        return self.mat.convert_values(values_csr, to="slots")

    def csr_values(self, values_slots: torch.Tensor) -> torch.Tensor:
        """Slot-order values (or their gradient) -> CSR order."""
        return self.mat.convert_values(values_slots, to="csr")

    def close(self):
        self.mat.close()


class _SpMM(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, X, op: SparseOperator, mode: str, order: str):
        v = values.detach()
        op.ensure_values(v, order)
        Xd = X.detach().contiguous()
        ctx.save_for_backward(v, Xd)
        ctx.op, ctx.mode, ctx.order = op, mode, order
        return op.mat.spmm(Xd)

    @staticmethod
    def backward(ctx, Ybar):
        v, X = ctx.saved_tensors
        op = ctx.op
        op.ensure_values(v, ctx.order)  # the operator may have seen other values since
        want_v = ctx.needs_input_grad[0]
        Xbar, vbar = op.mat.adjoint(Ybar.contiguous(), X if want_v else None, mode=ctx.mode,
                                    want_vbar=want_v, order=ctx.order)
        return ((vbar if ctx.needs_input_grad[0] else None),
                (Xbar if ctx.needs_input_grad[1] else None), None, None, None)


def spmm(values: torch.Tensor, X: torch.Tensor, op: SparseOperator,
         mode: str = "deterministic", order: str = "csr") -> torch.Tensor:
    """Y = A(values) X with gradients for values and X.  mode: "deterministic" (transposed
    layout, bit-reproducible) or "atomic" (atomic adds into X's gradient); order: "csr"
    (values in the CSR order of the structure) or "slots" (op.slot_values order)."""
    return _SpMM.apply(values, X, op, mode, order)
