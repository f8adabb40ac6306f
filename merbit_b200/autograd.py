"""Differentiable sparse products: Y = A(vals) @ X with gradients for vals
and X, running on the C ABI's kernels.

Backward:
  dX    = A^T G     merge-path SpMM on the transpose plan
                    (merbit_plan_transpose: stable column sort, so every sum
                    is taken in a fixed order -- no float atomics)
  dvals = G[row] . X[col]   per nonzero
When both are needed they come from one launch (merbit_spmm_dval: the
transpose SpMM forms each dval from the G row it gathers); otherwise, or for
shapes that launch does not take, merbit_spmm and merbit_dval run apart.
"""
from __future__ import annotations

import torch

from . import Plan, _check, _dptr, _P, _stream_ptr, lib


class SparseMatrix:
    """A CSR matrix on one GPU whose values can carry gradients.

    row_ptr, col_idx: int32 CUDA tensors (structure, fixed); vals: float64,
    float32 or bfloat16 CUDA tensor (may be replaced or modified between
    products).  ``matmul(X)`` / ``A @ X`` differentiate with respect to the
    values passed and to X.
    """

    def __init__(self, row_ptr: torch.Tensor, col_idx: torch.Tensor, vals: torch.Tensor,
                 ncol: int | None = None):
        self.plan = Plan(row_ptr, col_idx, vals, ncol=ncol)
        self.vals = vals
        self._tplan = None
        self._tkey = None
        self.shape = (self.plan.nrow, self.plan.ncol)

    # -- plumbing ---------------------------------------------------------
    def _bind(self, vals: torch.Tensor) -> None:
        if vals.data_ptr() != self.plan.vals.data_ptr():
            self.plan.set_values(vals)
        self.vals = vals

    def transpose_plan(self, vals: torch.Tensor | None = None) -> Plan:
        """The plan of A^T, with values refreshed when A's changed."""
        vals = self.vals if vals is None else vals
        self._bind(vals)
        key = (vals.data_ptr(), vals._version)
        if self._tplan is None:
            h = _P()
            _check(lib().merbit_plan_transpose(self.plan._h, C_byref(h), _stream_ptr(None)))
            self._tplan = _TransposePlan(h, self.plan)
        elif key != self._tkey:
            _check(lib().merbit_plan_transpose_refresh(self._tplan._h, _dptr(vals),
                                                       _stream_ptr(None)))
        self._tkey = key
        return self._tplan

    def dval(self, G: torch.Tensor, X: torch.Tensor) -> torch.Tensor:
        """dval[e] = G[row_e] . X[col_e] (the gradient of <G, A X> in vals)."""
        k = X.shape[1]
        out = torch.empty(self.plan.nnz, dtype=self.plan.xy_dtype, device=self.plan.device)
        _check(lib().merbit_dval(self.plan._h, k, _dptr(G), G.stride(0) if G.shape[0] > 1 else k,
                                 _dptr(X), X.stride(0) if X.shape[0] > 1 else k, _dptr(out),
                                 _stream_ptr(None)))
        return out

    def backward_fused(self, G: torch.Tensor, X: torch.Tensor, vals: torch.Tensor | None = None):
        """(dX, dval) of Y = A X from one launch on the transpose plan, or
        None when that launch does not take these operands."""
        k = X.shape[1]
        if self.plan.dtype == 2 or k not in (1, 2, 4, 8, 16, 32):
            return None
        T = self.transpose_plan(vals)
        dX = torch.empty(self.plan.ncol, k, dtype=self.plan.xy_dtype, device=self.plan.device)
        dval = torch.empty(self.plan.nnz, dtype=self.plan.xy_dtype, device=self.plan.device)
        ldg = G.stride(0) if G.shape[0] > 1 else k
        ldx = X.stride(0) if X.shape[0] > 1 else k
        st = lib().merbit_spmm_dval(T._h, k, _dptr(G), ldg, _dptr(X), ldx, _dptr(dX), k,
                                    _dptr(dval), _stream_ptr(None))
        if st == 6:  # MERBIT_ERR_UNSUPPORTED
            return None
        _check(st)
        return dX, dval

    # -- user API -----------------------------------------------------------
    def matmul(self, X: torch.Tensor, vals: torch.Tensor | None = None) -> torch.Tensor:
        vals = self.vals if vals is None else vals
        return _SpMM.apply(vals, X, self)

    def __matmul__(self, X: torch.Tensor) -> torch.Tensor:
        return self.matmul(X)


def C_byref(h):
    import ctypes

    return ctypes.byref(h)


class _TransposePlan(Plan):
    """A Plan wrapping a handle made by merbit_plan_transpose (it owns its
    arrays; the source plan's tensors stay referenced for safety)."""

    def __init__(self, handle, src: Plan):  # noqa: D401 - no Plan.__init__
        self._h = handle
        self._keep = [src]
        self.dtype = src.dtype
        self.xy_dtype = src.xy_dtype
        self.nrow, self.ncol, self.nnz = src.ncol, src.nrow, src.nnz
        self.device = src.device
        self.vals = None


class _SpMM(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, X, mat: SparseMatrix):
        vec = X.dim() == 1
        X2 = (X.unsqueeze(1) if vec else X).contiguous()
        mat._bind(vals)
        Y = mat.plan.spmm(X2)
        ctx.save_for_backward(vals, X2)
        ctx.mat = mat
        ctx.vec = vec
        return Y.squeeze(1) if vec else Y

    @staticmethod
    def backward(ctx, G):
        vals, X2 = ctx.saved_tensors
        mat: SparseMatrix = ctx.mat
        G2 = (G.unsqueeze(1) if ctx.vec else G).contiguous()
        dvals = dX = None
        if ctx.needs_input_grad[0] and ctx.needs_input_grad[1]:
            fused = mat.backward_fused(G2, X2, vals)
            if fused is not None:
                dX, dv = fused
                return dv.to(vals.dtype), (dX.squeeze(1) if ctx.vec else dX), None
        if ctx.needs_input_grad[1]:
            dX = mat.transpose_plan(vals).spmm(G2)
            if ctx.vec:
                dX = dX.squeeze(1)
        if ctx.needs_input_grad[0]:
            mat._bind(vals)
            dvals = mat.dval(G2, X2).to(vals.dtype)
        return dvals, dX, None


def spmm(row_ptr: torch.Tensor, col_idx: torch.Tensor, vals: torch.Tensor, X: torch.Tensor,
         ncol: int | None = None) -> torch.Tensor:
    """One-shot differentiable Y = A(vals) @ X (builds the plan each call;
    keep a SparseMatrix to reuse it)."""
    return SparseMatrix(row_ptr, col_idx, vals, ncol=ncol).matmul(X)
