"""Differentiable tensor contraction over the library's C ABI (test binding).

``contract(A, idx_A, B, idx_B, idx_C, level=1)`` returns
``C(idx_C) = sum A(idx_A) * B(idx_B)`` and supports ``backward``.  The adjoints
are contractions themselves, run through the same entry points and kernels as
the forward pass (the reference computes every contraction through
``tblis_tensor_mult`` / ``stra_tblis_tensor_mult``; it has no autograd):

    dA(idx_A) = sum over the labels not in idx_A of dC(idx_C) * B(idx_B)
    dB(idx_B) = sum over the labels not in idx_B of A(idx_A) * dC(idx_C)

Labels only in A (summed in the forward pass) become broadcast labels of dA;
labels only in C need ``out_sizes``.  Nothing is checkpointed: the ABC
variant keeps no workspace between calls, and the backward pass only needs
the saved inputs.
"""
from __future__ import annotations

import torch

from . import tblis_stra as _t


def _extents(idx_A, A, idx_B, B, out_sizes):
    ext = dict(out_sizes or {})
    for idx, X in ((idx_A, A), (idx_B, B)):
        for c, n in zip(idx, X.shape):
            if c in ext and ext[c] != n:
                raise ValueError(f"label {c!r} has extents {ext[c]} and {n}")
            ext[c] = n
    return ext


class _Contract(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A, B, idx_A, idx_B, idx_C, level, impl, out_sizes):
        ext = _extents(idx_A, A, idx_B, B, out_sizes)
        missing = [c for c in idx_C if c not in ext]
        if missing:
            raise ValueError(f"extents of output-only labels {missing} must be given in out_sizes")
        C = torch.zeros([ext[c] for c in idx_C], dtype=A.dtype, device=A.device)
        _t.contract(level, 1.0, A, idx_A, B, idx_B, 0.0, C, idx_C, impl=impl,
                    stream=torch.cuda.current_stream(A.device) if A.is_cuda else None)
        ctx.save_for_backward(A, B)
        ctx.meta = (idx_A, idx_B, idx_C, level, impl)
        return C

    @staticmethod
    def backward(ctx, dC):
        A, B = ctx.saved_tensors
        idx_A, idx_B, idx_C, level, impl = ctx.meta
        stream = torch.cuda.current_stream(dC.device) if dC.is_cuda else None
        dA = dB = None
        if ctx.needs_input_grad[0]:
            dA = torch.zeros_like(A, memory_format=torch.contiguous_format)
            _t.contract(level, 1.0, dC, idx_C, B, idx_B, 0.0, dA, idx_A, impl=impl, stream=stream)
        if ctx.needs_input_grad[1]:
            dB = torch.zeros_like(B, memory_format=torch.contiguous_format)
            _t.contract(level, 1.0, A, idx_A, dC, idx_C, 0.0, dB, idx_B, impl=impl, stream=stream)
        return dA, dB, None, None, None, None, None, None


def contract(A: torch.Tensor, idx_A: str, B: torch.Tensor, idx_B: str, idx_C: str,
             level: int = 1, impl: int = 1, out_sizes: dict | None = None) -> torch.Tensor:
    """Differentiable C(idx_C) = sum A(idx_A) B(idx_B) at Strassen level `level`."""
    return _Contract.apply(A, B, idx_A, idx_B, idx_C, level, impl, out_sizes)
