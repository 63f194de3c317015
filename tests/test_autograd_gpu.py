"""Differentiation form: forward plus adjoint contractions through the library,
behind torch.autograd.

Checks, in FP64:
  * small contractions (batch, A-only, C-only, diagonal labels) against torch
    autograd on torch.einsum;
  * the two-contraction chain C(a,b,i,j) = sum_{e,f} A(a,b,e,f) B(e,f,i,j),
    D(a,b,k,l) = sum_{i,j} C E(i,j,k,l), loss = sum D*W with a,b,e,f = 128 and
    i,j,k,l = 48, at L = 0 and 1: sampled gradient entries against FP64 central
    differences (h = 1e-6; the loss is linear in each input, so the difference
    quotient is exact up to rounding), and whole gradients against adjoints
    formed by the reference's own L = 0 contraction when it is built here.
"""
import importlib
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ag(tsb):
    return importlib.import_module("tblis_strassen_b200.autograd")


SMALL = [
    ("abcd", "efac", "fbde", dict(a=6, b=5, c=4, d=7, e=3, f=8), None),
    ("abz", "akz", "kbz", dict(a=9, b=7, k=11, z=3), None),
    ("abw", "akx", "kb", dict(a=5, b=6, k=7, x=3, w=4), {"w": 4}),
    ("ab", "aak", "kb", dict(a=5, b=4, k=6), None),
]


@pytest.mark.parametrize("ic,ia,ib,ext,out", SMALL, ids=[c[0] + "=" + c[1] + "*" + c[2] for c in SMALL])
@pytest.mark.parametrize("level", [0, 1, 2])
def test_small_vs_torch_einsum(ag, cuda, ic, ia, ib, ext, out, level):
    import torch
    g = torch.Generator(device=cuda).manual_seed(3)
    A = (torch.rand([ext[c] for c in ia], dtype=torch.float64, device=cuda, generator=g) * 2 - 1).requires_grad_()
    B = (torch.rand([ext[c] for c in ib], dtype=torch.float64, device=cuda, generator=g) * 2 - 1).requires_grad_()
    W = torch.rand([ext[c] for c in ic], dtype=torch.float64, device=cuda, generator=g) * 2 - 1
    C = ag.contract(A, ia, B, ib, ic, level=level, out_sizes=out)
    (C * W).sum().backward()
    gA, gB = A.grad.clone(), B.grad.clone()
    A.grad = None
    B.grad = None

    # torch reference: einsum cannot repeat a label in one operand as a
    # diagonal input, so build the diagonal explicitly
    def ref_forward(A, B):
        if ia == "aak":
            Ad = torch.diagonal(A, dim1=0, dim2=1).permute(1, 0)  # (a, k)
            return torch.einsum("ak,kb->ab", Ad, B)
        if ic == "abw":
            return torch.einsum("akx,kb->ab", A, B)[:, :, None].expand(-1, -1, out["w"])
        return torch.einsum(f"{ia},{ib}->{ic}", A, B)

    (ref_forward(A, B) * W).sum().backward()
    tol = 1e-11
    assert torch.allclose(C, ref_forward(A, B), atol=tol, rtol=0)
    assert torch.allclose(gA, A.grad, atol=tol, rtol=0)
    assert torch.allclose(gB, B.grad, atol=tol, rtol=0)


def _chain(ag, A, B, E, W, level):
    C = ag.contract(A, "abef", B, "efij", "abij", level=level)
    D = ag.contract(C, "abij", E, "ijkl", "abkl", level=level)
    return (D * W).sum()


@pytest.mark.parametrize("level", [0, 1])
def test_two_contraction_chain_central_differences(ag, cuda, level):
    import torch
    g = torch.Generator(device=cuda).manual_seed(11)
    n, m = 128, 48
    A = (torch.rand((n, n, n, n), dtype=torch.float64, device=cuda, generator=g) * 2 - 1).requires_grad_()
    B = (torch.rand((n, n, m, m), dtype=torch.float64, device=cuda, generator=g) * 2 - 1).requires_grad_()
    E = (torch.rand((m, m, m, m), dtype=torch.float64, device=cuda, generator=g) * 2 - 1).requires_grad_()
    W = torch.rand((n, n, m, m), dtype=torch.float64, device=cuda, generator=g) * 2 - 1
    loss = _chain(ag, A, B, E, W, level)
    loss.backward()
    rng = np.random.default_rng(level)
    h = 1e-6
    with torch.no_grad():
        for X in (A, B, E):
            grad = X.grad
            scale = float(grad.abs().max())
            for _ in range(6):
                idx = tuple(int(rng.integers(0, s)) for s in X.shape)
                old = float(X[idx])
                X[idx] = old + h
                lp = float(_chain(ag, A, B, E, W, level))
                X[idx] = old - h
                lm = float(_chain(ag, A, B, E, W, level))
                X[idx] = old
                fd = (lp - lm) / (2 * h)
                # rounding of the loss (~1e-16 * |loss| * sqrt(terms)) over 2h
                assert abs(fd - float(grad[idx])) <= 1e-5 * scale + 1e-3, (X.shape, idx, fd, float(grad[idx]))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_chain_adjoints_vs_reference_L0(ag, cuda):
    """Whole gradients of the chain at L=1 against adjoint contractions formed
    by the reference's L=0 tblis_tensor_mult (same inputs, FP64), at
    a,b,e,f = 64 so the CPU side stays within seconds."""
    import torch
    g = torch.Generator(device=cuda).manual_seed(5)
    n, m = 64, 48
    A = (torch.rand((n, n, n, n), dtype=torch.float64, device=cuda, generator=g) * 2 - 1).requires_grad_()
    B = (torch.rand((n, n, m, m), dtype=torch.float64, device=cuda, generator=g) * 2 - 1).requires_grad_()
    E = (torch.rand((m, m, m, m), dtype=torch.float64, device=cuda, generator=g) * 2 - 1).requires_grad_()
    W = torch.rand((n, n, m, m), dtype=torch.float64, device=cuda, generator=g) * 2 - 1
    _chain(ag, A, B, E, W, 1).backward()

    An, Bn, En, Wn = (np.ascontiguousarray(X.detach().cpu().numpy()) for X in (A, B, E, W))
    oracle.ref_set_threads(os.cpu_count() or 1)
    C = np.zeros((n, n, m, m))
    oracle.ref_mult(0, 1, 1.0, An, "abef", Bn, "efij", 0.0, C, "abij")
    G = np.zeros((n, n, m, m))          # dL/dC = sum_kl W(a,b,k,l) E(i,j,k,l)
    oracle.ref_mult(0, 1, 1.0, Wn, "abkl", En, "ijkl", 0.0, G, "abij")
    dA = np.zeros_like(An)
    oracle.ref_mult(0, 1, 1.0, G, "abij", Bn, "efij", 0.0, dA, "abef")
    dB = np.zeros_like(Bn)
    oracle.ref_mult(0, 1, 1.0, An, "abef", G, "abij", 0.0, dB, "efij")
    dE = np.zeros_like(En)
    oracle.ref_mult(0, 1, 1.0, C, "abij", Wn, "abkl", 0.0, dE, "ijkl")
    # bound: two chained contractions at L=1; sums of 48*48 and 64*64 terms
    for got, ref, k in ((A.grad, dA, m * m), (B.grad, dB, n * n), (E.grad, dE, n * n)):
        got = got.cpu().numpy()
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 4 * 12 * (n * n + m * m) * 2.0 ** -53 * scale * 10, (k,)


# ---- the split-BF16 form (FP32 tensors on the tcgen05 path) -------------------

def _chain64(tsb, A, B, E, W):
    """The chain's loss in FP64 on the given values (the library's FP64 L=0
    contractions): the function the FP32 gradients are differences of."""
    import torch
    A, B, E, W = (X.double() for X in (A, B, E, W))
    C = torch.zeros((A.shape[0], A.shape[1], B.shape[2], B.shape[3]), dtype=torch.float64, device=A.device)
    tsb.contract(0, 1.0, A, "abef", B, "efij", 0.0, C, "abij")
    D = torch.zeros((A.shape[0], A.shape[1], E.shape[2], E.shape[3]), dtype=torch.float64, device=A.device)
    tsb.contract(0, 1.0, C, "abij", E, "ijkl", 0.0, D, "abkl")
    return float((D * W).sum())


@pytest.mark.parametrize("level", [0, 1])
def test_split_bf16_chain_central_differences(tsb, ag, cuda, level):
    """FP32 chain (a,b,e,f = 128, i,j,k,l = 48) on the split-BF16 path at L=0
    and L=1: sampled gradient entries against FP64 central differences
    (h = 1e-6) of the same loss evaluated in FP64 on the FP32 values."""
    import torch
    g = torch.Generator(device=cuda).manual_seed(21)
    n, m = 128, 48
    A = (torch.rand((n, n, n, n), dtype=torch.float32, device=cuda, generator=g) * 2 - 1).requires_grad_()
    B = (torch.rand((n, n, m, m), dtype=torch.float32, device=cuda, generator=g) * 2 - 1).requires_grad_()
    E = (torch.rand((m, m, m, m), dtype=torch.float32, device=cuda, generator=g) * 2 - 1).requires_grad_()
    W = torch.rand((n, n, m, m), dtype=torch.float32, device=cuda, generator=g) * 2 - 1
    _chain(ag, A, B, E, W, level).backward()
    rng = np.random.default_rng(10 + level)
    h = 1e-6
    with torch.no_grad():
        A64, B64, E64 = A.double(), B.double(), E.double()
        for X, X64 in ((A, A64), (B, B64), (E, E64)):
            grad = X.grad
            scale = float(grad.abs().max())
            for _ in range(4):
                idx = tuple(int(rng.integers(0, s)) for s in X.shape)
                old = float(X64[idx])
                X64[idx] = old + h
                lp = _chain64(tsb, A64, B64, E64, W)
                X64[idx] = old - h
                lm = _chain64(tsb, A64, B64, E64, W)
                X64[idx] = old
                fd = (lp - lm) / (2 * h)
                # split-BF16 (6 terms) is within ~1e-6 of FP32-exact per product;
                # the difference quotient carries the FP64 loss rounding over 2h
                assert abs(fd - float(grad[idx])) <= 2e-5 * scale + 1e-3, (X.shape, idx, fd, float(grad[idx]))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("level", [0, 1])
def test_split_bf16_chain_adjoints_vs_reference_L0(tsb, ag, cuda, level):
    """Whole FP32 gradients of the chain (split-BF16, L=0 and L=1) against the
    adjoint contractions formed in FP64 by the reference's L=0
    tblis_tensor_mult on the same FP32 values, normwise within 1e-5."""
    import torch
    g = torch.Generator(device=cuda).manual_seed(6)
    n, m = 64, 48
    A = (torch.rand((n, n, n, n), dtype=torch.float32, device=cuda, generator=g) * 2 - 1).requires_grad_()
    B = (torch.rand((n, n, m, m), dtype=torch.float32, device=cuda, generator=g) * 2 - 1).requires_grad_()
    E = (torch.rand((m, m, m, m), dtype=torch.float32, device=cuda, generator=g) * 2 - 1).requires_grad_()
    W = torch.rand((n, n, m, m), dtype=torch.float32, device=cuda, generator=g) * 2 - 1
    _chain(ag, A, B, E, W, level).backward()
    An, Bn, En, Wn = (np.ascontiguousarray(X.detach().double().cpu().numpy()) for X in (A, B, E, W))
    oracle.ref_set_threads(os.cpu_count() or 1)
    C = np.zeros((n, n, m, m))
    oracle.ref_mult(0, 1, 1.0, An, "abef", Bn, "efij", 0.0, C, "abij")
    G = np.zeros((n, n, m, m))
    oracle.ref_mult(0, 1, 1.0, Wn, "abkl", En, "ijkl", 0.0, G, "abij")
    dA = np.zeros_like(An)
    oracle.ref_mult(0, 1, 1.0, G, "abij", Bn, "efij", 0.0, dA, "abef")
    dB = np.zeros_like(Bn)
    oracle.ref_mult(0, 1, 1.0, An, "abef", G, "abij", 0.0, dB, "efij")
    dE = np.zeros_like(En)
    oracle.ref_mult(0, 1, 1.0, C, "abij", Wn, "abkl", 0.0, dE, "ijkl")
    for got, ref in ((A.grad, dA), (B.grad, dB), (E.grad, dE)):
        got = got.double().cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-5
