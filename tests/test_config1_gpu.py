"""Parity at the headline correctness case itself, against the reference.

The contraction C(a,b,c,d) += A(e,f,a,c) * B(f,b,d,e) with all six extents 64
(NIm = NJn = NPk = 4096), column-major operands whose entries are i.i.d.
U[-1, 1] drawn from one seed-0 stream (A first, then B), C = 0, alpha =
beta = 1.  Every GPU result -- the reference-named drop-in symbols
tblis_tensor_mult, stra_tblis_tensor_mult and stra_tblis_tensor_mult_2level at
impl 1/2/3, and the allocation-free entry point -- is compared over the WHOLE
of C with the reference library's own L=0 contraction of the same inputs
(tblis_tensor_mult compiled from the reference sources, run on the host
cores), the check test_strassen makes (test/test_strassen.cxx:245-276, which
always computes C_ref with the L=0 mult), within the FP64 bound

    max|C - Cref| <= 4 * 12^L * NPk * 2^-53 * max|A| * max|B|.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

E = 64
IA, IB, IC = "efac", "fbde", "abcd"


@pytest.fixture(scope="module")
def config1(tsb, cuda):
    import torch
    if not oracle.ref_available():
        pytest.skip("the reference library (oracle/_ref) is not built on this machine")
    A, B = oracle.uniform_pair((E,) * 4, (E,) * 4, seed=0)
    Cref = np.zeros((E,) * 4, order="F")
    import os
    oracle.ref_set_threads(os.cpu_count() or 1)
    oracle.ref_mult(0, 1, 1.0, A, IA, B, IB, 1.0, Cref, IC)

    def dev(x):
        t = torch.empty_strided(x.shape, [s // 8 for s in x.strides], dtype=torch.float64, device=cuda)
        t.copy_(torch.from_numpy(x))
        return t

    return dict(A=A, B=B, Cref=Cref, dA=dev(A), dB=dev(B), dev=dev,
                maxA=float(np.abs(A).max()), maxB=float(np.abs(B).max()))


def _check(c, C, level):
    bound = oracle.error_bound(level, E * E, c["maxA"], c["maxB"])
    err = float(np.abs(C - c["Cref"]).max())
    assert err <= bound, (level, err, bound)
    return err


@pytest.mark.parametrize("level,impl", [(0, 1), (1, 1), (1, 2), (1, 3), (2, 1), (2, 2), (2, 3)])
def test_config1_drop_in_vs_reference_L0(tsb, cuda, config1, level, impl):
    import torch
    c = config1
    C = c["dev"](np.zeros((E,) * 4, order="F"))
    tsb.set_impl(impl)
    try:
        tsb.contract(level, 1.0, c["dA"], IA, c["dB"], IB, 1.0, C, IC, drop_in=True)
    finally:
        tsb.set_impl(1)
    torch.cuda.synchronize()
    _check(c, C.cpu().numpy(), level)


@pytest.mark.parametrize("level", [1, 2])
def test_config1_fused_no_workspace_vs_reference_L0(tsb, cuda, config1, level):
    """The ABC kernel that forms the operand sums inside the GEMM (no packed
    workspace), on the same inputs."""
    import torch
    c = config1
    C = c["dev"](np.zeros((E,) * 4, order="F"))
    tsb.set_workspace_limit(0)
    try:
        tsb.contract(level, 1.0, c["dA"], IA, c["dB"], IB, 1.0, C, IC)
    finally:
        tsb.set_workspace_limit(None)
    torch.cuda.synchronize()
    _check(c, C.cpu().numpy(), level)


def test_config1_host_operands_vs_reference_L0(tsb, cuda, config1):
    """The drop-in call on host (numpy) operands: staged through device memory
    and copied back inside the call."""
    c = config1
    C = np.zeros((E,) * 4, order="F")
    tsb.contract(1, 1.0, c["A"], IA, c["B"], IB, 1.0, C, IC, drop_in=True)
    _check(c, C, 1)
