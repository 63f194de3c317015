"""Failure detection on the GPU, in forms that fault, trap or hang nothing.

* Bounded waits: the warp-specialised kernels (packed FP64 GEMM, the fused
  no-workspace kernels in their gather and element-pair forms, split-BF16
  tcgen05 GEMM) bound every pipeline wait.  A test shortens the bound to one
  SM clock cycle (tblis_stra_set_wait_limit) and turns on the wait injection
  (tblis_stra_set_wait_injection), under which each pipeline wait behaves as
  a wait on a flag that nothing sets, so the first one runs out whatever the
  timing of the copies (at these sizes a copy has often landed before its
  wait starts); the kernel then stops issuing work, lets its own copies and
  MMAs land, frees its tensor memory and ends, and the blocking call reports
  TBLIS_STRA_ERR_TIMEOUT.  The next call with the default bound and no
  injection must succeed on the same context and match the oracle.
* Allocation failure: a per-thread ceiling on single device allocations
  (tblis_stra_set_alloc_limit) makes the library's own allocations fail as an
  out-of-memory device would; the call returns TBLIS_STRA_ERR_ALLOC and C is
  untouched.
"""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

ERR_ALLOC, ERR_TIMEOUT = 7, 11


def _dev(torch, x, dev):
    t = torch.empty_strided(x.shape, [s // x.itemsize for s in x.strides], dtype=torch.float64
                            if x.dtype == np.float64 else torch.float32, device=dev)
    t.copy_(torch.from_numpy(x))
    return t


def _problem(n=512, seed=40):
    A = oracle.uniform((n, n), seed)
    B = oracle.uniform((n, n), seed + 1)
    ref = np.zeros((n, n), order="F")
    oracle.contract(1.0, A, "ik", B, "kj", 0.0, ref, "ij")
    return A, B, ref


@pytest.mark.parametrize("level", [0, 1])
def test_wait_timeout_fp64_then_recovery(tsb, cuda, level):
    import torch
    A, B, ref = _problem()
    dA, dB = _dev(torch, A, cuda), _dev(torch, B, cuda)
    C = torch.zeros_like(dA)
    tsb.set_wait_limit(1)
    tsb.set_wait_injection(True)
    try:
        with pytest.raises(tsb.TblisStraError) as ei:
            tsb.contract(level, 1.0, dA, "ik", dB, "kj", 0.0, C, "ij", drop_in=True)
        assert ei.value.status == ERR_TIMEOUT
    finally:
        tsb.set_wait_limit(0)
        tsb.set_wait_injection(False)
    C.zero_()
    tsb.contract(level, 1.0, dA, "ik", dB, "kj", 0.0, C, "ij", drop_in=True)
    err = float(np.abs(C.cpu().numpy() - ref).max())
    assert err <= oracle.error_bound(level, 512, np.abs(A).max(), np.abs(B).max())


@pytest.mark.parametrize("level", [0, 1, 2])
def test_wait_timeout_fused_no_workspace_then_recovery(tsb, cuda, level):
    """The fused no-workspace kernel (raw-block copies at L <= 1, register
    sums at L = 2): a one-cycle bound, TBLIS_STRA_ERR_TIMEOUT, then a correct
    call on the same context."""
    import torch
    A, B, ref = _problem()
    dA, dB = _dev(torch, A, cuda), _dev(torch, B, cuda)
    C = torch.zeros_like(dA)
    tsb.set_workspace_limit(0)
    try:
        tsb.set_wait_limit(1)
        tsb.set_wait_injection(True)
        try:
            with pytest.raises(tsb.TblisStraError) as ei:
                tsb.contract(level, 1.0, dA, "ik", dB, "kj", 0.0, C, "ij", drop_in=True)
            assert ei.value.status == ERR_TIMEOUT
        finally:
            tsb.set_wait_limit(0)
            tsb.set_wait_injection(False)
        C.zero_()
        tsb.contract(level, 1.0, dA, "ik", dB, "kj", 0.0, C, "ij", drop_in=True)
    finally:
        tsb.set_workspace_limit(None)
    err = float(np.abs(C.cpu().numpy() - ref).max())
    assert err <= oracle.error_bound(level, 512, np.abs(A).max(), np.abs(B).max())


@pytest.mark.parametrize("level,producer", [(0, "tma"), (1, "tma"), (0, "pairs"), (1, "pairs"), (2, "pairs")])
def test_wait_timeout_pair_kernel_then_recovery(tsb, cuda, level, producer):
    """The element-pair form of the no-workspace kernel, with each of its
    producers and both slot shapes (16 k per slot at L <= 1, 8 k at L = 2):
    a one-cycle bound, TBLIS_STRA_ERR_TIMEOUT, then a correct call on the same
    context.  Tensor-map boxes: A(k, i), B(k, j) (128-byte runs); pair
    copies: the headline contraction's layout at 512^3."""
    import torch
    if producer == "tma":
        A, B, ref = _problem()
        hA, hB = np.asfortranarray(A.T), B            # A(k, i): k contiguous
        ia, ib, ic, shape_c, k, mA, mB = "ki", "kj", "ij", (512, 512), 512, np.abs(A).max(), np.abs(B).max()
    else:
        ext = dict(a=16, b=16, c=32, d=32, e=16, f=32)
        ia, ib, ic = "efac", "fbde", "abcd"
        hA = oracle.uniform([ext[c] for c in ia], 60)
        hB = oracle.uniform([ext[c] for c in ib], 61)
        shape_c = tuple(ext[c] for c in ic)
        ref = np.zeros(shape_c, order="F")
        oracle.contract(1.0, hA, ia, hB, ib, 0.0, ref, ic)
        k, mA, mB = 512, np.abs(hA).max(), np.abs(hB).max()
    dA, dB = _dev(torch, hA, cuda), _dev(torch, hB, cuda)
    C = _dev(torch, np.zeros(shape_c, order="F"), cuda)
    kind = "fused_tma" if producer == "tma" else "fused_pairs"
    tsb.set_workspace_limit(0)
    tsb.set_kernel_timing(True)
    try:
        tsb.set_wait_limit(1)
        tsb.set_wait_injection(True)
        try:
            with pytest.raises(tsb.TblisStraError) as ei:
                tsb.contract(level, 1.0, dA, ia, dB, ib, 0.0, C, ic, drop_in=True)
            assert ei.value.status == ERR_TIMEOUT
        finally:
            tsb.set_wait_limit(0)
            tsb.set_wait_injection(False)
        C.zero_()
        tsb.contract(level, 1.0, dA, ia, dB, ib, 0.0, C, ic, drop_in=True)
        assert tsb.kernel_timing(kind)[0] == 2
    finally:
        tsb.set_kernel_timing(False)
        tsb.set_workspace_limit(None)
    err = float(np.abs(C.cpu().numpy() - ref).max())
    assert err <= oracle.error_bound(level, k, mA, mB)


@pytest.mark.parametrize("level", [0, 1])
def test_wait_timeout_split_bf16_then_recovery(tsb, cuda, level):
    import torch
    A, B, _ = _problem()
    A32, B32 = A.astype(np.float32), B.astype(np.float32)
    ref = np.zeros((512, 512), order="F")
    oracle.contract(1.0, A32.astype(np.float64), "ik", B32.astype(np.float64), "kj", 0.0, ref, "ij")
    dA, dB = _dev(torch, np.asfortranarray(A32), cuda), _dev(torch, np.asfortranarray(B32), cuda)
    C = torch.zeros_like(dA)
    tsb.set_wait_limit(1)
    tsb.set_wait_injection(True)
    try:
        with pytest.raises(tsb.TblisStraError) as ei:
            tsb.contract(level, 1.0, dA, "ik", dB, "kj", 0.0, C, "ij", drop_in=True)
        assert ei.value.status == ERR_TIMEOUT
    finally:
        tsb.set_wait_limit(0)
        tsb.set_wait_injection(False)
    C.zero_()
    tsb.contract(level, 1.0, dA, "ik", dB, "kj", 0.0, C, "ij", drop_in=True)
    got = C.double().cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6


def test_alloc_ceiling_fails_cleanly_on_host_operands(tsb, cuda):
    """Host operands of a shape not planned before: the first allocation (the
    scatter-vector table) is refused; C on the host is untouched."""
    A = oracle.uniform((37, 41), 50)
    B = oracle.uniform((41, 43), 51)
    C = oracle.uniform((37, 43), 52)
    C0 = C.copy()
    tsb.set_alloc_limit(64)
    try:
        with pytest.raises(tsb.TblisStraError) as ei:
            tsb.contract(1, 1.0, A, "ik", B, "kj", 1.0, C, "ij", drop_in=True)
        assert ei.value.status == ERR_ALLOC
    finally:
        tsb.set_alloc_limit(None)
    assert np.array_equal(C, C0)
    ref = C0.copy(order="F")
    oracle.contract(1.0, A, "ik", B, "kj", 1.0, ref, "ij")
    tsb.contract(1, 1.0, A, "ik", B, "kj", 1.0, C, "ij", drop_in=True)
    assert float(np.abs(C - ref).max()) <= oracle.error_bound(1, 41, 1.0, 1.0) + 4 * 2.0 ** -53


def test_alloc_ceiling_fails_cleanly_on_workspace(tsb, cuda):
    """Device operands whose tables are already cached: the packed workspace
    (several MB) is above a 1 MiB ceiling, so the call fails before any kernel
    runs and C on the device is untouched."""
    import torch
    A, B, ref = _problem()
    dA, dB = _dev(torch, A, cuda), _dev(torch, B, cuda)
    C = torch.zeros_like(dA)
    tsb.contract(1, 1.0, dA, "ik", dB, "kj", 0.0, C, "ij", drop_in=True)      # caches the plan
    C.fill_(3.0)
    tsb.set_alloc_limit(1 << 20)
    try:
        with pytest.raises(tsb.TblisStraError) as ei:
            tsb.contract(1, 1.0, dA, "ik", dB, "kj", 0.0, C, "ij", drop_in=True)
        assert ei.value.status == ERR_ALLOC
    finally:
        tsb.set_alloc_limit(None)
    torch.cuda.synchronize()
    assert bool((C == 3.0).all())
