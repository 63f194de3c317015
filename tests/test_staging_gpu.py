"""Host-resident operands: the drop-in calls stage them through device memory.
When all three are on the host and large (>= 64 MiB together), the call
splits C's slowest label that belongs to exactly one of A and B into 4 chunks
and, when C's layout allows a second cut, the other operand in 2 along one of
its C labels (8 chunks), and overlaps the copies of one chunk with the
computation of another.  Each chunk is the same contraction on sub-views, so
the result matches the all-device call within the Strassen bound (both are
within it of the exact contraction)."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


def bound(level, k, beta=1.0):
    return 2 * oracle.error_bound(level, k, 1.0, 1.0) + 8 * 2.0 ** -53 * abs(beta)


def run_pair(tsb, cuda, level, A, ia, B, ib, C0, ic, pinned):
    import torch
    hA, hB, hC = (torch.from_numpy(X) for X in (A, B, C0.copy(order="K")))
    if pinned:
        hA, hB, hC = hA.pin_memory(), hB.pin_memory(), hC.pin_memory()
    before = tsb.launch_count()
    tsb.contract(level, 1.0, hA, ia, hB, ib, 1.0, hC, ic, drop_in=True)
    launches = tsb.launch_count() - before
    dA, dB, dC = hA.to(cuda), hB.to(cuda), torch.from_numpy(C0.copy(order="K")).to(cuda)
    tsb.contract(level, 1.0, dA, ia, dB, ib, 1.0, dC, ic)
    torch.cuda.synchronize()
    return hC.numpy(), dC.cpu().numpy(), launches


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("level", [0, 1])
def test_pipelined_split_of_b_and_c(tsb, cuda, level, pinned):
    """Column-major config-1 pattern: C's slowest label d is in B and C."""
    e = 42                                   # 3 x 24.9 MB
    A = oracle.uniform((e,) * 4, 1)
    B = oracle.uniform((e,) * 4, 2)
    C0 = oracle.uniform((e,) * 4, 3)
    got, want, launches = run_pair(tsb, cuda, level, A, "efac", B, "fbde", C0, "abcd", pinned)
    assert np.abs(got - want).max() <= bound(level, e * e)
    # L=0 (28 tiles, k 1764: k-split in 3 pieces): 2 packs + the GEMM over the
    # pieces + the combine; L=1 (14 tiles per product, product-parallel):
    # 2 group packs + the GEMM over the 7 products + the combine
    per_call = 4
    assert launches == 8 * per_call          # d in 4 chunks x c in 2


def test_pipelined_split_of_a_and_c_row_major(tsb, cuda):
    """Row-major operands: C's slowest label a is in A and C."""
    e = 42
    A = np.ascontiguousarray(oracle.uniform((e,) * 4, 4))
    B = np.ascontiguousarray(oracle.uniform((e,) * 4, 5))
    C0 = np.ascontiguousarray(oracle.uniform((e,) * 4, 6))
    got, want, launches = run_pair(tsb, cuda, 1, A, "aefc", B, "fbde", C0, "abcd", True)
    assert np.abs(got - want).max() <= bound(1, e * e)
    assert launches == 8 * 4                 # a in 4 x b in 2; product-parallel L=1 per chunk


def test_pipelined_fp32(tsb, cuda):
    import torch
    e = 52                                   # 3 x 29 MB of FP32
    A = oracle.uniform((e,) * 4, 7, dtype=np.float32)
    B = oracle.uniform((e,) * 4, 8, dtype=np.float32)
    C0 = oracle.uniform((e,) * 4, 9, dtype=np.float32)
    got, want, launches = run_pair(tsb, cuda, 0, A, "efac", B, "fbde", C0, "abcd", True)
    d = np.linalg.norm((got.astype(np.float64) - want).ravel()) / np.linalg.norm(want.ravel())
    assert d <= 2e-6
    # 8 chunks of 1352 x 676 x 2704 (66 tiles: k-split in 5 pieces): 2 scales,
    # 2 packs, the GEMM over the pieces, the combine
    assert launches == 8 * 6


def test_pipelined_one_cut_with_batch_label(tsb, cuda):
    """A batch label z outermost in C leaves no 2-D block of C for a second
    cut: d alone is cut in 4 chunks, A copied whole."""
    e, z = 32, 3                             # 3 x 25 MB
    A = np.asfortranarray(oracle.uniform((e, e, e, e, z), 19))
    B = np.asfortranarray(oracle.uniform((e, e, e, e, z), 20))
    C0 = np.asfortranarray(oracle.uniform((e, e, e, e, z), 21))
    got, want, launches = run_pair(tsb, cuda, 1, A, "efacz", B, "fbdez", C0, "abcdz", True)
    assert np.abs(got - want).max() <= bound(1, e * e)
    assert launches == 4 * 4                 # 4 chunks; product-parallel L=1 per chunk


def test_small_or_unsliceable_operands_stage_whole(tsb, cuda):
    """Below 64 MiB (or when no label slices into plain rows) the operands are
    staged whole: one contraction's launches."""
    e = 20
    A = oracle.uniform((e,) * 4, 10)
    B = oracle.uniform((e,) * 4, 11)
    C0 = oracle.uniform((e,) * 4, 12)
    got, want, launches = run_pair(tsb, cuda, 1, A, "efac", B, "fbde", C0, "abcd", True)
    assert np.abs(got - want).max() <= bound(1, e * e)
    assert launches == 4                     # product-parallel L=1


def test_host_views_with_gaps_are_staged_whole(tsb, cuda):
    """A host C that is a strided view (every other element of a larger
    array) has no dense slices: the call stages the operands whole (one
    contraction's launches) and still meets the bound."""
    import torch
    e = 42
    A = oracle.uniform((e,) * 4, 13)
    B = oracle.uniform((e,) * 4, 14)
    big = np.asfortranarray(oracle.uniform((2 * e, e, e, e), 15))
    C0 = big[::2]                                  # gap between rows
    R = np.array(C0, copy=True, order="F")
    oracle_bound = bound(1, e * e)
    hA, hB = torch.from_numpy(A), torch.from_numpy(B)
    hBig = torch.from_numpy(big)
    hC = hBig[::2]
    dA, dB, dR = hA.to(cuda), hB.to(cuda), torch.from_numpy(R).to(cuda)
    before = tsb.launch_count()
    tsb.contract(1, 1.0, hA, "efac", hB, "fbde", 1.0, hC, "abcd", drop_in=True)
    assert tsb.launch_count() - before == 4    # product-parallel L=1
    tsb.contract(1, 1.0, dA, "efac", dB, "fbde", 1.0, dR, "abcd")
    torch.cuda.synchronize()
    assert np.abs(hC.numpy() - dR.cpu().numpy()).max() <= oracle_bound
    # the untouched rows between the view's rows are unchanged
    assert np.array_equal(hBig[1::2].numpy(), big[1::2])


def test_negative_strides_on_host(tsb, cuda):
    """Host operands with a reversed axis (negative stride) are staged whole."""
    import torch
    e = 42
    A = oracle.uniform((e,) * 4, 16)
    B = oracle.uniform((e,) * 4, 17)
    C0 = oracle.uniform((e,) * 4, 18)
    hA = torch.from_numpy(A).flip(0)               # torch flip copies; use numpy views instead
    nA = A[::-1]
    R = C0.copy(order="F")
    dC = torch.from_numpy(R).to(cuda)
    tsb.contract(1, 1.0, torch.from_numpy(np.ascontiguousarray(nA)).to(cuda), "efac",
                 torch.from_numpy(B).to(cuda), "fbde", 1.0, dC, "abcd")
    hC = C0.copy(order="F")
    tsb.contract(1, 1.0, nA, "efac", B, "fbde", 1.0, hC, "abcd", drop_in=True)
    torch.cuda.synchronize()
    assert np.abs(hC - dC.cpu().numpy()).max() <= bound(1, e * e)
    del hA
