"""tblis_stra_mult_noalloc: the entry point for callers that cannot allocate
device memory (an application pool owning the whole device, a plug-in host
that forbids device allocations, or code that cannot take cudaMalloc's
implicit synchronisation).  It writes each contraction's scatter vectors into
one static 2 MiB device array instead of allocating them.

The GPU tests call it through the C ABI, several calls in a row with different
shapes (so each call overwrites the previous call's table), and check every
result against the oracle (the plain-C restatement of the reference's
contraction) within the FP64 bound the parity tests use, and against the
regular entry point tblis_stra_mult.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from oracle import oracle

ERR_ARG, ERR_TOO_LARGE, ERR_UNSUPPORTED = 5, 8, 9


def _fn(tsb):
    f = tsb.lib.tblis_stra_mult_noalloc
    T = ctypes.POINTER(tsb.tblis_tensor)
    f.argtypes = [ctypes.c_int, T, ctypes.c_char_p, T, ctypes.c_char_p, T, ctypes.c_char_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _call(tsb, level, alpha, A, ia, B, ib, beta, C, ic):
    va = tsb.tblis_stra._View(A, alpha)
    vb = tsb.tblis_stra._View(B, 1.0, va.code)
    vc = tsb.tblis_stra._View(C, beta, va.code)
    return _fn(tsb)(level, ctypes.byref(va.t), ia.encode(), ctypes.byref(vb.t), ib.encode(),
                    ctypes.byref(vc.t), ic.encode(), None)


def test_noalloc_symbol_declared_and_exported(tsb):
    assert hasattr(tsb.lib, "tblis_stra_mult_noalloc")


def test_noalloc_rejects_too_large_before_any_gpu_work(tsb):
    # 2*(m + n + k) = 2*(100000 + 100000 + 8) > 262144: rejected during planning
    A = np.zeros((1, 1)); B = np.zeros((1, 1)); C = np.zeros((1, 1))
    va, vb, vc = (tsb.tblis_stra._View(x, 1.0) for x in (A, B, C))
    for v, shp in ((va, (100000, 8)), (vb, (8, 100000)), (vc, (100000, 100000))):
        v.len[0], v.len[1] = shp
        v.stride[0], v.stride[1] = 1, shp[0]
    st = _fn(tsb)(1, ctypes.byref(va.t), b"ik", ctypes.byref(vb.t), b"kj", ctypes.byref(vc.t), b"ij", None)
    assert st == ERR_TOO_LARGE


def test_noalloc_rejects_fp32_before_any_gpu_work(tsb):
    # FP64 operands only: an FP32 request is refused after planning, before
    # any CUDA call (so this runs without a GPU).
    A = np.ones((4, 4), dtype=np.float32); B = np.ones((4, 4), dtype=np.float32)
    C = np.zeros((4, 4), dtype=np.float32)
    assert _call(tsb, 1, 1.0, A, "ik", B, "kj", 0.0, C, "ij") == ERR_UNSUPPORTED


def _colmajor_np(shape, seed):
    return oracle.uniform(shape, seed)


def _dev(torch, x, dev):
    t = torch.empty_strided(x.shape, [s // 8 for s in x.strides], dtype=torch.float64, device=dev)
    t.copy_(torch.from_numpy(x))
    return t


# (level, alpha, beta, idx_A, idx_B, idx_C, extents)
CASES = [
    (1, 1.5, 0.5, "efac", "fbde", "abcd", dict(a=26, b=20, c=24, d=18, e=24, f=20)),
    (2, 1.0, 0.0, "ik", "kj", "ij", dict(i=300, j=257, k=190)),
    (0, -0.75, 1.0, "kia", "jk", "ija", dict(i=33, j=40, k=65, a=3)),
    # batch label b (in A, B and C) and a C-only label z (broadcast)
    (1, 1.0, 0.5, "bik", "bkj", "bijz", dict(b=3, i=40, j=36, k=44, z=2)),
    # alpha = 0: C = beta * C, no product
    (2, 0.0, -2.0, "ik", "kj", "ij", dict(i=50, j=60, k=70)),
    (1, 2.0, 1.0, "efac", "fbde", "abcd", dict(a=9, b=7, c=6, d=5, e=8, f=7)),
]


@pytest.mark.gpu
def test_noalloc_matches_oracle_and_regular_entry_point(tsb, cuda):
    import torch
    for i, (level, alpha, beta, ia, ib, ic, ext) in enumerate(CASES):
        A = _colmajor_np([ext[c] for c in ia], 100 + 3 * i)
        B = _colmajor_np([ext[c] for c in ib], 101 + 3 * i)
        C0 = _colmajor_np([ext[c] for c in ic], 102 + 3 * i)
        ref = C0.copy(order="F")
        oracle.contract(alpha, A, ia, B, ib, beta, ref, ic)
        dA, dB = _dev(torch, A, cuda), _dev(torch, B, cuda)
        C_new, C_reg = _dev(torch, C0, cuda), _dev(torch, C0, cuda)
        st = _call(tsb, level, alpha, dA, ia, dB, ib, beta, C_new, ic)
        tsb.contract(level, alpha, dA, ia, dB, ib, beta, C_reg, ic)
        torch.cuda.synchronize()
        assert st == 0, (i, tsb.status_string(st))
        k = int(np.prod([v for c, v in ext.items() if c in ia and c in ib and c not in ic])) or 1
        bound = (oracle.error_bound(level, k, float(np.abs(A).max()), float(np.abs(B).max())) * abs(alpha)
                 + 4 * 2.0 ** -53 * abs(beta) * float(np.abs(C0).max()))
        got = C_new.cpu().numpy()
        err = float(np.abs(got - ref).max())
        assert err <= bound, ("vs oracle", i, level, err, bound)
        err_reg = float((C_new - C_reg).abs().max())
        assert err_reg <= 2 * bound, ("vs regular entry point", i, level, err_reg, bound)


@pytest.mark.gpu
def test_noalloc_rejects_host_operands(tsb, cuda):
    A = np.ones((4, 4)); B = np.ones((4, 4)); C = np.zeros((4, 4))
    assert _call(tsb, 1, 1.0, A, "ik", B, "kj", 0.0, C, "ij") == ERR_ARG


@pytest.mark.gpu
def test_noalloc_config1_vs_reference_L0(tsb, cuda):
    """C(abcd) += A(efac) B(fbde), extents 64 (NIm = NJn = NPk = 4096), seed-0
    U[-1,1] column-major inputs: the whole C against the reference library's
    own L=0 contraction, at L = 1 and then L = 2 (two calls in a row)."""
    import os
    import torch
    if not oracle.ref_available():
        pytest.skip("the reference library (oracle/_ref) is not built on this machine")
    e = 64
    A, B = oracle.uniform_pair((e,) * 4, (e,) * 4, seed=0)
    Cref = np.zeros((e,) * 4, order="F")
    oracle.ref_set_threads(os.cpu_count() or 1)
    oracle.ref_mult(0, 1, 1.0, A, "efac", B, "fbde", 1.0, Cref, "abcd")
    dA, dB = _dev(torch, A, cuda), _dev(torch, B, cuda)
    for level in (1, 2):
        C = _dev(torch, np.zeros((e,) * 4, order="F"), cuda)
        st = _call(tsb, level, 1.0, dA, "efac", dB, "fbde", 1.0, C, "abcd")
        torch.cuda.synchronize()
        assert st == 0, tsb.status_string(st)
        bound = oracle.error_bound(level, e * e, float(np.abs(A).max()), float(np.abs(B).max()))
        err = float(np.abs(C.cpu().numpy() - Cref).max())
        assert err <= bound, (level, err, bound)
