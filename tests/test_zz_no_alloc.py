"""tblis_stra_mult_noalloc: the entry point for callers that cannot allocate
device memory (an application pool owning the whole device, a plug-in host
that forbids device allocations, or code that cannot take cudaMalloc's
implicit synchronisation).  It keeps each contraction's scatter vectors in one
static 2 MiB device array instead of allocating them.

The GPU test calls it through the C ABI twice in a row (different shapes, so
the second call overwrites the first call's table) and checks each result
against the regular entry point tblis_stra_mult within the FP64 bound the
parity tests use.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from oracle import oracle


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


def _colmajor(torch, shape, gen, dev):
    t = torch.empty(tuple(reversed(shape)), dtype=torch.float64, device=dev)
    t.uniform_(-1, 1, generator=gen)
    return t.permute(*reversed(range(len(shape))))


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
    assert st == 8   # TBLIS_STRA_ERR_TOO_LARGE


@pytest.mark.gpu
def test_noalloc_matches_regular_entry_point_twice(tsb, cuda):
    import torch
    gen = torch.Generator(device=cuda).manual_seed(11)
    cases = [
        (1, (24, 20, 22, 18), (22, 18, 26, 24), "efac", "fbde", "abcd", dict(a=26, b=20, c=24, d=18, e=24, f=20)),
        (2, None, None, "ik", "kj", "ij", dict(i=300, j=257, k=190)),
    ]
    for level, _, _, ia, ib, ic, ext in cases:
        A = _colmajor(torch, [ext[c] for c in ia], gen, cuda)
        B = _colmajor(torch, [ext[c] for c in ib], gen, cuda)
        C0 = _colmajor(torch, [ext[c] for c in ic], gen, cuda)
        C_reg = C0.clone()
        C_new = C0.clone()
        tsb.contract(level, 1.5, A, ia, B, ib, 0.5, C_reg, ic)
        st = _call(tsb, level, 1.5, A, ia, B, ib, 0.5, C_new, ic)
        torch.cuda.synchronize()
        assert st == 0, tsb.status_string(st)
        k = int(np.prod([v for c, v in ext.items() if c not in ic]))
        bound = (oracle.error_bound(level, k, float(A.abs().max()), float(B.abs().max())) * 1.5
                 + 4 * 2.0 ** -53 * 0.5 * float(C0.abs().max()))
        err = float((C_new - C_reg).abs().max())
        assert err <= 2 * bound, (level, err, bound)


@pytest.mark.gpu
def test_noalloc_rejects_host_operands(tsb, cuda):
    A = np.ones((4, 4)); B = np.ones((4, 4)); C = np.zeros((4, 4))
    assert _call(tsb, 1, 1.0, A, "ik", B, "kj", 0.0, C, "ij") == 5   # TBLIS_STRA_ERR_ARG
