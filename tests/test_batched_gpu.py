"""Batched uneven form: many contractions planned once (tblis_stra_batch_*),
executed as grouped persistent launches captured in one CUDA graph, with
autotuned and fixed Strassen levels; every problem checked against the
library's single-contraction L=0 path (itself checked against the oracle)
and two problems against the oracle directly."""
import numpy as np
import pytest

from oracle import oracle
from tests.batched_cases import draw_problem

pytestmark = pytest.mark.gpu


def make_batch(cuda, n, seed, dtype, lo, hi, pmin, pmax, level):
    import torch
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=cuda).manual_seed(seed)
    probs = []
    for i in range(n):
        ext, ia, ib, ic = draw_problem(rng, lo, hi, pmin, pmax)
        A = torch.rand([ext[c] for c in ia], dtype=dtype, device=cuda, generator=g) * 2 - 1
        B = torch.rand([ext[c] for c in ib], dtype=dtype, device=cuda, generator=g) * 2 - 1
        C = torch.rand([ext[c] for c in ic], dtype=dtype, device=cuda, generator=g) * 2 - 1
        lv = level if level != "mixed" else (-1 if i % 2 else i % 3)
        probs.append((1.0 + 0.25 * (i % 3), A, ia, B, ib, 0.5 * (i % 2), C, ic, lv))
    return probs


@pytest.mark.parametrize("level", [-1, 0, 1, 2, "mixed"])
def test_batched_fp64_matches_single_calls(tsb, cuda, level):
    import torch
    probs = make_batch(cuda, 24, 3, torch.float64, 4, 20, 64, 1024, level)
    refs = []
    for alpha, A, ia, B, ib, beta, C, ic, _ in probs:
        R = C.clone()
        tsb.contract(0, alpha, A, ia, B, ib, beta, R, ic)
        refs.append(R)
    batch = tsb.Batch(probs)
    levels = batch.levels()
    assert all(l in (0, 1, 2) for l in levels)
    if level in (0, 1, 2):
        assert levels == [level] * len(probs)
    batch.execute()
    torch.cuda.synchronize()
    for (alpha, A, ia, B, ib, beta, C, ic, _), R, lv in zip(probs, refs, levels):
        k = int(np.prod([s for c, s in zip(ia, A.shape) if c not in ic]))
        bound = oracle.error_bound(lv, k, 1.0, 1.0) * 2 + 1e-13
        assert float((C - R).abs().max()) <= bound, (ia, ib, ic, lv)
    # a second execution of the same graph gives the same contraction again
    before = [C.clone() for (_, _, _, _, _, _, C, _, _) in probs]
    batch.execute()
    torch.cuda.synchronize()
    for (alpha, A, ia, B, ib, beta, C, ic, _), C1 in zip(probs, before):
        R = C1.clone()
        tsb.contract(0, alpha, A, ia, B, ib, beta, R, ic)
        assert torch.allclose(C, R, atol=1e-10, rtol=0)
    batch.close()


def test_batched_against_oracle(tsb, cuda):
    import torch
    probs = make_batch(cuda, 6, 9, torch.float64, 3, 9, 16, 128, -1)
    host = [(alpha, A.cpu().numpy(), ia, B.cpu().numpy(), ib, beta, C.cpu().numpy().copy(), ic)
            for alpha, A, ia, B, ib, beta, C, ic, _ in probs]
    batch = tsb.Batch(probs)
    batch.execute()
    torch.cuda.synchronize()
    for (alpha, A, ia, B, ib, beta, C0, ic), p, lv in zip(host, probs, batch.levels()):
        R = np.asarray(C0, dtype=np.float64).copy()
        oracle.contract(alpha, np.ascontiguousarray(A), ia, np.ascontiguousarray(B), ib, beta, R, ic)
        k = int(np.prod([s for c, s in zip(ia, A.shape) if c not in ic]))
        assert np.abs(p[6].cpu().numpy() - R).max() <= oracle.error_bound(lv, k, 1.0, 1.0) * 2 + 1e-13


def test_batched_fp32_split(tsb, cuda):
    import torch
    probs = make_batch(cuda, 8, 5, torch.float32, 4, 16, 64, 512, -1)
    refs = []
    for alpha, A, ia, B, ib, beta, C, ic, _ in probs:
        R = C.double()
        tsb.contract(0, alpha, A.double(), ia, B.double(), ib, beta, R, ic)
        refs.append(R)
    batch = tsb.Batch(probs)
    batch.execute()
    torch.cuda.synchronize()
    for (alpha, A, ia, B, ib, beta, C, ic, _), R in zip(probs, refs):
        err = float(torch.linalg.norm((C.double() - R).flatten()) / torch.linalg.norm(R.flatten()))
        assert err <= 1e-6, err


@pytest.mark.parametrize("schedule", ["fused", "fused_small", "packed_grouped", "packed"])
@pytest.mark.parametrize("level", [-1, 0, 1, 2])
def test_batched_fp64_each_schedule(tsb, cuda, schedule, level):
    """Every FP64 schedule, alone, against single L=0 calls; packed_grouped
    with a 1 MiB chunk limit, so every problem is its own chunk and the two
    chunk workspaces alternate (packing of chunk c waits for the GEMM of
    chunk c-2)."""
    import os
    import torch
    probs = make_batch(cuda, 12, 21, torch.float64, 4, 20, 64, 1024, level)
    refs = []
    for alpha, A, ia, B, ib, beta, C, ic, _ in probs:
        R = C.clone()
        tsb.contract(0, alpha, A, ia, B, ib, beta, R, ic)
        refs.append(R)
    os.environ["TBLIS_STRA_BATCH_CHUNK_BYTES"] = str(1 << 20)
    try:
        tsb.set_batch_schedules([schedule])
        if (schedule == "fused_small" and level == 1) or (schedule == "packed_grouped" and level in (1, 2)):
            with pytest.raises(tsb.TblisStraError):
                tsb.Batch(probs)
            return
        batch = tsb.Batch(probs)
    finally:
        tsb.set_batch_schedules(None)
        del os.environ["TBLIS_STRA_BATCH_CHUNK_BYTES"]
    levels, sched = batch.levels(), batch.schedule()
    assert set(sched) == {schedule}
    if level >= 0:
        assert levels == [level] * len(probs)
    for rep in range(2):
        if rep:   # the second execution starts from the first one's C
            refs = []
            for alpha, A, ia, B, ib, beta, C, ic, _ in probs:
                R = C.clone()
                tsb.contract(0, alpha, A, ia, B, ib, beta, R, ic)
                refs.append(R)
        batch.execute()
        torch.cuda.synchronize()
        for (alpha, A, ia, B, ib, beta, C, ic, _), R, lv in zip(probs, refs, levels):
            k = int(np.prod([s for c, s in zip(ia, A.shape) if c not in ic]))
            bound = oracle.error_bound(lv, k, 1.0, 1.0) * 2 + 1e-13
            assert float((C - R).abs().max()) <= bound, (schedule, ia, ib, ic, lv, rep)
    c, t, n = batch.stats()
    assert c >= t >= 0.0 and n >= 0
    batch.close()


def test_batched_fp64_large_levels(tsb, cuda):
    """Problems large enough for the tuner to consider L=1 (blocks of 1024 in
    every dimension), mixed with small ones, against single L=0 calls."""
    import torch
    g = torch.Generator(device=cuda).manual_seed(4)
    shapes = [((48, 48), (48, 48), (48, 48)), ((8, 16), (32, 8), (16, 16)), ((64, 40), (40, 64), (32, 64))]
    probs, refs = [], []
    for (m1, m2), (n1, n2), (k1, k2) in shapes:
        A = torch.rand((m1, k1, m2, k2), dtype=torch.float64, device=cuda, generator=g) * 2 - 1
        B = torch.rand((k2, n1, k1, n2), dtype=torch.float64, device=cuda, generator=g) * 2 - 1
        C = torch.rand((n1, m1, m2, n2), dtype=torch.float64, device=cuda, generator=g) * 2 - 1
        probs.append((1.0, A, "aibj", B, "jcid", 1.0, C, "cabd", -1))
        R = C.clone()
        tsb.contract(0, 1.0, A, "aibj", B, "jcid", 1.0, R, "cabd")
        refs.append(R)
    batch = tsb.Batch(probs)
    batch.execute()
    torch.cuda.synchronize()
    for (_, A, ia, B, ib, _, C, ic, _), R, lv in zip(probs, refs, batch.levels()):
        k = int(np.prod([s for c, s in zip(ia, A.shape) if c not in ic]))
        assert float((C - R).abs().max()) <= oracle.error_bound(lv, k, 1.0, 1.0) * 2 + 1e-13


@pytest.mark.parametrize("schedule", ["split", "split_grouped"])
def test_batched_fp32_each_schedule(tsb, cuda, schedule):
    """FP32 problems through one schedule, against single L=0 FP64 calls of the
    same values; split_grouped with a 1 MiB chunk limit, so chunks alternate
    between the two workspaces."""
    import os
    import torch
    probs = make_batch(cuda, 10, 31, torch.float32, 4, 16, 64, 512, 0)
    refs = []
    for alpha, A, ia, B, ib, beta, C, ic, _ in probs:
        R = C.double()
        tsb.contract(0, alpha, A.double(), ia, B.double(), ib, beta, R, ic)
        refs.append(R)
    os.environ["TBLIS_STRA_BATCH_CHUNK_BYTES"] = str(1 << 20)
    try:
        tsb.set_batch_schedules([schedule])
        batch = tsb.Batch(probs)
    finally:
        tsb.set_batch_schedules(None)
        del os.environ["TBLIS_STRA_BATCH_CHUNK_BYTES"]
    assert set(batch.schedule()) == {schedule}
    batch.execute()
    torch.cuda.synchronize()
    for (alpha, A, ia, B, ib, beta, C, ic, _), R in zip(probs, refs):
        err = float(torch.linalg.norm((C.double() - R).flatten()) / torch.linalg.norm(R.flatten()))
        assert err <= 1e-6, (schedule, err)
    batch.close()


def test_batch_rejects_host_tensors(tsb):
    A = np.ones((4, 4)); B = np.ones((4, 4)); C = np.zeros((4, 4))
    with pytest.raises(tsb.TblisStraError):
        tsb.Batch([(1.0, A, "ik", B, "kj", 0.0, C, "ij", 0)])


def test_batch_empty_and_trivial_problems(tsb, cuda):
    """No problems; a problem with an empty C; alpha = 0 (C = beta*C); an empty
    contracted range (C = beta*C) -- next to an ordinary problem."""
    import torch
    b0 = tsb.Batch([])
    b0.execute()
    b0.close()
    g = torch.Generator(device=cuda).manual_seed(8)
    rnd = lambda *s: torch.rand(s, dtype=torch.float64, device=cuda, generator=g) * 2 - 1
    A, B, C = rnd(30, 40), rnd(40, 20), rnd(30, 20)
    E_A, E_B, E_C = rnd(0, 40), rnd(40, 20), rnd(0, 20)           # m = 0
    K_A, K_B, K_C = rnd(30, 0), rnd(0, 20), rnd(30, 20)           # k = 0
    Z_C = rnd(30, 20)
    C0, K0, Z0 = C.clone(), K_C.clone(), Z_C.clone()
    probs = [(1.0, A, "ik", B, "kj", 0.5, C, "ij", -1),
             (1.0, E_A, "ik", E_B, "kj", 1.0, E_C, "ij", -1),
             (1.0, K_A, "ik", K_B, "kj", 0.25, K_C, "ij", -1),
             (0.0, A, "ik", B, "kj", 2.0, Z_C, "ij", 1)]
    batch = tsb.Batch(probs)
    assert batch.schedule()[2] == "scale" and batch.schedule()[3] == "scale"
    batch.execute()
    torch.cuda.synchronize()
    R = 0.5 * C0 + A @ B
    assert float((C - R).abs().max()) <= oracle.error_bound(2, 40, 1.0, 1.0) * 2 + 1e-13
    assert torch.equal(K_C, 0.25 * K0)
    assert torch.equal(Z_C, 2.0 * Z0)
    batch.close()
