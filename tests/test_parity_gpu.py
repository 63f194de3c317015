"""Parity of the CUDA path with the oracle and with the reference's own
outputs (golden fixtures), through the C ABI, on the GPU.

Bound (FP64):  max|C - Cref| <= 4 * 12^L * NPk * 2^-53 * max|A| * max|B|
scaled by |alpha| and widened by the rounding of beta*C (4 * 2^-53 * |beta| *
max|C0|), where NPk is the length of the summed index range.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "manifest.json")) as f:
    MANIFEST = json.load(f)


def tol(level, k, A, B, alpha=1.0, beta=0.0, C0=None):
    t = oracle.error_bound(level, max(k, 1), np.abs(A).max(), np.abs(B).max()) * max(abs(alpha), 1.0)
    if beta != 0.0 and C0 is not None and C0.size:
        t += 4 * 2.0 ** -53 * abs(beta) * np.abs(C0).max()
    return t + 1e-300


def to_dev(x, cuda):
    import torch
    # keep the numpy strides (column-major stays column-major)
    out = torch.empty_strided(x.shape, [s // x.itemsize for s in x.strides], dtype=torch.float64, device=cuda)
    out.copy_(torch.from_numpy(x))
    return out


@pytest.fixture(params=["packed", "packed_single", "packed_parallel", "fused"])
def schedule(request, tsb, monkeypatch):
    """ABC runs packed operand sums (at L >= 1 the 7 sums of a product group
    formed in one pass, the group's products run tile by tile in one GEMM),
    packed sums one product at a time (workspace limited to one product's S
    and T), all products side by side into M_p and one combine pass
    (product-parallel, the automatic choice for small grids), or, with no
    workspace, the fully fused kernel; all must meet the same bound."""
    tsb.set_product_parallel(1 if request.param == "packed_parallel" else 0)
    if request.param == "packed_single":
        orig = tsb.contract

        def contract(level, alpha, A, ia, B, ib, beta, C, ic, **kw):
            tsb.set_workspace_limit(single_product_bytes(tsb, level, A, ia, B, ib, C, ic))
            try:
                return orig(level, alpha, A, ia, B, ib, beta, C, ic, **kw)
            finally:
                tsb.set_workspace_limit(None)

        monkeypatch.setattr(tsb, "contract", contract)
    else:
        tsb.set_workspace_limit(None if request.param == "packed" else 0)
    yield request.param
    tsb.set_workspace_limit(None)
    tsb.set_product_parallel(-1)


def single_product_bytes(tsb, level, A, ia, B, ib, C, ic):
    """Workspace of one product's packed S and T (tile rows 128, k padded to 32)."""
    q = tsb.plan_query(A, ia, B, ib, C, ic, scatter=False)
    H = 1 << level
    cdiv = lambda a, b: -(-a // b)
    ms, ns, ks = cdiv(q["m"], H), cdiv(q["n"], H), cdiv(q["k"], H)
    kpad = cdiv(ks, 32) * 32
    return 8 * q["batch"] * (cdiv(ms, 128) + cdiv(ns, 128)) * 128 * kpad


def run_gpu(tsb, cuda, level, impl, alpha, A, ia, B, ib, beta, C0, ic):
    import torch
    dA, dB, dC = to_dev(A, cuda), to_dev(B, cuda), to_dev(C0, cuda)
    tsb.contract(level, alpha, dA, ia, dB, ib, beta, dC, ic, impl=impl)
    torch.cuda.synchronize()
    return dC.cpu().numpy()


def summed_len(ext, ic):
    return int(np.prod([v for c, v in ext.items() if c not in ic])) if ext else 1


@pytest.mark.parametrize("case", MANIFEST, ids=[c["name"] for c in MANIFEST])
def test_golden_all_levels_and_impls(tsb, cuda, case, schedule):
    d = np.load(os.path.join(GOLDEN, case["name"] + ".npz"))
    A, B, C0 = (np.asfortranarray(d[x]) for x in ("A", "B", "C0"))
    k = summed_len(case["extents"], case["idx_C"])
    for level in (0, 1, 2):
        for impl in ((1,) if level == 0 else (1, 2, 3)):
            C = run_gpu(tsb, cuda, level, impl, case["alpha"], A, case["idx_A"], B, case["idx_B"],
                        case["beta"], C0, case["idx_C"])
            key = f"L{level}_impl{impl}" if level else "L0"
            ref = d[key] if key in d.files else d["L0"]   # reference Strassen invalid -> judge against L=0
            t = tol(level, k, A, B, case["alpha"], case["beta"], C0)
            err = np.abs(C - ref).max()
            assert err <= t, (key, err, t)


def rand_case(seed):
    rng = np.random.default_rng(seed)
    labels = "abcdef"
    ext = {c: int(rng.integers(3, 21)) for c in labels}
    # I = {a, c}, J = {b, d}, P = {e, f}; random operand orders
    ia = "".join(rng.permutation(list("acef")))
    ib = "".join(rng.permutation(list("bdef")))
    ic = "".join(rng.permutation(list("abcd")))
    return ext, ia, ib, ic


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("level", [0, 1, 2])
def test_random_4d_vs_oracle(tsb, cuda, seed, level, schedule):
    ext, ia, ib, ic = rand_case(seed)
    order = "F" if seed % 2 == 0 else "C"
    A = oracle.uniform([ext[c] for c in ia], seed, order)
    B = oracle.uniform([ext[c] for c in ib], seed + 50, order)
    C0 = oracle.uniform([ext[c] for c in ic], seed + 99, order)
    for alpha, beta in ((1.0, 1.0), (-2.0, 0.0), (0.5, 0.5)):
        Co = C0.copy(order="K")
        oracle.contract(alpha, A, ia, B, ib, beta, Co, ic)
        for impl in ((1,) if level == 0 else (1, 2, 3)):
            C = run_gpu(tsb, cuda, level, impl, alpha, A, ia, B, ib, beta, C0, ic)
            t = tol(level, ext["e"] * ext["f"], A, B, alpha, beta, C0)
            assert np.abs(C - Co).max() <= t, (impl, alpha, beta)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (1, 7, 3), (5, 1, 9), (129, 130, 17), (257, 3, 300), (2, 2, 1)])
@pytest.mark.parametrize("level", [0, 1, 2])
def test_matrix_edges(tsb, cuda, m, n, k, level, schedule):
    A = oracle.uniform((m, k), 1)
    B = oracle.uniform((k, n), 2)
    C0 = oracle.uniform((m, n), 3)
    ref = 1.25 * (A @ B) + 0.75 * C0
    for impl in ((1,) if level == 0 else (1, 2, 3)):
        C = run_gpu(tsb, cuda, level, impl, 1.25, A, "ik", B, "kj", 0.75, C0, "ij")
        assert np.abs(C - ref).max() <= tol(level, k, A, B, 1.25, 0.75, C0) + 1e-13


def test_beta_zero_ignores_nan_in_c(tsb, cuda):
    A = oracle.uniform((40, 30), 1)
    B = oracle.uniform((30, 20), 2)
    C0 = np.full((40, 20), np.nan)
    for level in (0, 1, 2):
        C = run_gpu(tsb, cuda, level, 1, 1.0, A, "ik", B, "kj", 0.0, C0, "ij")
        assert np.isfinite(C).all()
        assert np.abs(C - A @ B).max() < 1e-12


def test_alpha_zero_and_empty_k(tsb, cuda):
    A = oracle.uniform((6, 5), 1)
    B = oracle.uniform((5, 4), 2)
    C0 = oracle.uniform((6, 4), 3)
    C = run_gpu(tsb, cuda, 1, 1, 0.0, A, "ik", B, "kj", 0.5, C0, "ij")
    np.testing.assert_allclose(C, 0.5 * C0, rtol=0, atol=1e-15)
    C = run_gpu(tsb, cuda, 1, 1, 0.0, A, "ik", B, "kj", 0.0, C0, "ij")
    assert not C.any()
    Ae = np.zeros((6, 0)); Be = np.zeros((0, 4))
    C = run_gpu(tsb, cuda, 2, 1, 1.0, Ae, "ik", Be, "kj", 2.0, C0, "ij")
    np.testing.assert_allclose(C, 2.0 * C0, rtol=0, atol=1e-15)


def test_host_pointers_are_staged(tsb, cuda):
    A = oracle.uniform((8, 8, 8, 8), 5)
    B = oracle.uniform((8, 8, 8, 8), 6)
    C = oracle.uniform((8, 8, 8, 8), 7)
    Co = C.copy(order="F")
    oracle.contract(1.0, A, "efac", B, "fbde", 1.0, Co, "abcd")
    for level in (0, 1, 2):
        Ch = C.copy(order="F")
        tsb.contract(level, 1.0, A, "efac", B, "fbde", 1.0, Ch, "abcd", drop_in=True)
        assert np.abs(Ch - Co).max() <= tol(level, 64, A, B, 1.0, 1.0, C)


def test_strided_views_leave_gaps_untouched(tsb, cuda):
    import torch
    big = torch.full((20, 30), 7.0, dtype=torch.float64, device=cuda)
    Cv = big[2:18:2, 3:27:3]          # 8 x 8 view with gaps
    A = torch.rand(8, 5, dtype=torch.float64, device=cuda)
    B = torch.rand(5, 8, dtype=torch.float64, device=cuda)
    tsb.contract(1, 1.0, A, "ik", B, "kj", 0.0, Cv, "ij")
    torch.cuda.synchronize()
    assert torch.allclose(Cv, A @ B, atol=1e-13)
    mask = torch.ones_like(big, dtype=torch.bool)
    mask[2:18:2, 3:27:3] = False
    assert bool((big[mask] == 7.0).all())


def test_async_stream_entry_point(tsb, cuda):
    import torch
    s = torch.cuda.Stream()
    A = torch.rand(300, 200, dtype=torch.float64, device=cuda)
    B = torch.rand(200, 100, dtype=torch.float64, device=cuda)
    C = torch.zeros(300, 100, dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        tsb.contract(1, 1.0, A, "ik", B, "kj", 0.0, C, "ij", stream=s)
    s.synchronize()
    assert torch.allclose(C, A @ B, atol=1e-12)


@pytest.mark.parametrize("order", ["F", "C"])
@pytest.mark.parametrize("level", [1, 2])
def test_product_parallel_batch_and_beta0(tsb, cuda, level, order):
    """Product-parallel ABC with a batch label, ragged blocks, both M layouts
    (C column- or row-major) and beta = 0 over a NaN-filled C: C is written,
    never read."""
    ext = dict(i=131, j=67, k=150, z=3)
    A = oracle.uniform((ext["i"], ext["k"], ext["z"]), 4, order)
    B = oracle.uniform((ext["k"], ext["j"], ext["z"]), 5, order)
    C0 = np.full((ext["i"], ext["j"], ext["z"]), np.nan, order=order)
    R = np.zeros(C0.shape, order=order)
    oracle.contract(-1.5, A, "ikz", B, "kjz", 0.0, R, "ijz")
    tsb.set_product_parallel(1)
    try:
        C = run_gpu(tsb, cuda, level, 1, -1.5, A, "ikz", B, "kjz", 0.0, C0, "ijz")
    finally:
        tsb.set_product_parallel(-1)
    assert np.isfinite(C).all()
    assert np.abs(C - R).max() <= tol(level, ext["k"], A, B, -1.5)


@pytest.mark.parametrize("order", ["F", "C"])
def test_ksplit_small_grid_large_k(tsb, cuda, order):
    """L=0 with fewer C tiles than SMs and a long summed range: k is cut into
    pieces run side by side and summed by the combine pass (9 pieces here:
    4 tiles, k = 5000), with a batch label and beta = 0 over a NaN-filled C."""
    import torch
    ext = dict(i=200, j=190, k=5000, z=2)
    A = oracle.uniform((ext["i"], ext["k"], ext["z"]), 31, order)
    B = oracle.uniform((ext["k"], ext["j"], ext["z"]), 32, order)
    C0 = np.full((ext["i"], ext["j"], ext["z"]), np.nan, order=order)
    R = np.zeros(C0.shape, order=order)
    oracle.contract(0.5, A, "ikz", B, "kjz", 0.0, R, "ijz")
    before = tsb.launch_count()
    C = run_gpu(tsb, cuda, 0, 1, 0.5, A, "ikz", B, "kjz", 0.0, C0, "ijz")
    # tiles: 2 x 2 x batch 2 = 8; pieces min(ceil(296 / 8), 5000 // 512) = 9:
    # one pack per operand, the GEMM over the pieces, the combine
    assert tsb.launch_count() - before == 4
    assert np.isfinite(C).all()
    assert np.abs(C - R).max() <= tol(0, ext["k"], A, B, 0.5)
    tsb.set_product_parallel(0)
    try:
        before = tsb.launch_count()
        C = run_gpu(tsb, cuda, 0, 1, 0.5, A, "ikz", B, "kjz", 0.0, C0, "ijz")
        assert tsb.launch_count() - before == 3        # no split: 2 packs + GEMM
    finally:
        tsb.set_product_parallel(-1)
    assert np.abs(C - R).max() <= tol(0, ext["k"], A, B, 0.5)


def test_launch_counter_moves(tsb, cuda):
    A = oracle.uniform((16, 16), 1)
    tsb.set_workspace_limit(0)
    try:
        before = tsb.launch_count()
        run_gpu(tsb, cuda, 1, 1, 1.0, A, "ik", A, "kj", 0.0, A, "ij")
        assert tsb.launch_count() == before + 1     # fused ABC: one persistent launch
    finally:
        tsb.set_workspace_limit(None)
    before = tsb.launch_count()
    run_gpu(tsb, cuda, 1, 1, 1.0, A, "ik", A, "kj", 0.0, A, "ij")
    assert tsb.launch_count() == before + 4         # small grid: pack 7 S, pack 7 T, GEMM of all 7, combine
    before = tsb.launch_count()
    run_gpu(tsb, cuda, 2, 1, 1.0, A, "ik", A, "kj", 0.0, A, "ij")
    assert tsb.launch_count() == before + 16        # L=2: 7 groups x 2 packs, GEMM of all 49, combine
    tsb.set_product_parallel(0)
    try:
        before = tsb.launch_count()
        run_gpu(tsb, cuda, 1, 1, 1.0, A, "ik", A, "kj", 0.0, A, "ij")
        assert tsb.launch_count() == before + 3     # grouped: pack 7 S, pack 7 T, one GEMM for the group
        tsb.set_workspace_limit(single_product_bytes(tsb, 1, A, "ik", A, "kj", A, "ij"))
        before = tsb.launch_count()
        run_gpu(tsb, cuda, 1, 1, 1.0, A, "ik", A, "kj", 0.0, A, "ij")
        assert tsb.launch_count() == before + 21    # one product at a time: 7 x (pack S, pack T, GEMM)
    finally:
        tsb.set_workspace_limit(None)
        tsb.set_product_parallel(-1)


@pytest.mark.parametrize("level", [1, 2])
def test_sampled_entries_at_config1_size(tsb, cuda, level, schedule):
    """Config-1 pattern at extent 64 (NIm=NJn=NPk=4096): too large for the
    oracle's loop, so 4096 sampled entries of C are checked against exact
    dot products, and L vs L=0 on the GPU against the bound."""
    import torch
    e = 64
    g = torch.Generator(device=cuda).manual_seed(0)
    A = (torch.rand((e,) * 4, dtype=torch.float64, device=cuda, generator=g) * 2 - 1).permute(3, 2, 1, 0).contiguous().permute(3, 2, 1, 0)
    B = (torch.rand((e,) * 4, dtype=torch.float64, device=cuda, generator=g) * 2 - 1).permute(3, 2, 1, 0).contiguous().permute(3, 2, 1, 0)
    C0 = torch.zeros((e,) * 4, dtype=torch.float64, device=cuda).permute(3, 2, 1, 0).contiguous().permute(3, 2, 1, 0)
    C0.zero_()
    C1 = C0.clone(memory_format=torch.preserve_format)
    tsb.contract(0, 1.0, A, "efac", B, "fbde", 0.0, C0, "abcd")
    tsb.contract(level, 1.0, A, "efac", B, "fbde", 0.0, C1, "abcd")
    torch.cuda.synchronize()
    bound = oracle.error_bound(level, e * e, 1.0, 1.0)
    assert float((C1 - C0).abs().max()) <= bound
    rng = np.random.default_rng(1)
    idx = rng.integers(0, e, size=(4096, 4))
    An, Bn, Cn = A.cpu().numpy(), B.cpu().numpy(), C1.cpu().numpy()
    for a, b, c, d in idx[:512]:
        exact = np.sum(An[:, :, a, c] * Bn[:, b, d, :].T)
        assert abs(Cn[a, b, c, d] - exact) <= bound
