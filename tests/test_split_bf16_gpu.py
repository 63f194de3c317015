"""Precision form: FP32 contractions on the BF16 tensor cores (tcgen05) with
each operand sum split into bf16 planes, checked against the FP64 oracle on
the same FP32 values (normwise error ||C - Cref||_F / ||Cref||_F):

  6 terms (hi/mid/lo: hh, hm, mh, hl, mm, lh):  <= 1e-6
  3 terms (hi/mid:    hh, hm, mh):              <= 6e-5

for entries uniform in [-1, 1] and log-uniform magnitudes in [1e-3, 1e3] with
random sign, at Strassen levels 0, 1, 2."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

TOL = {6: 1e-6, 3: 6e-5}


def draw(shape, seed, dist):
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    if dist == "uniform":
        x = rng.uniform(-1, 1, n)
    else:
        x = np.sign(rng.uniform(-1, 1, n)) * 10.0 ** rng.uniform(-3, 3, n)
    return np.asfortranarray(x.reshape(shape, order="F").astype(np.float32))


def to_dev(x, cuda):
    import torch
    out = torch.empty_strided(x.shape, [s // x.itemsize for s in x.strides], dtype=torch.float32, device=cuda)
    out.copy_(torch.from_numpy(x))
    return out


def normwise(C, R):
    d = np.linalg.norm((C.astype(np.float64) - R).ravel())
    r = np.linalg.norm(R.ravel())
    return d / r if r else d


@pytest.fixture(params=[6, 3])
def terms(request, tsb):
    tsb.set_fp32_terms(request.param)
    yield request.param
    tsb.set_fp32_terms(6)


@pytest.fixture(params=["grouped", "parallel"])
def fp32_schedule(request, tsb):
    """L >= 1 runs each group of 7 products tile by tile in one GEMM launch
    (grouped), or every product side by side into M_p and one combine pass
    (parallel, the automatic choice for small grids)."""
    tsb.set_product_parallel(1 if request.param == "parallel" else 0)
    yield request.param
    tsb.set_product_parallel(-1)


@pytest.mark.parametrize("dist", ["uniform", "loguniform"])
@pytest.mark.parametrize("level", [0, 1, 2])
def test_fp32_4d_vs_fp64_oracle(tsb, cuda, terms, level, dist, fp32_schedule):
    import torch
    ext = dict(a=24, b=20, c=10, d=12, e=18, f=16)
    ia, ib, ic = "efac", "fbde", "abcd"
    A = draw([ext[c] for c in ia], 1, dist)
    B = draw([ext[c] for c in ib], 2, dist)
    C0 = draw([ext[c] for c in ic], 3, dist)
    R = C0.astype(np.float64, order="F")
    oracle.contract(1.5, A.astype(np.float64, order="F"), ia, B.astype(np.float64, order="F"), ib, 0.5, R, ic)
    dC = to_dev(C0, cuda)
    tsb.contract(level, 1.5, to_dev(A, cuda), ia, to_dev(B, cuda), ib, 0.5, dC, ic)
    torch.cuda.synchronize()
    err = normwise(dC.cpu().numpy(), R)
    assert err <= TOL[terms], err


@pytest.mark.parametrize("level", [0, 1, 2])
def test_fp32_ragged_batch_and_beta0(tsb, cuda, terms, level, fp32_schedule):
    import torch
    ext = dict(i=131, j=67, k=150, z=3)
    A = draw((ext["i"], ext["k"], ext["z"]), 4, "uniform")
    B = draw((ext["k"], ext["j"], ext["z"]), 5, "uniform")
    C0 = np.full((ext["i"], ext["j"], ext["z"]), np.nan, dtype=np.float32, order="F")
    R = np.zeros(C0.shape, order="F")
    oracle.contract(1.0, A.astype(np.float64, order="F"), "ikz", B.astype(np.float64, order="F"), "kjz", 0.0, R, "ijz")
    dC = to_dev(C0, cuda)
    tsb.contract(level, 1.0, to_dev(A, cuda), "ikz", to_dev(B, cuda), "kjz", 0.0, dC, "ijz")
    torch.cuda.synchronize()
    out = dC.cpu().numpy()
    assert np.isfinite(out).all()
    assert normwise(out, R) <= TOL[terms]


@pytest.mark.parametrize("level", [0, 1, 2])
def test_fp32_config1_size_vs_fp64_gpu(tsb, cuda, terms, level, fp32_schedule):
    """NIm = NJn = NPk = 4096 (extents 64): the FP64 GPU path (itself checked
    against the oracle bound) is the reference; log-uniform magnitudes."""
    import torch
    e = 64
    A = draw((e,) * 4, 7, "loguniform")
    B = draw((e,) * 4, 8, "loguniform")
    dA, dB = to_dev(A, cuda), to_dev(B, cuda)
    C32 = torch.zeros((e,) * 4, dtype=torch.float32, device=cuda)
    C64 = torch.zeros((e,) * 4, dtype=torch.float64, device=cuda)
    tsb.contract(level, 1.0, dA, "efac", dB, "fbde", 0.0, C32, "abcd")
    tsb.contract(0, 1.0, dA.double(), "efac", dB.double(), "fbde", 0.0, C64, "abcd")
    torch.cuda.synchronize()
    err = float(torch.linalg.norm((C32.double() - C64).flatten()) / torch.linalg.norm(C64.flatten()))
    assert err <= TOL[terms], err


def test_fp32_host_pointers(tsb, cuda):
    A = draw((40, 30), 9, "uniform")
    B = draw((30, 20), 10, "uniform")
    C = np.zeros((40, 20), dtype=np.float32, order="F")
    tsb.contract(1, 1.0, A, "ik", B, "kj", 0.0, C, "ij", drop_in=True)
    R = A.astype(np.float64) @ B.astype(np.float64)
    assert normwise(C, R) <= 1e-6


def fp32_single_product_bytes(tsb, level, A, ia, B, ib, C, ic, terms):
    """Workspace of the split path with one product's planes at a time
    (row scales + P planes of 128 x 64 bf16 blocks for S and T)."""
    q = tsb.plan_query(A, ia, B, ib, C, ic, scatter=False)
    H = 1 << level
    cdiv = lambda a, b: -(-a // b)
    ms, ns, ks = cdiv(q["m"], H), cdiv(q["n"], H), cdiv(q["k"], H)
    sc = cdiv(q["batch"] * (ms + ns) * 2 * 4, 256) * 256
    P = 2 if terms == 3 else 3
    return sc + P * q["batch"] * (cdiv(ms, 128) + cdiv(ns, 128)) * cdiv(ks, 64) * 128 * 64 * 2


@pytest.mark.parametrize("level", [1, 2])
def test_fp32_per_product_packing(tsb, cuda, terms, level):
    """With workspace for one product's planes only, the split sums are packed
    product by product instead of seven per pass: same bound."""
    import torch
    ext = dict(a=24, b=20, c=10, d=12, e=18, f=16)
    ia, ib, ic = "efac", "fbde", "abcd"
    A = draw([ext[c] for c in ia], 11, "loguniform")
    B = draw([ext[c] for c in ib], 12, "loguniform")
    C0 = draw([ext[c] for c in ic], 13, "uniform")
    R = C0.astype(np.float64, order="F")
    oracle.contract(1.0, A.astype(np.float64, order="F"), ia, B.astype(np.float64, order="F"), ib, 1.0, R, ic)
    dA, dB, dC = to_dev(A, cuda), to_dev(B, cuda), to_dev(C0, cuda)
    tsb.set_workspace_limit(fp32_single_product_bytes(tsb, level, dA, ia, dB, ib, dC, ic, terms))
    try:
        before = tsb.launch_count()
        tsb.contract(level, 1.0, dA, ia, dB, ib, 1.0, dC, ic)
        torch.cuda.synchronize()
        # 2 scale launches, then per product: pack S, pack T, GEMM
        assert tsb.launch_count() - before == 2 + 3 * 7 ** level
    finally:
        tsb.set_workspace_limit(None)
    err = normwise(dC.cpu().numpy(), R)
    assert err <= TOL[terms], err


@pytest.mark.parametrize("level", [1, 2])
def test_fp32_group_launches(tsb, cuda, terms, level):
    """With room for a group's planes, each group of 7 products takes one
    pass over A, one over B and one GEMM launch that runs the 7 products for
    each tile position; the result keeps the bound."""
    import torch
    ext = dict(a=24, b=20, c=10, d=12, e=18, f=16)
    ia, ib, ic = "efac", "fbde", "abcd"
    A = draw([ext[c] for c in ia], 14, "loguniform")
    B = draw([ext[c] for c in ib], 15, "loguniform")
    C0 = draw([ext[c] for c in ic], 16, "uniform")
    R = C0.astype(np.float64, order="F")
    oracle.contract(0.75, A.astype(np.float64, order="F"), ia, B.astype(np.float64, order="F"), ib, -0.5, R, ic)
    for mode, launches in ((0, 2 + 3 * 7 ** (level - 1)), (-1, 2 + 2 * 7 ** (level - 1) + 2)):
        # grouped: 2 scale launches, then per group pack 7 S, pack 7 T, GEMM;
        # automatic on this small grid (product-parallel): 2 scales, the
        # group packs, one GEMM over all products, the combine
        dA, dB, dC = to_dev(A, cuda), to_dev(B, cuda), to_dev(C0, cuda)
        tsb.set_product_parallel(mode)
        try:
            before = tsb.launch_count()
            tsb.contract(level, 0.75, dA, ia, dB, ib, -0.5, dC, ic)
            torch.cuda.synchronize()
            assert tsb.launch_count() - before == launches, mode
        finally:
            tsb.set_product_parallel(-1)
        err = normwise(dC.cpu().numpy(), R)
        assert err <= TOL[terms], (mode, err)


def test_fp32_ksplit_small_grid_large_k(tsb, cuda, terms):
    """L=0 with fewer C tiles than SMs and a long summed range: the split
    planes of 9 k pieces run side by side and the combine pass sums them in
    FP64 (batch label, beta = 0 over a NaN-filled C)."""
    import torch
    ext = dict(i=200, j=190, k=5000, z=2)
    A = draw((ext["i"], ext["k"], ext["z"]), 41, "loguniform")
    B = draw((ext["k"], ext["j"], ext["z"]), 42, "loguniform")
    C0 = np.full((ext["i"], ext["j"], ext["z"]), np.nan, dtype=np.float32, order="F")
    R = np.zeros(C0.shape, order="F")
    oracle.contract(1.0, A.astype(np.float64, order="F"), "ikz", B.astype(np.float64, order="F"), "kjz",
                    0.0, R, "ijz")
    dC = to_dev(C0, cuda)
    before = tsb.launch_count()
    tsb.contract(0, 1.0, to_dev(A, cuda), "ikz", to_dev(B, cuda), "kjz", 0.0, dC, "ijz")
    torch.cuda.synchronize()
    # 2 scales, one pack per operand (9 pieces), the GEMM over the pieces,
    # the combine
    assert tsb.launch_count() - before == 6
    out = dC.cpu().numpy()
    assert np.isfinite(out).all()
    assert normwise(out, R) <= TOL[terms]
