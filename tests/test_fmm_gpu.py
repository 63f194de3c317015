"""Fast matrix-multiplication families on the GPU (tblis_stra_set_algorithm):
the classical <2,2,2;8>, Strassen beside classical products for <3,2,2>,
<2,3,2> and <2,2,3> (11 products), and a registered algorithm (Strassen's
coefficients with its products reordered), through the FP64 ABC variant in
both of its forms (operand sums packed product by product; the fused kernel
with no workspace), against the oracle within the FP64 bound."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

CASES = [
    ("efac", "fbde", "abcd", dict(a=9, b=7, c=6, d=5, e=8, f=7)),      # ragged: 54 x 35 x 56
    ("ik", "kj", "ij", dict(i=300, j=257, k=190)),
    ("bik", "bkj", "bij", dict(b=2, i=64, j=96, k=48)),
]


def _dev(torch, x, dev):
    t = torch.empty_strided(x.shape, [s // 8 for s in x.strides], dtype=torch.float64, device=dev)
    t.copy_(torch.from_numpy(x))
    return t


@pytest.fixture(params=["packed", "fused"])
def form(request, tsb):
    tsb.set_workspace_limit(None if request.param == "packed" else 0)
    yield request.param
    tsb.set_workspace_limit(None)


@pytest.mark.parametrize("alg", [1, 2, 3, 4, "registered"])
def test_family_matches_oracle(tsb, cuda, form, alg):
    import torch
    if alg == "registered":
        perm = [3, 0, 6, 1, 5, 2, 4]
        alg = tsb.register_algorithm(2, 2, 2, *(X[:, perm] for X in (oracle.U, oracle.V, oracle.W)))
    levels = tsb.algorithm_info(alg)["levels"]
    tsb.set_algorithm(alg)
    try:
        for i, (ia, ib, ic, ext) in enumerate(CASES):
            A = oracle.uniform([ext[c] for c in ia], 60 + i)
            B = oracle.uniform([ext[c] for c in ib], 70 + i)
            C0 = oracle.uniform([ext[c] for c in ic], 80 + i)
            ref = C0.copy(order="F")
            oracle.contract(1.25, A, ia, B, ib, 0.5, ref, ic)
            k = int(np.prod([v for c, v in ext.items() if c in ia and c in ib and c not in ic]))
            for level in range(1, levels + 1):
                C = _dev(torch, C0, cuda)
                tsb.contract(level, 1.25, _dev(torch, A, cuda), ia, _dev(torch, B, cuda), ib, 0.5, C, ic)
                torch.cuda.synchronize()
                bound = 1.25 * oracle.error_bound(level, k, 1.0, 1.0) + 4 * 2.0 ** -53 * 0.5
                err = float(np.abs(C.cpu().numpy() - ref).max())
                assert err <= bound, (alg, form, i, level, err, bound)
    finally:
        tsb.set_algorithm(0)


def test_family_limits(tsb, cuda):
    """Other algorithms than Strassen run FP64 ABC only; level 2 of an
    11-product family has 121 products, beyond the kernels' 49."""
    import torch
    A = torch.rand(64, 64, dtype=torch.float64, device=cuda)
    C = torch.zeros(64, 64, dtype=torch.float64, device=cuda)
    tsb.set_algorithm(4)
    try:
        for kw in (dict(level=1, impl=2), dict(level=1, impl=3), dict(level=2, impl=1)):
            with pytest.raises(tsb.TblisStraError) as ei:
                tsb.contract(kw["level"], 1.0, A, "ik", A, "kj", 0.0, C, "ij", impl=kw["impl"])
            assert ei.value.status == 9
        with pytest.raises(tsb.TblisStraError) as ei:
            tsb.contract(1, 1.0, A.float(), "ik", A.float(), "kj", 0.0, C.float(), "ij")
        assert ei.value.status == 9
        tsb.contract(0, 1.0, A, "ik", A, "kj", 0.0, C, "ij")       # level 0 ignores the algorithm
        torch.cuda.synchronize()
        assert torch.allclose(C, A @ A, atol=1e-12, rtol=0)
    finally:
        tsb.set_algorithm(0)
