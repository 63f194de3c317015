"""The oracle pinned against the reference: golden fixtures made by the
reference itself (tests/golden/make_golden.py) and, where the reference
library is built here, live comparison on fresh inputs."""
import json
import os

import numpy as np
import pytest

from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "manifest.json")) as f:
    MANIFEST = json.load(f)


def bound(level, k, A, B):
    return oracle.error_bound(level, max(k, 1), np.abs(A).max(), np.abs(B).max())


@pytest.mark.parametrize("case", MANIFEST, ids=[c["name"] for c in MANIFEST])
def test_oracle_matches_golden(case):
    d = np.load(os.path.join(GOLDEN, case["name"] + ".npz"))
    A, B, C0 = (np.asfortranarray(d[x]) for x in ("A", "B", "C0"))
    C = C0.copy(order="F")
    oracle.contract(case["alpha"], A, case["idx_A"], B, case["idx_B"], case["beta"], C, case["idx_C"])
    # the summed extent of the k bundle and of labels only in A or only in B
    ext = case["extents"]
    ksum = int(np.prod([ext[c] for c in ext if c not in case["idx_C"]])) if ext else 1
    for out in case["outputs"]:
        level = int(out[1])
        tol = bound(level, ksum, A, B) * max(1.0, abs(case["alpha"])) + 1e-300
        err = np.abs(C - d[out]).max()
        assert err <= tol, (out, err, tol)


def test_strassen_schedule_restatement():
    rng = np.random.default_rng(0)
    for level in (1, 2):
        A = rng.uniform(-1, 1, (32, 24))
        B = rng.uniform(-1, 1, (24, 40))
        assert np.abs(oracle.strassen_matmul(A, B, level) - A @ B).max() < 1e-12


def test_level2_coeffs_are_kronecker_square():
    U2, V2, W2 = oracle.level_coeffs(2)
    assert U2.shape == (16, 49)
    # each column of a level-2 coefficient matrix has nnz = product of level-1 nnz
    nnzU = (oracle.U != 0).sum(0)
    assert sorted((U2 != 0).sum(0)) == sorted(int(a * b) for a in nnzU for b in nnzU)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_matches_live_reference(seed):
    rng = np.random.default_rng(seed)
    ext = dict(a=int(rng.integers(2, 9)), b=int(rng.integers(2, 9)), c=4, d=6, e=int(rng.integers(2, 9)), f=4)
    ic, ia, ib = "abcd", "efac", "fbde"
    A = oracle.uniform([ext[c] for c in ia], seed)
    B = oracle.uniform([ext[c] for c in ib], seed + 1)
    C0 = oracle.uniform([ext[c] for c in ic], seed + 2)
    for beta in (0.0, 0.5, 1.0):
        Cr = C0.copy(order="F")
        Co = C0.copy(order="F")
        oracle.ref_mult(0, 1, 1.5, A, ia, B, ib, beta, Cr, ic)
        oracle.contract(1.5, A, ia, B, ib, beta, Co, ic)
        assert np.abs(Cr - Co).max() <= 1.5 * bound(0, ext["e"] * ext["f"], A, B)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_reference_strassen_beta_quirk_documented():
    """The reference's L=1 ABC applies beta inside every product
    (src/stra_internal/3t/stra_mult.cxx:441-443), so it is exact only for
    beta == 1.  The oracle (and this library) apply beta once."""
    ext = dict(a=4, b=4, c=4, d=4, e=4, f=4)
    A = oracle.uniform([4] * 4, 7)
    B = oracle.uniform([4] * 4, 8)
    C0 = oracle.uniform([4] * 4, 9)
    Cr = C0.copy(order="F")
    Co = C0.copy(order="F")
    oracle.ref_mult(1, 1, 1.0, A, "efac", B, "fbde", 0.0, Cr, "abcd")
    oracle.contract(1.0, A, "efac", B, "fbde", 0.0, Co, "abcd")
    assert np.abs(Cr - Co).max() > 1e-3
