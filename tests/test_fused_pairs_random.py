"""Randomised coverage of the element-pair form of the no-workspace ABC
kernel, beside the hand-picked layouts of test_fused_pairs.py.

CPU (no GPU): seeded random contractions -- one or two modes in each of the
row, column and contracted bundles, every operand's modes in a random order
(column-major storage), extents from 1 to 40 with odd and ragged ones among
them -- planned at Strassen levels 0, 1 and 2.  Every plan the planner
accepts is replayed: both operands take the same k in every MMA step, every
slot k is taken once per fragment row and column, no quarter or half warp
touches one bank at two addresses, and every producer copy lands where the
consumers read that element.

GPU: a seeded sample of such contractions run with no workspace (whichever
no-workspace kernel takes them) against the oracle, the plain-C restatement
of the reference's contraction (src/internal/3t/mult.cxx:100-165), with
random alpha and beta.
"""
import os
import sys

import numpy as np
import pytest

from oracle import oracle

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_fused_pairs import _dev, _query, check_lane_tables, check_producer_copies  # noqa: E402

EXTENTS = [1, 2, 3, 4, 5, 6, 7, 8, 12, 16, 24, 31, 32, 40]


def random_case(rng, extents=EXTENTS):
    """(idx_A, idx_B, idx_C, extents) of a random contraction."""
    letters = iter("abcdefghjkmnpq")
    rows = [next(letters) for _ in range(int(rng.integers(1, 3)))]
    cols = [next(letters) for _ in range(int(rng.integers(1, 3)))]
    ks = [next(letters) for _ in range(int(rng.integers(1, 3)))]
    ext = {c: int(rng.choice(extents)) for c in rows + cols + ks}
    ia, ib, ic = list(rows + ks), list(ks + cols), list(rows + cols)
    rng.shuffle(ia)
    rng.shuffle(ib)
    rng.shuffle(ic)
    return "".join(ia), "".join(ib), "".join(ic), ext


def test_random_layouts_plan_consistently(tsb):
    rng = np.random.default_rng(20261204)
    accepted = {0: 0, 1: 0, 2: 0}
    for _ in range(800):
        ia, ib, ic, ext = random_case(rng)
        for level in (0, 1, 2):
            q = _query(tsb, level, ia, ib, ic, ext)
            if not q["pairs"]:
                continue
            accepted[level] += 1
            case = (level, ia, ib, ic, ext)
            assert q["conflicts"] == 0, case
            assert q["tb"] == (8 if level == 2 else 16), case
            try:
                check_lane_tables(q)
                if q["producer"] == "pairs":
                    check_producer_copies(q)
            except AssertionError as e:
                raise AssertionError(f"{case}: {e}") from e
    # the generator reaches the element-pair form at every level
    assert min(accepted.values()) >= 20, accepted


def _gpu_cases():
    rng = np.random.default_rng(7)
    out = []
    while len(out) < 24:
        ia, ib, ic, ext = random_case(rng, [2, 3, 4, 6, 8, 12, 16, 24, 31, 32, 40])
        size = lambda idx: int(np.prod([ext[c] for c in idx]))
        if max(size(ia), size(ib), size(ic)) > 200_000:
            continue
        level = int(rng.integers(0, 3))
        alpha = float(rng.choice([1.0, -0.5, 2.0]))
        beta = float(rng.choice([0.0, 1.0, -1.5]))
        out.append((level, alpha, beta, ia, ib, ic, ext))
    return out


GPU_CASES = _gpu_cases()


@pytest.mark.gpu
@pytest.mark.parametrize("case", GPU_CASES, ids=[f"{c[0]}-{c[3]}-{c[4]}-{c[5]}" for c in GPU_CASES])
def test_random_no_workspace_matches_oracle(tsb, cuda, case):
    import torch
    level, alpha, beta, ia, ib, ic, ext = case
    i = GPU_CASES.index(case)
    A = oracle.uniform([ext[c] for c in ia], 500 + 3 * i)
    B = oracle.uniform([ext[c] for c in ib], 501 + 3 * i)
    C0 = oracle.uniform([ext[c] for c in ic], 502 + 3 * i)
    ref = C0.copy(order="F")
    oracle.contract(alpha, A, ia, B, ib, beta, ref, ic)
    dA, dB, dC = _dev(torch, A, cuda), _dev(torch, B, cuda), _dev(torch, C0, cuda)
    tsb.set_workspace_limit(0)
    try:
        tsb.contract(level, alpha, dA, ia, dB, ib, beta, dC, ic)
        torch.cuda.synchronize()
    finally:
        tsb.set_workspace_limit(None)
    k = int(np.prod([ext[c] for c in ia if c in ib]))
    bound = (oracle.error_bound(level, k, float(np.abs(A).max()), float(np.abs(B).max())) * abs(alpha)
             + 4 * 2.0 ** -53 * abs(beta) * float(np.abs(C0).max()))
    err = float(np.abs(dC.cpu().numpy() - ref).max())
    assert err <= bound, (case, err, bound)
