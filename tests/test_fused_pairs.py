"""The element-pair form of the fused no-workspace ABC kernel.

CPU tests (no GPU): the host planner (tblis_stra_fused_pairs_query) decides
where the unit-stride mode of A and of B is a contracted mode, so that tiles
can be staged as contiguous 16-byte k pairs, and picks the shared-memory
layout and the consumers' lane tables.  A ring slot holds tb = 16 k of up to
2 blocks per operand (levels 0 and 1) or tb = 8 k of up to 4 blocks (level 2,
whose operand sums have up to 4 blocks).  The tests replay the kernel's
address arithmetic on those tables -- tile row r at tb r doubles, the slot's
tb k at the planned row positions, the swizzle of the chosen span (16-byte
chunk bits XOR the row bits above bit 7), fragment rows and columns permuted
by sigA/sigB -- and check that
  * in every MMA step both operands' lanes take the same k, and the tb k of a
    slot are each taken once per fragment row and column;
  * every read lands on the fragment row (column) the epilogue writes back;
  * every producer copy lands where the consumers read that element;
  * no quarter warp (16-byte reads and copies) or half warp (8-byte reads)
    touches one bank at two addresses (the count the planner reports is 0).

GPU tests: parity of the kernel with the oracle (the plain-C restatement of
the reference's contraction, src/internal/3t/mult.cxx:100-165) on layouts the
planner accepts -- the headline contraction's (C(abcd) += A(efac) B(fbde)),
a transposed GEMM whose B is read in pairs, ragged extents whose last rows
and k lie past the tensors (read as zero) and a batched case, at levels 0, 1
and 2 -- with the
kernel-timing record confirming which producer ran (tensor-map boxes where
tile rows are 128-byte runs, 16-byte pair copies elsewhere).
"""
import numpy as np
import pytest

from oracle import oracle


def _view(shape, lead=None):
    """A column-major host array of this shape (leading extent padded to
    `lead`) that is never read (planning only)."""
    st, acc = [], 8
    for d, n in enumerate(shape):
        st.append(acc)
        acc *= (lead if d == 0 and lead else n)
    return np.lib.stride_tricks.as_strided(np.zeros(1), tuple(shape), tuple(st))


def _query(tsb, level, ia, ib, ic, ext, lead=None):
    A = _view([ext[c] for c in ia], lead)
    B = _view([ext[c] for c in ib], lead)
    C = _view([ext[c] for c in ic])
    return tsb.fused_pairs_query(level, A, ia, B, ib, C, ic)


# (level, idx_A, idx_B, idx_C, extents, padded leading extent of A and B, producer)
ACCEPTED = [
    # the headline contraction's layout (k modes contiguous in different
    # operands, 32-byte runs): pair copies
    (0, "efac", "fbde", "abcd", dict(a=64, b=64, c=64, d=64, e=64, f=64), None, "pairs"),
    (1, "efac", "fbde", "abcd", dict(a=64, b=64, c=64, d=64, e=64, f=64), None, "pairs"),
    (1, "efac", "fbde", "abcd", dict(a=128, b=128, c=128, d=128, e=128, f=128), None, "pairs"),
    (1, "efac", "fbde", "abcd", dict(a=9, b=7, c=10, d=5, e=8, f=12), None, "pairs"),
    # k-major GEMM operands: 128-byte runs, tensor-map boxes (B read in pairs)
    (1, "ki", "kj", "ij", dict(i=512, j=256, k=512), None, "tma"),
    (0, "ki", "kj", "ij", dict(i=255, j=383, k=46), None, "tma"),
    (1, "ki", "kj", "ij", dict(i=255, j=255, k=63), 64, "tma"),
    # block rows of 150: not whole tiles, so pair copies
    (1, "ki", "kj", "ij", dict(i=300, j=200, k=64), None, "pairs"),
    # batch label in all three operands
    (1, "kib", "kjb", "ijb", dict(i=256, j=256, k=64, b=3), None, "tma"),
    # level 2: sums of up to 4 blocks, 8 k per slot, pair copies only
    (2, "efac", "fbde", "abcd", dict(a=64, b=64, c=64, d=64, e=64, f=64), None, "pairs"),
    (2, "efac", "fbde", "abcd", dict(a=9, b=7, c=10, d=5, e=8, f=12), None, "pairs"),
    (2, "efac", "fbde", "abcd", dict(a=9, b=7, c=10, d=5, e=4, f=16), None, "pairs"),
    (2, "ki", "kj", "ij", dict(i=512, j=512, k=512), None, "pairs"),
    (2, "ki", "kj", "ij", dict(i=255, j=255, k=127), 128, "pairs"),
    (2, "kib", "kjb", "ijb", dict(i=256, j=256, k=64, b=3), None, "pairs"),
]

REJECTED = [
    (1, "ik", "kj", "ij", dict(i=512, j=512, k=512), None, None),     # A's unit stride is a row mode
    (2, "ki", "kj", "ij", dict(i=256, j=256, k=48), None, None),     # k blocks of 12: not whole 8-k slots
    (1, "ki", "kj", "ij", dict(i=256, j=256, k=62), None, None),     # k blocks of 31: slots would straddle them
    (0, "ki", "kj", "ij", dict(i=256, j=256, k=47), None, None),     # odd column stride: pairs not 16-byte aligned
]


@pytest.mark.parametrize("case", ACCEPTED)
def test_planner_accepts_pair_tiles_conflict_free(tsb, case):
    level, ia, ib, ic, ext, lead, producer = case
    q = _query(tsb, level, ia, ib, ic, ext, lead)
    assert q["pairs"], case
    assert q["producer"] == producer
    assert q["tb"] == (8 if level == 2 else 16)
    assert q["conflicts"] == 0, q
    if producer == "tma":
        assert 1 <= q["rank_A"] <= 5 and 1 <= q["rank_B"] <= 5


@pytest.mark.parametrize("case", REJECTED)
def test_planner_rejects(tsb, case):
    level, ia, ib, ic, ext, lead, _ = case
    assert not _query(tsb, level, ia, ib, ic, ext, lead)["pairs"], case


def _swizzle(byte, span):
    """Swizzle of a tile aligned to its repeat: 16-byte chunk bits [4, 4+s)
    XOR bits [7, 7+s), s = log2(span / 16); its own inverse."""
    if span == 0:
        return byte
    s = {32: 1, 64: 2, 128: 3}[span]
    return byte ^ (((byte >> 7) & ((1 << s) - 1)) << 4)


def _decode(off, koff, span, tb):
    """(row, slot k) of the double at offset `off` (doubles) of a tile whose
    rows hold tb doubles."""
    u = _swizzle(off * 8, span) // 8
    row, pos = divmod(u, tb)
    return row, koff.index(pos)


def _replay(q):
    """The consumer's reads, as the kernel computes them (lane offsets of a
    warp at tile row and column 0).  Returns, per lane (g, t4), the list over
    steps of (kA, kB), and the offsets read by A's and B's loads grouped by
    instruction."""
    tb = q["tb"]
    assert sorted(q["koffA"]) == list(range(tb)) and sorted(q["koffB"]) == list(range(tb))
    sa_of, sb_of = q["sigA"], q["sigB"]
    assert sorted(sa_of) == list(range(8)) and sorted(sb_of) == list(range(8))
    steps, a_reads, b_reads = {}, {}, {}
    for lane in range(32):
        g = lane >> 2
        seq = []
        for qq in range(tb // 8):
            ao = q["aoff"][lane][qq]
            assert ao % 2 == 0                      # 16-byte aligned pair
            a_reads.setdefault(qq, []).append((lane, ao))
            for jj in range(2):
                ra, ka = _decode(ao + jj, q["koffA"], q["swz_A"], tb)
                assert ra == sa_of[g]
                if q["b_pairs"]:
                    bo = q["boff"][lane][2 * qq]
                    assert bo % 2 == 0
                    if jj == 0:
                        b_reads.setdefault(qq, []).append((lane, bo))
                    rb, kb = _decode(bo + jj, q["koffB"], q["swz_B"], tb)
                else:
                    bo = q["boff"][lane][2 * qq + jj]
                    b_reads.setdefault(2 * qq + jj, []).append((lane, bo))
                    rb, kb = _decode(bo, q["koffB"], q["swz_B"], tb)
                assert rb == sb_of[g]
                seq.append((ka, kb))
        steps[(g, lane & 3)] = seq
    return steps, a_reads, b_reads


def _bank_conflicts(reads, width, phase_lanes):
    """Sum over instructions and phases of (most distinct addresses on one
    4-byte bank) - 1; offsets in doubles."""
    total = 0
    for group in reads.values():
        by_lane = dict(group)
        for start in range(0, 32, phase_lanes):
            banks = {}
            for lane in range(start, start + phase_lanes):
                if lane not in by_lane:
                    continue
                word = by_lane[lane] * 2
                for w in range(width // 4):
                    banks.setdefault((word + w) % 32, set()).add(word + w)
            total += max(len(v) for v in banks.values()) - 1
    return total


def check_lane_tables(q):
    """The consumers' reads of a plan: both operands take the same k in every
    MMA step, each row (column) g takes the slot's tb k once over its tb / 4
    steps, and no quarter (half) warp hits one bank at two addresses."""
    steps, a_reads, b_reads = _replay(q)
    for (g, t4), seq in steps.items():
        for kA, kB in seq:
            assert kA == kB, (g, t4, seq)
    # each MMA step sums over the 4 lanes t4 of a row g; over its tb / 4
    # steps the tb k of the slot are each taken once
    tb = q["tb"]
    for g in range(8):
        ks = [steps[(g, t4)][s][0] for t4 in range(4) for s in range(tb // 4)]
        assert sorted(ks) == list(range(tb)), (g, ks)
    assert _bank_conflicts(a_reads, 16, 8) == 0
    assert _bank_conflicts(b_reads, 16 if q["b_pairs"] else 8, 8 if q["b_pairs"] else 16) == 0


def check_producer_copies(q):
    """The pair producer of a plan: with P = tb / 2 pairs per tile row,
    thread (warp w, lane l) copies pair pbase[l % P] of tile rows (32 / P) w +
    l / P + (128 / P) i to swizzle((koff + tb r) * 8) / 8.  Every element of
    the tile is written once, the pair's second element (its k with the pair
    bit set) lands 8 bytes after the first, and a quarter warp's 8 copies hit
    8 different 16-byte bank groups."""
    tb = q["tb"]
    P = tb // 2
    rpw, rpp = 32 // P, 4 * 32 // P
    for op in "AB":
        koff, span, bit, pbase = q["koff" + op], q["swz_" + op], q["bit_" + op], q["pbase" + op]
        assert len(pbase) == P
        assert sorted(pbase + [k | (1 << bit) for k in pbase]) == list(range(tb))
        written = {}
        for warp in range(4):
            for lane in range(32):
                kp, r0 = lane % P, warp * rpw + lane // P
                kl = pbase[kp]
                assert not (kl >> bit) & 1
                d0 = (_swizzle((koff[kl] + tb * (r0 & 7)) * 8, span) >> 3) + tb * (r0 & ~7)
                for i in range(128 // rpp):
                    off = d0 + rpp * tb * i
                    assert off % 2 == 0
                    for half, k in ((0, kl), (1, kl | (1 << bit))):
                        assert _decode(off + half, koff, span, tb) == (r0 + rpp * i, k)
                        assert off + half not in written
                        written[off + half] = True
        assert len(written) == 128 * tb
        # quarter warps of one copy instruction: 8 consecutive lanes cover
        # 8 / P rows
        for quarter in range(4 * 4):
            units = set()
            for lane in range(8 * (quarter % 4), 8 * (quarter % 4) + 8):
                kp, r = lane % P, (quarter // 4) * rpw + lane // P
                units.add((_swizzle((koff[pbase[kp]] + tb * (r & 7)) * 8, span) >> 4) & 7)
            assert len(units) == 8


@pytest.mark.parametrize("case", ACCEPTED)
def test_lane_tables_pair_the_same_k_and_cover_the_slot(tsb, case):
    level, ia, ib, ic, ext, lead, _ = case
    check_lane_tables(_query(tsb, level, ia, ib, ic, ext, lead))


@pytest.mark.parametrize("case", ACCEPTED)
def test_producer_copies_land_where_consumers_read(tsb, case):
    level, ia, ib, ic, ext, lead, producer = case
    if producer != "pairs":
        pytest.skip("tiles copied as tensor-map boxes")
    check_producer_copies(_query(tsb, level, ia, ib, ic, ext, lead))


# ------------------------------------------------------------------ GPU parity

def _dev(torch, x, dev):
    t = torch.empty_strided(x.shape, [s // 8 for s in x.strides], dtype=torch.float64, device=dev)
    t.copy_(torch.from_numpy(x))
    return t


# (level, alpha, beta, idx_A, idx_B, idx_C, extents, padded leading extent of A and B)
GPU_CASES = [
    (1, -0.5, 0.25, "ki", "kj", "ij", dict(i=512, j=256, k=512), None),
    (0, 1.5, 0.0, "ki", "kj", "ij", dict(i=255, j=383, k=46), None),
    (0, 1.0, 1.0, "efac", "fbde", "abcd", dict(a=32, b=16, c=32, d=32, e=16, f=8), None),
    (1, 1.0, 1.0, "efac", "fbde", "abcd", dict(a=32, b=16, c=32, d=32, e=16, f=8), None),
    (1, 1.5, 0.5, "efac", "fbde", "abcd", dict(a=9, b=7, c=10, d=5, e=8, f=12), None),
    # the last row, column and k of the second blocks lie past the tensors
    (1, 1.0, -1.0, "ki", "kj", "ij", dict(i=255, j=255, k=63), 64),
    (1, 1.0, 1.0, "ki", "kj", "ij", dict(i=300, j=200, k=64), None),
    (1, 2.0, 0.5, "kib", "kjb", "ijb", dict(i=256, j=256, k=64, b=3), None),
    # level 2: sums of up to 4 blocks per operand, 8 k per slot
    (2, 1.0, 1.0, "efac", "fbde", "abcd", dict(a=32, b=16, c=32, d=32, e=16, f=8), None),
    (2, 1.5, 0.5, "efac", "fbde", "abcd", dict(a=9, b=7, c=10, d=5, e=8, f=12), None),
    (2, -0.5, 0.25, "ki", "kj", "ij", dict(i=512, j=256, k=512), None),
    (2, 1.0, -1.0, "ki", "kj", "ij", dict(i=255, j=255, k=127), 128),
    (2, 2.0, 0.5, "kib", "kjb", "ijb", dict(i=256, j=256, k=64, b=3), None),
]


def _operand(shape, seed, lead):
    if not lead:
        return oracle.uniform(shape, seed)
    full = oracle.uniform([lead] + list(shape[1:]), seed)
    return full[: shape[0]]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GPU_CASES)
def test_pair_kernel_matches_oracle(tsb, cuda, case):
    import torch
    level, alpha, beta, ia, ib, ic, ext, lead = case
    q = _query(tsb, level, ia, ib, ic, ext, lead)
    assert q["pairs"]
    kind = "fused_pairs" if q["producer"] == "pairs" else "fused_tma"
    i = GPU_CASES.index(case)
    A = _operand([ext[c] for c in ia], 300 + 3 * i, lead)
    B = _operand([ext[c] for c in ib], 301 + 3 * i, lead)
    C0 = oracle.uniform([ext[c] for c in ic], 302 + 3 * i)
    ref = C0.copy(order="F")
    oracle.contract(alpha, A, ia, B, ib, beta, ref, ic)
    dA, dB, dC = _dev(torch, A, cuda), _dev(torch, B, cuda), _dev(torch, C0, cuda)
    tsb.set_workspace_limit(0)
    tsb.set_kernel_timing(True)
    try:
        tsb.contract(level, alpha, dA, ia, dB, ib, beta, dC, ic)
        torch.cuda.synchronize()
        launches, _ = tsb.kernel_timing(kind)
    finally:
        tsb.set_kernel_timing(False)
        tsb.set_workspace_limit(None)
    assert launches == 1
    k = int(np.prod([v for c, v in ext.items() if c in ia and c in ib and c not in ic]))
    bound = (oracle.error_bound(level, k, float(np.abs(A).max()), float(np.abs(B).max())) * abs(alpha)
             + 4 * 2.0 ** -53 * abs(beta) * float(np.abs(C0).max()))
    err = float(np.abs(dC.cpu().numpy() - ref).max())
    assert err <= bound, (case, err, bound)


@pytest.mark.gpu
@pytest.mark.parametrize("level", [1, 2])
def test_pair_kernel_noalloc_entry_point(tsb, cuda, level):
    """The allocation-free entry point reaches the same kernel."""
    import torch
    ia, ib, ic = "efac", "fbde", "abcd"
    ext = dict(a=32, b=16, c=32, d=32, e=16, f=8)
    A = oracle.uniform([ext[c] for c in ia], 401)
    B = oracle.uniform([ext[c] for c in ib], 402)
    ref = np.zeros([ext[c] for c in ic], order="F")
    oracle.contract(1.0, A, ia, B, ib, 0.0, ref, ic)
    dA, dB = _dev(torch, A, cuda), _dev(torch, B, cuda)
    dC = torch.zeros_like(_dev(torch, ref, cuda))
    tsb.set_kernel_timing(True)
    try:
        tsb.noalloc_mult(level, 1.0, dA, ia, dB, ib, 0.0, dC, ic)
        torch.cuda.synchronize()
        launches, _ = tsb.kernel_timing("fused_pairs")
    finally:
        tsb.set_kernel_timing(False)
    assert launches == 1
    bound = oracle.error_bound(level, 16 * 8, float(np.abs(A).max()), float(np.abs(B).max()))
    assert float(np.abs(dC.cpu().numpy() - ref).max()) <= bound
