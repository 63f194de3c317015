"""Host logic of the library without a GPU: the bundle analysis behind
tblis_stra_plan_query must reduce every contraction to a batched product whose
scatter vectors reproduce the oracle's result."""
import numpy as np
import pytest

from oracle import oracle


def from_plan(plan, alpha, A, B, beta, C):
    """Evaluate C = alpha*A*B + beta*C in numpy through the plan's scatter vectors."""
    import ctypes

    class Flat:
        # element-offset addressing relative to the data pointer (offsets may be negative)
        def __init__(self, X):
            es = X.itemsize
            lo = sum(min(0, (n - 1) * s // es) for n, s in zip(X.shape, X.strides))
            hi = sum(max(0, (n - 1) * s // es) for n, s in zip(X.shape, X.strides))
            buf = (ctypes.c_double * (hi - lo + 1)).from_address(X.ctypes.data + lo * es)
            self.a, self.lo = np.frombuffer(buf, dtype=np.float64), lo

        def __getitem__(self, off):
            return self.a[off - self.lo]

        def __setitem__(self, off, v):
            self.a[off - self.lo] = v

    fa, fb, fc = Flat(A), Flat(B), Flat(C)
    m, n, k, nb = plan["m"], plan["n"], plan["k"], plan["batch"]
    for bi in range(nb):
        Am = fa[plan["bA"][bi] + plan["rsA"][:, None] + plan["ksA"][None, :]] if k else np.zeros((m, 0))
        Bm = fb[plan["bB"][bi] + plan["ksB"][:, None] + plan["csB"][None, :]] if k else np.zeros((0, n))
        idx = plan["bC"][bi] + plan["rsC"][:, None] + plan["csC"][None, :]
        Cm = fc[idx]
        val = alpha * (Am @ Bm)
        fc[idx] = val if beta == 0 else val + beta * Cm


CASES = [
    ("abcd", "efac", "fbde", dict(a=4, b=3, c=5, d=2, e=3, f=4)),       # config-1 pattern
    ("abc", "dca", "db", dict(a=4, b=8, c=2, d=8)),                      # example.txt shape
    ("ij", "ik", "kj", dict(i=7, j=5, k=6)),
    ("abz", "akz", "kbz", dict(a=3, b=4, k=5, z=3)),                     # batch
    ("abx", "aky", "kbw", dict(a=3, b=2, k=4, x=2, y=3, w=2)),           # A-, B-, C-only
    ("ab", "aakb", "kb", dict(a=4, b=3, k=5)),                           # diagonal in A
    ("aab", "ak", "kb", dict(a=3, b=4, k=2)),                            # diagonal in C
    ("ab", "a", "b", dict(a=5, b=6)),                                    # outer product
    ("", "ab", "ab", dict(a=5, b=6)),                                    # full contraction to a scalar
    ("abc", "ab", "bc", dict(a=3, b=1, c=4)),                            # extent-1 mode dropped
]


@pytest.mark.parametrize("ic,ia,ib,ext", CASES, ids=[c[0] + "=" + c[1] + "*" + c[2] for c in CASES])
@pytest.mark.parametrize("order", ["F", "C"])
def test_plan_reproduces_oracle(tsb, ic, ia, ib, ext, order):
    A = oracle.uniform([ext[c] for c in ia] or [], 1, order)
    B = oracle.uniform([ext[c] for c in ib] or [], 2, order)
    C0 = oracle.uniform([ext[c] for c in ic] or [], 3, order)
    for alpha, beta in ((1.0, 0.0), (1.5, 0.5)):
        plan = tsb.plan_query(A, ia, B, ib, C0, ic)
        Cp = C0.copy(order="K")
        from_plan(plan, alpha, A, B, beta, Cp)
        Co = C0.copy(order="K")
        oracle.contract(alpha, A, ia, B, ib, beta, Co, ic)
        np.testing.assert_allclose(Cp, Co, rtol=1e-12, atol=1e-12)


def test_fold_merges_contiguous_modes(tsb):
    # C(a,b,c,d) = A(a,b,e,f) B(e,f,c,d), column-major: (a,b), (e,f), (c,d) all fold
    A = np.zeros((4, 3, 5, 2), order="F"); B = np.zeros((5, 2, 6, 7), order="F"); C = np.zeros((4, 3, 6, 7), order="F")
    p = tsb.plan_query(A, "abef", B, "efcd", C, "abcd", scatter=True)
    assert (p["m"], p["n"], p["k"], p["batch"]) == (12, 42, 10, 1)
    assert np.array_equal(p["rsA"], np.arange(12))          # folded: unit stride over all of m
    assert np.array_equal(p["ksB"], np.arange(10))


def test_config1_does_not_fold(tsb):
    ext = 8
    A = np.zeros((ext,) * 4, order="F"); B = np.zeros((ext,) * 4, order="F"); C = np.zeros((ext,) * 4, order="F")
    p = tsb.plan_query(A, "efac", B, "fbde", C, "abcd")
    assert (p["m"], p["n"], p["k"]) == (64, 64, 64)
    # A rows (a,c): strides 64, 4096/... uniform in A, not in C
    assert np.all(np.diff(p["rsA"]) == ext * ext)
    assert len(set(np.diff(p["rsC"]))) == 2


@pytest.mark.parametrize("bad", ["extent", "type", "conj"])
def test_plan_errors(tsb, bad):
    A = np.zeros((3, 4)); B = np.zeros((4, 5)); C = np.zeros((3, 5))
    if bad == "extent":
        B = np.zeros((6, 5))
        code = 3
    elif bad == "type":
        B = np.zeros((4, 5), dtype=np.float32)
        code = 2
    else:
        va = tsb.tblis_stra._View(A, 1.0)
        vb = tsb.tblis_stra._View(B, 1.0)
        vc = tsb.tblis_stra._View(C, 0.0)
        va.t.conj = 1
        import ctypes
        st = tsb.lib.tblis_stra_plan_query(ctypes.byref(va.t), b"ik", ctypes.byref(vb.t), b"kj",
                                           ctypes.byref(vc.t), b"ij", None, None, *([None] * 9))
        assert st == 4
        return
    with pytest.raises(tsb.TblisStraError) as e:
        tsb.plan_query(A, "ik", B, "kj", C, "ij")
    assert e.value.status == code


def test_negative_strides(tsb):
    A = oracle.uniform((5, 6), 4)[::-1, :]
    B = oracle.uniform((6, 7), 5)[:, ::-1]
    C = np.zeros((5, 7))
    p = tsb.plan_query(A, "ik", B, "kj", C, "ij")
    Cp = C.copy()
    from_plan(p, 1.0, A, B, 0.0, Cp)
    np.testing.assert_allclose(Cp, A @ B, rtol=1e-12, atol=1e-12)
