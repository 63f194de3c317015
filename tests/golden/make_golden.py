"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs only where the reference library has been compiled from its sources
(oracle/build_ref.sh -> oracle/_ref/libtblis_ref.so).  For every case it
draws seeded inputs (oracle.uniform: U[-1, 1], column-major), runs the
reference's own entry points -- tblis_tensor_mult (L=0) and, where the
reference's Strassen is valid (beta == 1 and every bundle product divisible by
2^L), stra_tblis_tensor_mult[_2level] with impl 1/2/3 -- and stores inputs and
outputs in <case>.npz plus a manifest.json.

Usage:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle  # noqa: E402

# (name, idx_C, idx_A, idx_B, extents, alpha, beta)
CASES = [
    # shape of the reference's bin/example.txt line "abc dca db"
    ("example", "abc", "dca", "db", dict(a=4, b=8, c=2, d=8), 1.0, 1.0),
    # config-1 pattern C(a,b,c,d) += A(e,f,a,c) B(f,b,d,e), reduced extents
    ("cfg1_e8", "abcd", "efac", "fbde", dict(a=8, b=8, c=8, d=8, e=8, f=8), 1.0, 1.0),
    ("cfg1_e6", "abcd", "efac", "fbde", dict(a=6, b=6, c=6, d=6, e=6, f=6), 1.0, 1.0),
    # shape-dependence pattern "abij abef efij" (bin/shape.txt), reduced extents
    ("shape_small", "abij", "abef", "efij", dict(a=8, b=8, e=12, f=4, i=6, j=10), 1.0, 1.0),
    # two indices per bundle with mixed orders
    ("perm_mixed", "dbca", "ceaf", "fbed", dict(a=12, b=4, c=4, d=8, e=8, f=6), 1.0, 1.0),
    # matrix product (one index per bundle)
    ("matrix", "ij", "ik", "kj", dict(i=32, j=24, k=40), 1.0, 1.0),
    # beta / alpha variants (reference Strassen valid only for beta == 1)
    ("beta0", "abcd", "efac", "fbde", dict(a=8, b=4, c=4, d=8, e=4, f=8), 1.0, 0.0),
    ("beta_half", "abcd", "efac", "fbde", dict(a=8, b=4, c=4, d=8, e=4, f=8), 2.0, 0.5),
    # ragged (odd) extents
    ("odd", "abcd", "efac", "fbde", dict(a=5, b=7, c=3, d=3, e=9, f=5), 1.0, 1.0),
    # batch index (in A, B and C) plus contracted and free indices
    ("batch", "abz", "akz", "kbz", dict(a=12, b=10, k=14, z=3), 1.0, 1.0),
    # indices only in A (summed), only in B (summed), only in C (broadcast)
    ("only_idx", "abx", "aky", "kbw", dict(a=6, b=4, k=8, x=3, y=2, w=3), 1.0, 0.5),
    # repeated label (diagonal) inside A
    ("diag", "ab", "aakb", "kb", dict(a=6, b=5, k=7), 1.0, 1.0),
]


def run_case(name, ic, ia, ib, ext, alpha, beta, seed):
    A = oracle.uniform([ext[c] for c in ia], seed)
    B = oracle.uniform([ext[c] for c in ib], seed + 1)
    C0 = oracle.uniform([ext[c] for c in ic], seed + 2)
    out = {}
    bad = run_case.bad = {}
    C = C0.copy(order="F")
    oracle.ref_mult(0, 1, alpha, A, ia, B, ib, beta, C, ic)
    out["L0"] = C
    prod = lambda s: int(np.prod([ext[c] for c in s])) if s else 1
    sa, sb, sc = set(ia), set(ib), set(ic)
    m = prod([c for c in ext if c in sa and c in sc and c not in sb])
    n = prod([c for c in ext if c in sb and c in sc and c not in sa])
    k = prod([c for c in ext if c in sa and c in sb and c not in sc])
    simple = all((c in sa) + (c in sb) + (c in sc) == 2 for c in ext) and len(set(ia)) == len(ia)
    for L in (1, 2):
        if beta != 1.0 or not simple or any(x % (1 << L) for x in (m, n, k)):
            continue
        for impl in (1, 2, 3):
            C = C0.copy(order="F")
            oracle.ref_mult(L, impl, alpha, A, ia, B, ib, beta, C, ic)
            err = float(np.abs(C - out["L0"]).max()) if np.isfinite(C).all() else float("inf")
            tol = oracle.error_bound(L, max(k, 1), np.abs(A).max(), np.abs(B).max())
            if err <= tol:
                out[f"L{L}_impl{impl}"] = C
            else:
                # The reference's Strassen is unreliable where a level's split
                # does not fall on mode boundaries (garbage or NaNs that vary run
                # to run, e.g. reading uninitialised workspace).  Such an output
                # is no fixture; the manifest records its error against the
                # reference's own L=0 instead.
                bad[f"L{L}_impl{impl}"] = err if np.isfinite(err) else "non-finite" 
    return A, B, C0, out, dict(m=m, n=n, k=k)


def main():
    if not oracle.ref_available():
        sys.exit("reference library not built: run oracle/build_ref.sh first")
    manifest = []
    for i, (name, ic, ia, ib, ext, alpha, beta) in enumerate(CASES):
        A, B, C0, out, mnk = run_case(name, ic, ia, ib, ext, alpha, beta, seed=100 + 10 * i)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), A=A, B=B, C0=C0, **out)
        manifest.append(dict(name=name, idx_C=ic, idx_A=ia, idx_B=ib, extents=ext, alpha=alpha,
                             beta=beta, outputs=sorted(out), reference_invalid=run_case.bad, **mnk))
        print(name, sorted(out))
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
