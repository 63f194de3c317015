"""test_strassen for the B200 library: the reference's benchmark driver
(test/test_strassen.cxx) with the same command line and output rows.

    python tblis-strassen_b200/test_strassen.py [-m M] [-n N] [-k K] [-niter R]
        [-level 0|1|2] [-impl 1|2|3] [-seed S] [-file FILE]

Without -file it times one random contraction whose row, column and summed
bundles have extent products M, N and K (test/test_strassen.cxx:129-286);
with -file it reads one contraction per line,

    idxC idxA idxB & a:4;b:8;c:6;

(labels of C, A and B, then the extent of every label, each entry ended by
';'; lines starting with '#' are skipped and the first empty line ends the
file, test/test_strassen.cxx:493-529), and times each.  Defaults as the
reference's (:420-491): M = N = K = 256, -niter 3, -impl 1, -level 1;
-level 0 forces -impl 1.

Each row is the reference's (:281, :409)::

    m n k   t_L0 t_L GFLOP   GFLOPS_L0 GFLOPS_L   err

with the times the minimum over -niter runs of the plain contraction
(tblis_tensor_mult, which also produces C_ref) and of the selected level,
each run preceded by an L2 flush (the reference trashes its caches the same
way, :68-95) and timed with CUDA events on the device; GFLOP = 2*m*n*k*1e-9
and err = ||C - C_ref||^2 / ||C_ref||^2 (squared, as the reference prints it,
:110-127).  Operands are device-resident, column-major (the reference's
tensors are column-major, src/util/basic_types.h:21), entries U[0, 1) from the
seed.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

ROW_FORMAT = "%5ld %5ld %5ld\t %10.3e %10.3e %8.3e\t %7.2lf %7.2lf\t %5.2lf"


def parse_lengths(text: str) -> dict:
    """'a:4;b:8;' -> {'a': 4, 'b': 8}.  Every entry is one label, ':' and the
    extent, ended by ';' (test/test_strassen.cxx:45-66)."""
    out = {}
    for tok in text.split(";")[:-1]:
        if len(tok) < 3 or tok[1] != ":":
            raise ValueError(f"bad length entry {tok!r}")
        out[tok[0]] = int(tok[2:])
    return out


def parse_file(lines):
    """Contractions of a -file: (idx_C, idx_A, idx_B, lengths) per line."""
    out = []
    for line in lines:
        line = line.rstrip("\n")
        if not line:
            break
        if line.startswith("#"):
            continue
        parts = line.split()
        if len(parts) < 5 or parts[3] != "&":
            raise ValueError(f"bad contraction line {line!r}")
        idx_C, idx_A, idx_B = parts[0], parts[1], parts[2]
        lengths = parse_lengths(parts[4])
        for c in idx_A + idx_B + idx_C:
            if c not in lengths:
                raise ValueError(f"label {c!r} has no extent in {line!r}")
        out.append((idx_C, idx_A, idx_B, lengths))
    return out


def split_extent(total: int, parts: int, rng) -> list:
    """`parts` extents (each >= 1) whose product is `total`, from the divisors
    of what remains (the bundle extents of a random contraction)."""
    out = []
    rest = total
    for p in range(parts - 1, 0, -1):
        small = [d for d in range(1, int(rest ** 0.5) + 1) if rest % d == 0]
        divs = sorted(set(small + [rest // d for d in small]))
        # favour balanced splits: divisors near rest^(1/(p+1))
        target = rest ** (1.0 / (p + 1))
        divs.sort(key=lambda d: abs(np.log(d) - np.log(target)))
        d = int(divs[int(rng.integers(0, min(3, len(divs))))])
        out.append(d)
        rest //= d
    out.append(rest)
    rng.shuffle(out)
    return out


def random_contraction(m: int, n: int, k: int, rng):
    """A random 3-bundle contraction: 1-3 labels per bundle (row bundle in A
    and C, column bundle in B and C, summed bundle in A and B) with extent
    products m, n, k, and a random label order per operand
    (test/test_strassen.cxx:129-216)."""
    labels = iter("abcdefghijklmnopqrstuvwxyz")
    lengths = {}
    bundles = []
    for total in (m, n, k):
        cnt = int(rng.integers(1, 4))
        ext = split_extent(total, cnt, rng)
        names = [next(labels) for _ in ext]
        lengths.update(zip(names, ext))
        bundles.append(names)
    I, J, P = bundles
    idx_A = list(I + P); idx_B = list(P + J); idx_C = list(I + J)
    for x in (idx_A, idx_B, idx_C):
        rng.shuffle(x)
    return "".join(idx_C), "".join(idx_A), "".join(idx_B), lengths


def format_row(m, n, k, dt, dt2, err) -> str:
    gflops = 2.0 * m * n * k * 1e-9
    return ROW_FORMAT % (m, n, k, dt, dt2, gflops, gflops / dt, gflops / dt2, err)


def run_case(tsb, torch, dev, idx_C, idx_A, idx_B, lengths, level, impl, niter, rng, flush):
    def colmajor(idx):
        shape = [lengths[c] for c in idx]
        t = torch.empty(tuple(reversed(shape)), dtype=torch.float64, device=dev)
        return t.permute(*reversed(range(len(shape))))

    A, B = colmajor(idx_A), colmajor(idx_B)
    A.copy_(torch.from_numpy(rng.random(A.shape)))
    B.copy_(torch.from_numpy(rng.random(B.shape)))
    C, C_ref = colmajor(idx_C), colmajor(idx_C)
    C.zero_()
    C_ref.zero_()
    m = int(np.prod([lengths[c] for c in idx_A if c in idx_C and c not in idx_B]))
    n = int(np.prod([lengths[c] for c in idx_B if c in idx_C and c not in idx_A]))
    k = int(np.prod([lengths[c] for c in idx_A if c in idx_B and c not in idx_C]))

    def timed(fn):
        best = float("inf")
        for _ in range(max(niter, 1)):
            flush.add_(1.0)                     # trash L2 (larger than its 126 MB)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e) / 1e3)
        return best

    # C_ref and C accumulate over the timed runs (beta = 1), as in the reference
    dt = timed(lambda: tsb.contract(0, 1.0, A, idx_A, B, idx_B, 1.0, C_ref, idx_C))
    dt2 = timed(lambda: tsb.contract(level, 1.0, A, idx_A, B, idx_B, 1.0, C, idx_C, impl=impl))
    num = float(torch.sum((C - C_ref) ** 2))
    den = float(torch.sum(C_ref ** 2)) or 1.0
    return format_row(m, n, k, dt, dt2, num / den)


def main(argv=None):
    ap = argparse.ArgumentParser(prefix_chars="-", description=__doc__.split("\n\n")[0])
    ap.add_argument("-m", type=int, default=256)
    ap.add_argument("-n", type=int, default=256)
    ap.add_argument("-k", type=int, default=256)
    ap.add_argument("-niter", type=int, default=3)
    ap.add_argument("-level", type=int, default=1)
    ap.add_argument("-impl", type=int, default=1)
    ap.add_argument("-seed", type=int, default=None)
    ap.add_argument("-file", default=None)
    a = ap.parse_args(argv)
    # the reference's fallbacks for out-of-range values (:426-470)
    niter = a.niter if a.niter >= 0 else 3
    m = a.m if a.m >= 0 else 256
    n = a.n if a.n >= 0 else 256
    k = a.k if a.k >= 0 else 256
    impl = a.impl if 1 <= a.impl <= 3 else 1
    level = a.level if 0 <= a.level <= 2 else 0
    if level == 0:
        impl = 1
    rng = np.random.default_rng(a.seed)

    import importlib.util
    import torch
    here = os.path.dirname(os.path.abspath(__file__))
    name = "tblis_strassen_b200"
    if name in sys.modules:
        tsb = sys.modules[name]
    else:
        spec = importlib.util.spec_from_file_location(name, os.path.join(here, "__init__.py"),
                                                      submodule_search_locations=[here])
        tsb = importlib.util.module_from_spec(spec)
        sys.modules[name] = tsb
        spec.loader.exec_module(tsb)
    dev = torch.device("cuda:0")
    flush = torch.empty(192 * 2 ** 20 // 4, dtype=torch.float32, device=dev).zero_()

    if a.file is None:
        cases = [random_contraction(m, n, k, rng)]
    else:
        with open(a.file) as f:
            cases = parse_file(f)
    for idx_C, idx_A, idx_B, lengths in cases:
        print(run_case(tsb, torch, dev, idx_C, idx_A, idx_B, lengths, level, impl, niter, rng, flush), flush=True)


if __name__ == "__main__":
    main()
