"""Random batched-contraction problems with the shape statistics of the
batched uneven form: 2-4 indices per bundle, extents uniform in [lo, hi],
bundle products rejection-sampled into [pmin, pmax], random index orders per
operand (seeded)."""
import numpy as np


def draw_bundle(rng, labels, lo, hi, pmin, pmax):
    for _ in range(1000):
        n = int(rng.integers(2, 5))
        ext = [int(rng.integers(lo, hi + 1)) for _ in range(n)]
        if pmin <= int(np.prod(ext)) <= pmax:
            return list(zip(labels[:n], ext))
    raise RuntimeError("rejection sampling failed")


def draw_problem(rng, lo=8, hi=96, pmin=512, pmax=8192):
    I = draw_bundle(rng, "abcd", lo, hi, pmin, pmax)
    J = draw_bundle(rng, "efgh", lo, hi, pmin, pmax)
    P = draw_bundle(rng, "ijkl", lo, hi, pmin, pmax)
    ext = dict(I + J + P)
    ia = "".join(rng.permutation([c for c, _ in I + P]))
    ib = "".join(rng.permutation([c for c, _ in P + J]))
    ic = "".join(rng.permutation([c for c, _ in I + J]))
    return ext, ia, ib, ic
