"""C-row sharding of one contraction over a process group
(tblis-strassen_b200/sharded.py), run as world-size 2 and 3 gloo groups on the
CPU: every rank computes its rows with the oracle standing in for the
single-GPU call, and root's reassembled C must equal the oracle's full
contraction (the partition does not change any element's sum, so the
comparison is exact up to the oracle's own rounding)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load_sharded():
    import importlib.util
    spec = importlib.util.spec_from_file_location("tsb_sharded", os.path.join(ROOT, "tblis-strassen_b200", "sharded.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_row_ranges_cover_and_balance():
    sh = _load_sharded()
    for ext in (1, 2, 7, 64, 129):
        for world in (1, 2, 3, 8):
            r = sh.row_ranges(ext, world)
            assert r[0][0] == 0 and r[-1][1] == ext
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [hi - lo for lo, hi in r]
            assert max(sizes) - min(sizes) <= 1


def test_split_label_choice():
    sh = _load_sharded()
    # C(abcd) += A(efac) B(fbde), column-major C: free row labels a (stride 1), c (stride a*b)
    assert sh.split_label("efac", "fbde", "abcd", [4, 5, 6, 7], [1, 4, 20, 120], 2) == "c"
    assert sh.split_label("efac", "fbde", "abcd", [4, 5, 1, 7], [1, 4, 20, 20], 2) == "a"
    assert sh.split_label("k", "kj", "j", [9], [1], 2) is None           # no free row label


CASES = [
    # (level, alpha, beta, idx_A, idx_B, idx_C, extents)
    (1, 1.0, 0.5, "efac", "fbde", "abcd", dict(a=6, b=5, c=7, d=4, e=3, f=8)),
    (2, -1.5, 0.0, "ik", "kj", "ij", dict(i=11, j=9, k=13)),
    (0, 1.0, 1.0, "bik", "bkj", "bij", dict(b=3, i=5, j=4, k=6)),     # batch label b stays whole
    (1, 1.0, 0.0, "k", "kj", "j", dict(j=5, k=7)),                     # nothing to split: root alone
]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    import sys
    sys.path.insert(0, ROOT)
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sh = _load_sharded()

    def local(level, alpha, A, ia, B, ib, beta, C, ic):
        oracle.contract(alpha, A.numpy(), ia, B.numpy(), ib, beta, C.numpy(), ic)

    try:
        for i, (level, alpha, beta, ia, ib, ic, ext) in enumerate(CASES):
            if rank == 0:
                A = oracle.uniform([ext[c] for c in ia], 10 + i)
                B = oracle.uniform([ext[c] for c in ib], 20 + i)
                C = oracle.uniform([ext[c] for c in ic], 30 + i)
                ref = C.copy(order="F")
                oracle.contract(alpha, A, ia, B, ib, beta, ref, ic)
                tA, tB, tC = (torch.from_numpy(x) for x in (A, B, C))
            else:
                tA = tB = tC = None
            label = sh.sharded_contract(level, alpha, tA, ia, tB, ib, beta, tC, ic, local=local,
                                        device=torch.device("cpu"))
            if rank == 0:
                err = float(np.abs(tC.numpy() - ref).max())
                q.put((i, label, err))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_contraction_matches_oracle(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in CASES)
    labels = [r[1] for r in res]
    assert labels == ["c", "i", "i", None]
    for i, label, err in res:
        assert err <= 1e-13, (i, err)

