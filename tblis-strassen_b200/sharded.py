"""C-row sharding of one contraction over the ranks of a torch.distributed
process group (one process per GPU).

The reference's only multi-process contraction is its MPI SUMMA driver
(dist/summa.cxx:68, summa_pdgemm: ring broadcasts of A and B panels over a
P x P mesh, then a local stra_mult per panel).  On one NVSwitch node every GPU
reaches every other at full bandwidth, so this uses the simplest partition
that needs no reduction: each rank owns a contiguous range of one free row
label of C (a label of A and C, not of B), so

    C[rows_r] = alpha * A[rows_r] * B + beta * C[rows_r]

is the same contraction on sub-views, run by the unmodified single-GPU call
(any Strassen level and variant; Strassen's block split happens inside each
rank's rows).  The data movement is one broadcast of B and one scatter of A's
(and, when beta != 0, C's) row slices from the root, then one gather of C's
slices back: NCCL collectives over NVLink on GPUs, gloo on CPUs.  Nothing in
the path waits on a peer inside a kernel.

``local_rows`` gives a rank its range when the operands are already
distributed (each rank holding its own slices), in which case no collective is
needed at all.
"""
from __future__ import annotations


def row_ranges(extent: int, world: int):
    """Contiguous [lo, hi) ranges of `extent` indices over `world` ranks,
    sizes differing by at most one (the first extent % world ranks get one
    more)."""
    base, extra = divmod(extent, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def local_rows(extent: int, rank: int, world: int):
    return row_ranges(extent, world)[rank]


def split_label(idx_A: str, idx_B: str, idx_C: str, len_C, stride_C, world: int):
    """The label whose range is sharded: a free row label (in A and C, not in
    B) with at least `world` indices; among those, the one with the largest C
    stride (so each rank's C slice is as contiguous as C's layout allows).
    None when no such label exists."""
    best = None
    for pos, c in enumerate(idx_C):
        if c in idx_A and c not in idx_B and idx_C.count(c) == 1 and idx_A.count(c) == 1 \
                and len_C[pos] >= world:
            key = abs(stride_C[pos])
            if best is None or key > best[0]:
                best = (key, c)
    return None if best is None else best[1]


def _narrow(t, idx: str, label: str, lo: int, hi: int):
    return t.narrow(idx.index(label), lo, hi - lo)


def sharded_contract(level, alpha, A, idx_A, B, idx_B, beta, C, idx_C, *, local, group=None, root=0,
                     device=None):
    """C = alpha * A * B + beta * C with C's rows sharded over the group.

    On `root`, A, B and C are the full operands (torch tensors; on the GPU
    or the host); on the other ranks they are ignored (pass None).  The
    broadcast/scatter/gather buffers live on `device` (the rank's GPU under
    NCCL, the CPU under gloo).  `local(level, alpha, A_r, idx_A, B, idx_B,
    beta, C_r, idx_C)` runs the single-device contraction on a rank's slices
    (the library's ``contract`` on the rank's GPU).  Returns the label that
    was split, or None when the contraction has no free row label with at
    least `world` indices (then root alone computes it).  Every rank takes
    the same collective steps in the same order.
    """
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    meta = [None]
    if rank == root:
        label = split_label(idx_A, idx_B, idx_C, list(C.shape), list(C.stride()), world)
        meta = [dict(label=label, dtype=A.dtype, shape_A=list(A.shape), shape_B=list(B.shape),
                     shape_C=list(C.shape), level=level, alpha=alpha, beta=beta)]
    dist.broadcast_object_list(meta, src=root, group=group)
    meta = meta[0]
    label = meta["label"]
    level, alpha, beta = meta["level"], meta["alpha"], meta["beta"]     # the root's
    if label is None:
        if rank == root:
            local(level, alpha, A, idx_A, B, idx_B, beta, C, idx_C)
        dist.barrier(group=group)
        return None
    dtype = meta["dtype"]
    ext = meta["shape_C"][idx_C.index(label)]
    ranges = row_ranges(ext, world)
    chunk = max(hi - lo for lo, hi in ranges)

    # 1. B to every rank (one broadcast).
    Bl = B.to(device).contiguous() if rank == root else torch.empty(meta["shape_B"], dtype=dtype, device=device)
    dist.broadcast(Bl, src=root, group=group)

    # 2. A's (and C's) row slices to their ranks: equal-size chunks along the
    #    split label (the last ones zero-padded), one scatter each.
    def chunk_shape(shape, idx):
        s = list(shape)
        s[idx.index(label)] = chunk
        return s

    def scatter_slices(X, idx, shape):
        out = torch.empty(chunk_shape(shape, idx), dtype=dtype, device=device)
        parts = None
        if rank == root:
            parts = []
            for lo, hi in ranges:
                buf = torch.zeros(chunk_shape(shape, idx), dtype=dtype, device=device)
                _narrow(buf, idx, label, 0, hi - lo).copy_(_narrow(X, idx, label, lo, hi))
                parts.append(buf)
        dist.scatter(out, parts, src=root, group=group)
        lo, hi = ranges[rank]
        return _narrow(out, idx, label, 0, hi - lo)

    Al = scatter_slices(A, idx_A, meta["shape_A"])
    if beta != 0:
        Cl = scatter_slices(C, idx_C, meta["shape_C"])
    else:
        lo, hi = ranges[rank]
        Cl = _narrow(torch.zeros(chunk_shape(meta["shape_C"], idx_C), dtype=dtype, device=device),
                     idx_C, label, 0, hi - lo)

    # 3. the unmodified single-device contraction on this rank's rows
    if Al.numel() and Cl.numel():
        local(level, alpha, Al, idx_A, Bl, idx_B, beta, Cl, idx_C)

    # 4. C's slices back to the root (one gather)
    full = torch.zeros(chunk_shape(meta["shape_C"], idx_C), dtype=dtype, device=device)
    _narrow(full, idx_C, label, 0, Cl.shape[idx_C.index(label)]).copy_(Cl)
    parts = [torch.empty_like(full) for _ in range(world)] if rank == root else None
    dist.gather(full, parts, dst=root, group=group)
    if rank == root:
        for (lo, hi), part in zip(ranges, parts):
            _narrow(C, idx_C, label, lo, hi).copy_(_narrow(part, idx_C, label, 0, hi - lo))
    return label
