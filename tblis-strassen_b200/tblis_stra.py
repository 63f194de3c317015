"""Python mirror of the reference's contraction API over this library's C ABI.

The reference exposes ``mult<T>``, ``stra_mult<T>`` and ``stra_mult_2level<T>``
(src/iface/3t/mult.h:26-62, src/stra_iface/3t/stra_mult.h:26-62,
src/stra_iface/3t/stra_mult_2level.h:26-62): ``(alpha, A, idx_A, B, idx_B,
beta, C, idx_C)`` computing ``C = alpha*A*B + beta*C`` over index-label
strings.  The functions here take the same arguments, with torch tensors (CUDA
or CPU) or numpy arrays as the tensor views, and call the extern "C" entry
points of ``libtblis_stra_b200.so`` through ctypes.  Errors the reference
would abort on (debug builds) raise :class:`TblisStraError` here.

The shared library is the product; this module only marshals arguments.  It
raises at import time when the library has not been built, so nothing can run
without the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtblis_stra_b200.so")

TYPE_FLOAT = 0
TYPE_DOUBLE = 1

IMPL_ABC, IMPL_AB, IMPL_NAIVE = 1, 2, 3


class TblisStraError(RuntimeError):
    """A contraction call returned a non-zero TBLIS_STRA_* status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"tblis_stra status {status}: {message}")
        self.status = status


class tblis_tensor(ctypes.Structure):
    """Layout of ``tblis_tensor`` (include/tblis_stra_b200.h)."""

    _fields_ = [
        ("type", ctypes.c_int),
        ("conj", ctypes.c_int),
        ("scalar", ctypes.c_double * 2),   # char[16], 8-byte aligned
        ("data", ctypes.c_void_p),
        ("ndim", ctypes.c_uint),
        ("len", ctypes.POINTER(ctypes.c_ssize_t)),
        ("stride", ctypes.POINTER(ctypes.c_ssize_t)),
    ]


class tblis_matrix(ctypes.Structure):
    """Layout of ``tblis_matrix`` (include/tblis_stra_b200.h)."""

    _fields_ = [
        ("type", ctypes.c_int),
        ("conj", ctypes.c_int),
        ("scalar", ctypes.c_double * 2),   # char[16], 8-byte aligned
        ("data", ctypes.c_void_p),
        ("m", ctypes.c_ssize_t), ("n", ctypes.c_ssize_t),
        ("rs", ctypes.c_ssize_t), ("cs", ctypes.c_ssize_t),
    ]


MATRIX_ENTRY = {
    (0, IMPL_ABC): "tblis_matrix_mult",
    (1, IMPL_ABC): "stra_tblis_matrix_mult", (1, IMPL_NAIVE): "stra_tblis_matrix_mult_naive",
    (1, IMPL_AB): "stra_tblis_matrix_mult_ab",
    (2, IMPL_ABC): "stra_tblis_matrix_mult_2level", (2, IMPL_NAIVE): "stra_tblis_matrix_mult_2level_naive",
    (2, IMPL_AB): "stra_tblis_matrix_mult_2level_ab",
}


class tblis_stra_problem(ctypes.Structure):
    """Layout of ``tblis_stra_problem`` (include/tblis_stra_b200.h)."""

    _fields_ = [
        ("A", ctypes.POINTER(tblis_tensor)), ("idx_A", ctypes.c_char_p),
        ("B", ctypes.POINTER(tblis_tensor)), ("idx_B", ctypes.c_char_p),
        ("C", ctypes.POINTER(tblis_tensor)), ("idx_C", ctypes.c_char_p),
        ("level", ctypes.c_int),
    ]


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(make -C tblis-strassen_b200, or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    T = ctypes.POINTER(tblis_tensor)
    S = ctypes.c_char_p
    for name in ("tblis_tensor_mult", "stra_tblis_tensor_mult", "stra_tblis_tensor_mult_2level"):
        fn = getattr(lib, name)
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, T, S, T, S, T, S]
        fn.restype = None
    M = ctypes.POINTER(tblis_matrix)
    for name in MATRIX_ENTRY.values():
        fn = getattr(lib, name)
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, M, M, M]
        fn.restype = None
    lib.tblis_stra_mult.argtypes = [ctypes.c_int, T, S, T, S, T, S, ctypes.c_void_p]
    lib.tblis_stra_mult.restype = ctypes.c_int
    lib.tblis_stra_set_impl.argtypes = [ctypes.c_int]
    lib.tblis_stra_set_impl.restype = ctypes.c_int
    lib.tblis_stra_get_impl.restype = ctypes.c_int
    lib.tblis_stra_last_status.restype = ctypes.c_int
    lib.tblis_stra_status_string.argtypes = [ctypes.c_int]
    lib.tblis_stra_status_string.restype = ctypes.c_char_p
    lib.tblis_stra_set_stream.argtypes = [ctypes.c_void_p]
    lib.tblis_stra_set_stream.restype = ctypes.c_int
    lib.tblis_stra_get_stream.restype = ctypes.c_void_p
    lib.tblis_stra_launch_count.restype = ctypes.c_ulonglong
    lib.tblis_stra_version.restype = ctypes.c_char_p
    lib.tblis_stra_last_error_detail.restype = ctypes.c_char_p
    P64 = ctypes.POINTER(ctypes.c_int64)
    lib.tblis_stra_plan_query.argtypes = [T, S, T, S, T, S, P64, ctypes.POINTER(ctypes.c_double)] + [P64] * 9
    lib.tblis_stra_plan_query.restype = ctypes.c_int
    lib.tblis_stra_fused_pairs_query.argtypes = [ctypes.c_int, T, S, T, S, T, S, ctypes.POINTER(ctypes.c_int),
                                                 ctypes.POINTER(ctypes.c_int)]
    lib.tblis_stra_fused_pairs_query.restype = ctypes.c_int
    lib.tblis_stra_set_wait_injection.argtypes = [ctypes.c_int]
    lib.tblis_stra_set_wait_injection.restype = ctypes.c_int
    lib.tblis_stra_get_wait_injection.restype = ctypes.c_int
    lib.tblis_stra_set_workspace_limit.argtypes = [ctypes.c_size_t]
    lib.tblis_stra_set_workspace_limit.restype = ctypes.c_int
    lib.tblis_stra_get_workspace_limit.restype = ctypes.c_size_t
    lib.tblis_stra_set_kernel_timing.argtypes = [ctypes.c_int]
    lib.tblis_stra_set_kernel_timing.restype = ctypes.c_int
    lib.tblis_stra_kernel_timing.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong),
                                             ctypes.POINTER(ctypes.c_double)]
    lib.tblis_stra_kernel_timing.restype = ctypes.c_int
    lib.tblis_stra_set_product_parallel.argtypes = [ctypes.c_int]
    lib.tblis_stra_set_product_parallel.restype = ctypes.c_int
    lib.tblis_stra_get_product_parallel.restype = ctypes.c_int
    lib.tblis_stra_set_fp32_terms.argtypes = [ctypes.c_int]
    lib.tblis_stra_set_fp32_terms.restype = ctypes.c_int
    lib.tblis_stra_get_fp32_terms.restype = ctypes.c_int
    PB = ctypes.POINTER(tblis_stra_problem)
    lib.tblis_stra_batch_create.argtypes = [ctypes.c_int, PB, ctypes.POINTER(ctypes.c_void_p)]
    lib.tblis_stra_batch_create.restype = ctypes.c_int
    lib.tblis_stra_batch_execute.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.tblis_stra_batch_execute.restype = ctypes.c_int
    lib.tblis_stra_batch_levels.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    lib.tblis_stra_batch_levels.restype = ctypes.c_int
    lib.tblis_stra_batch_schedule.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    lib.tblis_stra_batch_schedule.restype = ctypes.c_int
    lib.tblis_stra_batch_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    lib.tblis_stra_batch_stats.restype = ctypes.c_int
    lib.tblis_stra_set_batch_schedules.argtypes = [ctypes.c_uint]
    lib.tblis_stra_set_batch_schedules.restype = ctypes.c_int
    lib.tblis_stra_get_batch_schedules.restype = ctypes.c_uint
    lib.tblis_stra_batch_destroy.argtypes = [ctypes.c_void_p]
    lib.tblis_stra_batch_destroy.restype = None
    lib.tblis_stra_set_wait_limit.argtypes = [ctypes.c_longlong]
    lib.tblis_stra_set_wait_limit.restype = ctypes.c_int
    lib.tblis_stra_get_wait_limit.restype = ctypes.c_longlong
    lib.tblis_stra_set_alloc_limit.argtypes = [ctypes.c_size_t]
    lib.tblis_stra_set_alloc_limit.restype = ctypes.c_int
    lib.tblis_stra_get_alloc_limit.restype = ctypes.c_size_t
    lib.tblis_stra_measure_dmma_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                                 ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    lib.tblis_stra_measure_dmma_peak.restype = ctypes.c_int
    lib.tblis_stra_mult_noalloc.argtypes = [ctypes.c_int, T, S, T, S, T, S, ctypes.c_void_p]
    lib.tblis_stra_mult_noalloc.restype = ctypes.c_int
    lib.tblis_stra_set_algorithm.argtypes = [ctypes.c_int]
    lib.tblis_stra_set_algorithm.restype = ctypes.c_int
    lib.tblis_stra_get_algorithm.restype = ctypes.c_int
    PI = ctypes.POINTER(ctypes.c_int)
    lib.tblis_stra_algorithm_info.argtypes = [ctypes.c_int, PI, PI, PI, PI, PI]
    lib.tblis_stra_algorithm_info.restype = ctypes.c_int
    lib.tblis_stra_register_algorithm.argtypes = [ctypes.c_int] * 4 + [PI, PI, PI, PI]
    lib.tblis_stra_register_algorithm.restype = ctypes.c_int
    lib.tblis_get_num_threads.restype = ctypes.c_uint
    lib.tblis_set_num_threads.argtypes = [ctypes.c_uint]
    return lib


lib = _load()


def status_string(status: int) -> str:
    return lib.tblis_stra_status_string(status).decode()


def _check(status: int) -> None:
    if status != 0:
        msg = status_string(status)
        detail = lib.tblis_stra_last_error_detail()
        if detail:
            msg += " [" + detail.decode(errors="replace") + "]"
        raise TblisStraError(status, msg)


class _View:
    """A tblis_tensor plus the ctypes arrays it points into."""

    def __init__(self, obj, scalar: float, dtype_code: int | None = None):
        shape, strides, ptr, code = _describe(obj)
        if dtype_code is not None and code != dtype_code:
            raise TypeError("operand element types differ")
        self.obj = obj
        n = len(shape)
        self.len = (ctypes.c_ssize_t * max(n, 1))(*shape)
        self.stride = (ctypes.c_ssize_t * max(n, 1))(*strides)
        t = tblis_tensor()
        t.type = code
        t.conj = 0
        if code == TYPE_DOUBLE:
            t.scalar[0] = float(scalar)
        else:
            ctypes.memmove(ctypes.addressof(t.scalar), ctypes.byref(ctypes.c_float(scalar)), 4)
        t.data = ptr
        t.ndim = n
        t.len = ctypes.cast(self.len, ctypes.POINTER(ctypes.c_ssize_t))
        t.stride = ctypes.cast(self.stride, ctypes.POINTER(ctypes.c_ssize_t))
        self.t = t
        self.code = code


def _describe(obj):
    """(shape, element strides, data pointer, type code) of a torch tensor or numpy array."""
    mod = type(obj).__module__
    if mod.startswith("torch"):
        import torch
        if obj.dtype == torch.float64:
            code = TYPE_DOUBLE
        elif obj.dtype == torch.float32:
            code = TYPE_FLOAT
        else:
            raise TypeError(f"unsupported dtype {obj.dtype}")
        return list(obj.shape), list(obj.stride()), obj.data_ptr(), code
    import numpy as np
    arr = obj
    if arr.dtype == np.float64:
        code, es = TYPE_DOUBLE, 8
    elif arr.dtype == np.float32:
        code, es = TYPE_FLOAT, 4
    else:
        raise TypeError(f"unsupported dtype {arr.dtype}")
    if any(s % es for s in arr.strides):
        raise ValueError("strides must be whole elements")
    return list(arr.shape), [s // es for s in arr.strides], arr.ctypes.data, code


def _labels(idx: str, n: int) -> bytes:
    if len(idx) != n:
        raise ValueError(f"index string {idx!r} has {len(idx)} labels for a {n}-d tensor")
    return idx.encode()


def contract(level: int, alpha, A, idx_A: str, B, idx_B: str, beta, C, idx_C: str,
             impl: int | None = None, stream=None, drop_in: bool = False) -> None:
    """C = alpha*A*B + beta*C at Strassen level 0, 1 or 2.

    ``drop_in=True`` calls the reference-named blocking ``void`` symbols and
    reads the status afterwards; otherwise ``tblis_stra_mult`` is used
    (asynchronous on device pointers, on ``stream`` -- a torch.cuda.Stream, a
    raw handle or None for the thread's default).
    """
    va = _View(A, alpha)
    vb = _View(B, 1.0, va.code)
    vc = _View(C, beta, va.code)
    ia, ib, ic = _labels(idx_A, va.t.ndim), _labels(idx_B, vb.t.ndim), _labels(idx_C, vc.t.ndim)
    old_impl = None
    if impl is not None:
        old_impl = lib.tblis_stra_get_impl()
        _check(lib.tblis_stra_set_impl(impl))
    try:
        if drop_in:
            fn = (lib.tblis_tensor_mult, lib.stra_tblis_tensor_mult,
                  lib.stra_tblis_tensor_mult_2level)[level]
            fn(None, None, ctypes.byref(va.t), ia, ctypes.byref(vb.t), ib, ctypes.byref(vc.t), ic)
            _check(lib.tblis_stra_last_status())
        else:
            handle = None
            if stream is not None:
                handle = getattr(stream, "cuda_stream", stream)
            _check(lib.tblis_stra_mult(level, ctypes.byref(va.t), ia, ctypes.byref(vb.t), ib,
                                       ctypes.byref(vc.t), ic, handle))
    finally:
        if old_impl is not None:
            lib.tblis_stra_set_impl(old_impl)


def noalloc_mult(level: int, alpha, A, idx_A: str, B, idx_B: str, beta, C, idx_C: str, stream=None) -> None:
    """C = alpha*A*B + beta*C through tblis_stra_mult_noalloc: the ABC
    variant on device tensors of the current GPU (FP64), allocating no device
    memory (the scatter vectors go into the library's static device array);
    asynchronous on `stream`."""
    va = _View(A, alpha)
    vb = _View(B, 1.0, va.code)
    vc = _View(C, beta, va.code)
    ia, ib, ic = _labels(idx_A, va.t.ndim), _labels(idx_B, vb.t.ndim), _labels(idx_C, vc.t.ndim)
    handle = None if stream is None else getattr(stream, "cuda_stream", stream)
    _check(lib.tblis_stra_mult_noalloc(level, ctypes.byref(va.t), ia, ctypes.byref(vb.t), ib,
                                       ctypes.byref(vc.t), ic, handle))


def mult(alpha, A, idx_A, B, idx_B, beta, C, idx_C, **kw) -> None:
    """Plain (L=0) contraction; mirrors tblis::mult (src/iface/3t/mult.h:27)."""
    contract(0, alpha, A, idx_A, B, idx_B, beta, C, idx_C, **kw)


def stra_mult(alpha, A, idx_A, B, idx_B, beta, C, idx_C, **kw) -> None:
    """One-level Strassen; mirrors tblis::stra_mult (src/stra_iface/3t/stra_mult.h:27)."""
    contract(1, alpha, A, idx_A, B, idx_B, beta, C, idx_C, **kw)


def stra_mult_2level(alpha, A, idx_A, B, idx_B, beta, C, idx_C, **kw) -> None:
    """Two-level Strassen; mirrors tblis::stra_mult_2level (src/stra_iface/3t/stra_mult_2level.h:27)."""
    contract(2, alpha, A, idx_A, B, idx_B, beta, C, idx_C, **kw)


def set_impl(impl: int) -> None:
    """1 ABC, 2 AB, 3 Naive (the -impl knob of test/test_strassen.cxx:230-243)."""
    _check(lib.tblis_stra_set_impl(impl))


def get_impl() -> int:
    return lib.tblis_stra_get_impl()


def set_workspace_limit(nbytes: int | None) -> None:
    """Device workspace the ABC variant may use (None = unlimited, 0 = the
    fully fused kernel that packs nothing)."""
    _check(lib.tblis_stra_set_workspace_limit(ctypes.c_size_t(-1).value if nbytes is None else nbytes))


def get_workspace_limit() -> int:
    return int(lib.tblis_stra_get_workspace_limit())


SCHEDULES = {"fused": 0, "fused_small": 1, "packed_grouped": 2, "packed": 3, "split": 4, "scale": 5,
             "split_grouped": 6}
SCHEDULE_NAMES = {v: k for k, v in SCHEDULES.items()}


def set_batch_schedules(names) -> None:
    """Schedules the batch autotuner may pick on this thread (None = all):
    any of "fused", "fused_small", "packed_grouped", "packed" (FP64) and
    "split", "split_grouped" (FP32)."""
    if names is None:
        names = ["fused", "fused_small", "packed_grouped", "packed", "split", "split_grouped"]
    mask = 0
    for n in names:
        mask |= 1 << SCHEDULES[n]
    _check(lib.tblis_stra_set_batch_schedules(ctypes.c_uint(mask)))


class Batch:
    """Many contractions planned once and run as grouped launches in one CUDA
    graph (tblis_stra_batch_*).  ``problems``: iterable of
    ``(alpha, A, idx_A, B, idx_B, beta, C, idx_C, level)`` with device tensors;
    level -1 lets the autotuner choose."""

    def __init__(self, problems):
        self._views = []
        probs = []
        for alpha, A, ia, B, ib, beta, C, ic, level in problems:
            va = _View(A, alpha)
            vb = _View(B, 1.0, va.code)
            vc = _View(C, beta, va.code)
            la, lb, lc = _labels(ia, va.t.ndim), _labels(ib, vb.t.ndim), _labels(ic, vc.t.ndim)
            self._views.append((va, vb, vc, la, lb, lc))
            probs.append(tblis_stra_problem(ctypes.pointer(va.t), la, ctypes.pointer(vb.t), lb,
                                            ctypes.pointer(vc.t), lc, level))
        self.count = len(probs)
        arr = (tblis_stra_problem * max(self.count, 1))(*probs)
        self._arr = arr
        self._h = ctypes.c_void_p()
        _check(lib.tblis_stra_batch_create(self.count, arr, ctypes.byref(self._h)))

    def execute(self, stream=None) -> None:
        handle = None if stream is None else getattr(stream, "cuda_stream", stream)
        _check(lib.tblis_stra_batch_execute(self._h, handle))

    def levels(self):
        out = (ctypes.c_int * max(self.count, 1))()
        _check(lib.tblis_stra_batch_levels(self._h, out))
        return list(out)[: self.count]

    def schedule(self):
        """Schedule name of every problem (see SCHEDULES)."""
        out = (ctypes.c_int * max(self.count, 1))()
        _check(lib.tblis_stra_batch_schedule(self._h, out))
        return [SCHEDULE_NAMES[v] for v in list(out)[: self.count]]

    def stats(self):
        """(create seconds, autotune seconds, candidate timings run)."""
        c, t, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(lib.tblis_stra_batch_stats(self._h, ctypes.byref(c), ctypes.byref(t), ctypes.byref(n)))
        return c.value, t.value, n.value

    def close(self) -> None:
        if self._h:
            lib.tblis_stra_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


KERNEL_KINDS = {"fused": 0, "pack": 1, "packed_gemm": 2, "aux": 3, "split_gemm": 4, "fused_tma": 5,
                "fused_pairs": 6}


ALGORITHMS = {"strassen": 0, "classical222": 1, "strassen322": 2, "strassen232": 3, "strassen223": 4}


def set_algorithm(id_or_name) -> None:
    """Fast matrix-multiplication algorithm of the Strassen levels on this
    thread (an id, or a built-in name of ALGORITHMS)."""
    _check(lib.tblis_stra_set_algorithm(ALGORITHMS.get(id_or_name, id_or_name)))


def get_algorithm() -> int:
    return int(lib.tblis_stra_get_algorithm())


def algorithm_info(alg) -> dict:
    """Shape, rank and highest runnable level of an algorithm."""
    v = [ctypes.c_int() for _ in range(5)]
    _check(lib.tblis_stra_algorithm_info(ALGORITHMS.get(alg, alg), *[ctypes.byref(x) for x in v]))
    mb, kb, nb, rank, levels = (x.value for x in v)
    return {"mb": mb, "kb": kb, "nb": nb, "rank": rank, "levels": levels}


def register_algorithm(mb: int, kb: int, nb: int, U, V, W) -> int:
    """Adds an algorithm from its coefficient matrices (rows = block ids,
    columns = products) and returns its id."""
    import numpy as np
    U, V, W = (np.ascontiguousarray(np.asarray(X), dtype=np.int32) for X in (U, V, W))
    rank = U.shape[1]
    if U.shape != (mb * kb, rank) or V.shape != (kb * nb, rank) or W.shape != (mb * nb, rank):
        raise ValueError("coefficient matrices do not match the shape")
    out = ctypes.c_int()
    P = ctypes.POINTER(ctypes.c_int)
    _check(lib.tblis_stra_register_algorithm(mb, kb, nb, rank, U.ctypes.data_as(P), V.ctypes.data_as(P),
                                             W.ctypes.data_as(P), ctypes.byref(out)))
    return out.value


def parse_coefficients(text: str):
    """U, V, W from the reference's coefficient-file format
    (src/stra_internal/3t/strassen:1-14): three blocks of integer rows (one
    row per block id, one column per product) separated by '#' lines."""
    import numpy as np
    blocks, cur = [], []
    for line in text.splitlines():
        if line.strip().startswith("#"):
            if cur:
                blocks.append(cur)
            cur = []
        elif line.strip():
            cur.append([int(x) for x in line.split()])
    if cur:
        blocks.append(cur)
    if len(blocks) != 3:
        raise ValueError(f"expected U, V and W blocks, found {len(blocks)}")
    return tuple(np.array(b, dtype=np.int32) for b in blocks)


def load_algorithm_file(path: str, mb: int, kb: int, nb: int) -> int:
    """Registers the <mb, kb, nb> algorithm of a coefficient file in the
    reference's format (as its generator reads them) and returns its id."""
    with open(path) as f:
        U, V, W = parse_coefficients(f.read())
    return register_algorithm(mb, kb, nb, U, V, W)


def set_wait_limit(cycles: int) -> None:
    """Bound (SM clock cycles) on each pipeline wait of the warp-specialised
    kernels; 0 restores the default (about one second).  A wait that runs out
    ends the kernel cleanly and blocking calls raise status
    TBLIS_STRA_ERR_TIMEOUT."""
    _check(lib.tblis_stra_set_wait_limit(cycles))


def set_wait_injection(on: bool) -> None:
    """Failure test hook: with injection on, every pipeline wait of this
    thread's next calls runs out after the wait bound whatever the state of
    its copy or MMA (a wait on a flag that nothing sets), so the kernels take
    their timeout path and blocking calls raise TBLIS_STRA_ERR_TIMEOUT."""
    _check(lib.tblis_stra_set_wait_injection(1 if on else 0))


def get_wait_limit() -> int:
    return int(lib.tblis_stra_get_wait_limit())


def set_alloc_limit(nbytes: int | None) -> None:
    """Ceiling on any single device allocation a call makes (None = no
    ceiling); a call that would exceed it raises status TBLIS_STRA_ERR_ALLOC
    and leaves C untouched."""
    _check(lib.tblis_stra_set_alloc_limit(ctypes.c_size_t(-1).value if nbytes is None else nbytes))


def get_alloc_limit() -> int:
    return int(lib.tblis_stra_get_alloc_limit())


def set_product_parallel(mode: int) -> None:
    """Product-parallel ABC schedule for small grids: -1 automatic (default),
    0 never, 1 whenever its workspace fits."""
    _check(lib.tblis_stra_set_product_parallel(mode))


def get_product_parallel() -> int:
    return int(lib.tblis_stra_get_product_parallel())


def set_fp32_terms(terms: int) -> None:
    """Split-BF16 product terms for FP32 contractions: 6 (hi/mid/lo) or 3 (hi/mid)."""
    _check(lib.tblis_stra_set_fp32_terms(terms))


def get_fp32_terms() -> int:
    return int(lib.tblis_stra_get_fp32_terms())


def set_kernel_timing(on: bool) -> None:
    """Bracket every kernel launch with CUDA events (clears earlier records)."""
    _check(lib.tblis_stra_set_kernel_timing(1 if on else 0))


def kernel_timing(kind: str):
    """(launches, total milliseconds) of one kernel kind since timing was enabled."""
    n = ctypes.c_ulonglong()
    ms = ctypes.c_double()
    _check(lib.tblis_stra_kernel_timing(KERNEL_KINDS[kind], ctypes.byref(n), ctypes.byref(ms)))
    return int(n.value), float(ms.value)


def measure_dmma_peak(iterations: int = 20000, stream=None):
    """(TFLOP/s, ms): the FP64 tensor-pipe ceiling of the current GPU from
    register-only DMMA loops (the roofline denominator of the FP64 kernels)."""
    tf, ms = ctypes.c_double(), ctypes.c_double()
    handle = None if stream is None else getattr(stream, "cuda_stream", stream)
    _check(lib.tblis_stra_measure_dmma_peak(iterations, ctypes.byref(tf), ctypes.byref(ms), handle))
    return tf.value, ms.value


def launch_count() -> int:
    return int(lib.tblis_stra_launch_count())


def version() -> str:
    return lib.tblis_stra_version().decode()


def plan_query(A, idx_A, B, idx_B, C, idx_C, scatter: bool = True):
    """Bundle analysis of a contraction, without a GPU.

    Returns a dict with m, n, k, batch, alpha, beta and (if ``scatter``) the
    scatter vectors rsA, rsC, csB, csC, ksA, ksB, bA, bB, bC as numpy arrays.
    """
    import numpy as np
    va, vb, vc = _View(A, 1.0), _View(B, 1.0), _View(C, 0.0)
    ia, ib, ic = _labels(idx_A, va.t.ndim), _labels(idx_B, vb.t.ndim), _labels(idx_C, vc.t.ndim)
    sizes = (ctypes.c_int64 * 4)()
    ab = (ctypes.c_double * 2)()
    args = [ctypes.byref(va.t), ia, ctypes.byref(vb.t), ib, ctypes.byref(vc.t), ic, sizes, ab] + [None] * 9
    _check(lib.tblis_stra_plan_query(*args))
    m, n, k, b = (int(x) for x in sizes)
    out = {"m": m, "n": n, "k": k, "batch": b}
    if scatter:
        names = ["rsA", "rsC", "csB", "csC", "ksA", "ksB", "bA", "bB", "bC"]
        lens = [m, m, n, n, k, k, b, b, b]
        arrs = [np.zeros(max(L, 1), dtype=np.int64) for L in lens]
        ptrs = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)) for a in arrs]
        va2, vb2, vc2 = _View(A, 1.0), _View(B, 1.0), _View(C, 0.0)
        _check(lib.tblis_stra_plan_query(ctypes.byref(va2.t), ia, ctypes.byref(vb2.t), ib,
                                         ctypes.byref(vc2.t), ic, sizes, ab, *ptrs))
        for nm, a, L in zip(names, arrs, lens):
            out[nm] = a[:L]
    return out


def fused_pairs_query(level, A, idx_A, B, idx_B, C, idx_C):
    """How the no-workspace ABC kernel stages this contraction's tiles at
    `level` (host only, no GPU needed): a dict with ``pairs`` (bool: the
    element-pair form applies; otherwise the gather form runs) and its plan:
    ``producer`` ("pairs": 16-byte copies of contiguous k pairs; "tma":
    tensor-map boxes), ``conflicts`` (bank conflicts of the consumers' reads,
    0 = none), ``rank_A``, ``rank_B`` (tensor-map ranks, 0 for pair copies),
    ``b_pairs`` (B read in 16-byte pairs), ``swz_A``, ``swz_B`` (swizzle
    spans in bytes, 0 = none), ``bit_A``, ``bit_B`` (the slot k bit each
    16-byte pair spans), the per-lane read offsets ``aoff`` (32 x 2) and
    ``boff`` (32 x 4) in doubles, the fragment permutations ``sigA``,
    ``sigB``, the unswizzled row positions ``koffA``, ``koffB`` of the
    slot's k, the pair bases ``pbaseA``, ``pbaseB`` in copy order and ``tb``,
    the k per ring slot (16 for levels 0 and 1, 8 for level 2, whose operand
    sums have up to 4 blocks); the lists are cut to the entries in use."""
    va, vb, vc = _View(A, 1.0), _View(B, 1.0), _View(C, 0.0)
    ia, ib, ic = _labels(idx_A, va.t.ndim), _labels(idx_B, vb.t.ndim), _labels(idx_C, vc.t.ndim)
    ok = ctypes.c_int(0)
    tab = (ctypes.c_int * 266)()
    _check(lib.tblis_stra_fused_pairs_query(level, ctypes.byref(va.t), ia, ctypes.byref(vb.t), ib,
                                            ctypes.byref(vc.t), ic, ctypes.byref(ok), tab))
    t = list(tab)
    out = {"pairs": bool(ok.value)}
    if out["pairs"]:
        tb = t[265]
        nq, nj, np_ = tb // 8, tb // 4, tb // 2
        out.update(conflicts=t[0], producer=("tma", "pairs")[t[1]], rank_A=t[2], rank_B=t[3],
                   b_pairs=bool(t[4]), swz_A=t[5], swz_B=t[6], bit_A=t[7], bit_B=t[8],
                   aoff=[t[9 + 2 * i:9 + 2 * i + nq] for i in range(32)],
                   boff=[t[73 + 4 * i:73 + 4 * i + nj] for i in range(32)],
                   sigA=t[201:209], sigB=t[209:217], koffA=t[217:217 + tb], koffB=t[233:233 + tb],
                   pbaseA=t[249:249 + np_], pbaseB=t[257:257 + np_], tb=tb)
    return out


def matrix_mult(level: int, alpha, A, B, beta, C, impl: int = IMPL_ABC) -> None:
    """C = alpha*A*B + beta*C through the matrix-level entry points
    (``tblis_matrix_mult``, ``stra_tblis_matrix_mult[_naive|_ab]``,
    ``stra_tblis_matrix_mult_2level[_naive|_ab]``); 2-D torch tensors or numpy
    arrays of any strides.  Blocking, like the reference's calls."""
    views = []
    for X, s in ((A, alpha), (B, 1.0), (C, beta)):
        shape, strides, ptr, code = _describe(X)
        if len(shape) != 2:
            raise ValueError("matrix_mult takes 2-D operands")
        mtx = tblis_matrix()
        mtx.type = code
        mtx.conj = 0
        if code == TYPE_DOUBLE:
            mtx.scalar[0] = float(s)
        else:
            ctypes.memmove(ctypes.addressof(mtx.scalar), ctypes.byref(ctypes.c_float(s)), 4)
        mtx.data = ptr
        mtx.m, mtx.n = shape
        mtx.rs, mtx.cs = strides
        views.append(mtx)
    name = MATRIX_ENTRY.get((level, impl if level else IMPL_ABC))
    if name is None:
        raise ValueError(f"no matrix entry point for level {level}, impl {impl}")
    getattr(lib, name)(None, None, ctypes.byref(views[0]), ctypes.byref(views[1]), ctypes.byref(views[2]))
    _check(lib.tblis_stra_last_status())
