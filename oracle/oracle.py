"""Test infrastructure only -- the oracle (checker), never the product.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.

* :func:`contract` -- the plain-C restatement of the reference's contraction
  (oracle/contract_ref.c, following src/internal/3t/mult.cxx:100-165 and the
  label analysis of src/iface/3t/mult.cxx:21-126), compiled to
  oracle/liboracle.so;
* :func:`ref_mult` -- the reference library itself, compiled from its own
  sources by oracle/build_ref.sh into oracle/_ref/libtblis_ref.so (present
  only where that build ran); it is the pin for the restatement and the timed
  CPU baseline;
* :func:`strassen_matmul` -- numpy restatement of the reference's 1- and
  2-level Strassen product schedule on plain matrices (coefficients
  src/stra_internal/3t/strassen:1-14, products
  src/stra_internal/3t/stra_mult.cxx:426-590 and
  src/stra_internal/3t/stra_mult_2level.cxx:341-1485), used to check the
  product tables on the CPU;
* :func:`uniform` -- the seeded synthetic inputs (U[-1, 1]).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtblis_ref.so")


def build_oracle() -> str:
    """Compile oracle/contract_ref.c (seconds) if the .so is missing or stale."""
    src = os.path.join(HERE, "contract_ref.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-o", ORACLE_SO, src])
    return ORACLE_SO


_oracle = None
_ref = None
_P = ctypes.c_void_p


def _meta(X):
    es = X.dtype.itemsize
    return (np.array(X.shape, dtype=np.int64), np.array([s // es for s in X.strides], dtype=np.int64))


def _oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = ctypes.CDLL(build_oracle())
        _oracle.oracle_contract_d.argtypes = [ctypes.c_double,
                                              _P, ctypes.c_uint, _P, _P, ctypes.c_char_p,
                                              _P, ctypes.c_uint, _P, _P, ctypes.c_char_p,
                                              ctypes.c_double,
                                              _P, ctypes.c_uint, _P, _P, ctypes.c_char_p]
        _oracle.oracle_contract_d.restype = ctypes.c_int
    return _oracle


def contract(alpha, A, idx_A, B, idx_B, beta, C, idx_C) -> None:
    """In place: C = alpha*A*B + beta*C (float64 numpy arrays, any strides)."""
    lib = _oracle_lib()
    for X in (A, B, C):
        assert X.dtype == np.float64
    la, sa = _meta(A); lb, sb = _meta(B); lc, sc = _meta(C)
    st = lib.oracle_contract_d(alpha, A.ctypes.data, A.ndim, la.ctypes.data, sa.ctypes.data, idx_A.encode(),
                               B.ctypes.data, B.ndim, lb.ctypes.data, sb.ctypes.data, idx_B.encode(),
                               beta, C.ctypes.data, C.ndim, lc.ctypes.data, sc.ctypes.data, idx_C.encode())
    if st:
        raise ValueError(f"oracle_contract_d status {st}")


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _ref_lib():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
        _ref.oracle_ref_mult.argtypes = [ctypes.c_int, ctypes.c_double,
                                         _P, ctypes.c_uint, _P, _P, ctypes.c_char_p,
                                         _P, ctypes.c_uint, _P, _P, ctypes.c_char_p,
                                         ctypes.c_double,
                                         _P, ctypes.c_uint, _P, _P, ctypes.c_char_p]
        _ref.oracle_ref_mult.restype = ctypes.c_int
        _ref.oracle_ref_set_impl.argtypes = [ctypes.c_int]
        _ref.oracle_ref_set_threads.argtypes = [ctypes.c_uint]
        _ref.oracle_ref_get_threads.restype = ctypes.c_uint
    return _ref


def ref_set_threads(n: int) -> None:
    _ref_lib().oracle_ref_set_threads(n)


def ref_get_threads() -> int:
    return int(_ref_lib().oracle_ref_get_threads())


def ref_mult(level, impl, alpha, A, idx_A, B, idx_B, beta, C, idx_C) -> None:
    """The compiled reference: tblis_tensor_mult (level 0) or
    stra_tblis_tensor_mult[_2level] (levels 1, 2) with tblis::internal::impl =
    impl (1 ABC, 2 AB, 3 Naive).  In place on C (float64 numpy arrays)."""
    lib = _ref_lib()
    if lib.oracle_ref_set_impl(impl) != 0:
        raise ValueError("impl must be 1, 2 or 3")
    la, sa = _meta(A); lb, sb = _meta(B); lc, sc = _meta(C)
    st = lib.oracle_ref_mult(level, alpha, A.ctypes.data, A.ndim, la.ctypes.data, sa.ctypes.data, idx_A.encode(),
                             B.ctypes.data, B.ndim, lb.ctypes.data, sb.ctypes.data, idx_B.encode(),
                             beta, C.ctypes.data, C.ndim, lc.ctypes.data, sc.ctypes.data, idx_C.encode())
    if st:
        raise ValueError(f"oracle_ref_mult status {st}")


# ---- Strassen schedule restatement -----------------------------------------

# src/stra_internal/3t/strassen:1-14 (rows: sub-block id (0,0),(0,1),(1,0),(1,1); columns: products)
U = np.array([[1, 0, 1, 0, 1, -1, 0], [0, 0, 0, 0, 1, 0, 1], [0, 1, 0, 0, 0, 1, 0], [1, 1, 0, 1, 0, 0, -1]])
V = np.array([[1, 1, 0, -1, 0, 1, 0], [0, 0, 1, 0, 0, 1, 0], [0, 0, 0, 1, 0, 0, 1], [1, 0, -1, 0, 1, 0, 1]])
W = np.array([[1, 0, 0, 1, -1, 0, 1], [0, 0, 1, 0, 1, 0, 0], [0, 1, 0, 1, 0, 0, 0], [1, -1, 1, 0, 0, 1, 0]])


def level_coeffs(level: int):
    """Per-level coefficient matrices over an H x H block grid (H = 2^level):
    rows = block id (r*H + c), columns = products (7^level).  Level 2 is the
    Kronecker square, outer level most significant in both the block row/col
    and the product index."""
    if level == 0:
        one = np.ones((1, 1), dtype=np.int64)
        return one, one, one
    mats = []
    for M in (U, V, W):
        cur = np.ones((1, 1), dtype=np.int64)
        Hc = 1
        for _ in range(level):
            nxt = np.zeros((Hc * Hc * 4, cur.shape[1] * 7), dtype=np.int64)
            for bid in range(Hc * Hc):
                r0, c0 = divmod(bid, Hc)
                for sid in range(4):
                    r1, c1 = divmod(sid, 2)
                    row = (2 * r0 + r1) * (2 * Hc) + (2 * c0 + c1)
                    nxt[row] = np.kron(cur[bid], M[sid])
            cur = nxt
            Hc *= 2
        mats.append(cur)
    return tuple(mats)


def strassen_matmul(A: np.ndarray, B: np.ndarray, level: int) -> np.ndarray:
    """A @ B by the level-L Strassen schedule; dims must be divisible by 2^L."""
    H = 1 << level
    m, k = A.shape
    n = B.shape[1]
    ms, ks, ns = m // H, k // H, n // H
    Uc, Vc, Wc = level_coeffs(level)
    blk = lambda X, r, c, a, b: X[r * a:(r + 1) * a, c * b:(c + 1) * b]
    C = np.zeros((m, n))
    for p in range(Uc.shape[1]):
        S = sum(Uc[i, p] * blk(A, i // H, i % H, ms, ks) for i in range(H * H) if Uc[i, p])
        T = sum(Vc[i, p] * blk(B, i // H, i % H, ks, ns) for i in range(H * H) if Vc[i, p])
        M = S @ T
        for q in range(H * H):
            if Wc[q, p]:
                r, c = divmod(q, H)
                C[r * ms:(r + 1) * ms, c * ns:(c + 1) * ns] += Wc[q, p] * M
    return C


# ---- other fast matrix-multiplication families -----------------------------

def fmm_matmul(A: np.ndarray, B: np.ndarray, dims, U, V, W, level: int = 1) -> np.ndarray:
    """A @ B by the <mb, kb, nb> algorithm with coefficient matrices U (mb*kb x
    R), V (kb*nb x R), W (mb*nb x R) -- block id = row * cols + col, the layout
    of the reference's coefficient files (src/stra_internal/3t/strassen:1-14)
    -- applied recursively `level` times (outer level most significant).
    Ragged sizes are zero-padded to multiples of the grid."""
    mb, kb, nb = dims
    U, V, W = (np.asarray(X) for X in (U, V, W))
    if level == 0:
        return A @ B
    m, k = A.shape
    n = B.shape[1]
    ms, ks, ns = -(-m // mb), -(-k // kb), -(-n // nb)
    Ap = np.zeros((ms * mb, ks * kb)); Ap[:m, :k] = A
    Bp = np.zeros((ks * kb, ns * nb)); Bp[:k, :n] = B
    C = np.zeros((ms * mb, ns * nb))
    blk = lambda X, r, c, a, b: X[r * a:(r + 1) * a, c * b:(c + 1) * b]
    for p in range(U.shape[1]):
        S = sum(U[i, p] * blk(Ap, i // kb, i % kb, ms, ks) for i in range(mb * kb) if U[i, p])
        T = sum(V[j, p] * blk(Bp, j // nb, j % nb, ks, ns) for j in range(kb * nb) if V[j, p])
        if isinstance(S, int) or isinstance(T, int):
            continue
        M = fmm_matmul(S, T, dims, U, V, W, level - 1)
        for q in range(mb * nb):
            if W[q, p]:
                r, c = divmod(q, nb)
                C[r * ms:(r + 1) * ms, c * ns:(c + 1) * ns] += W[q, p] * M
    return C[:m, :n]


def parse_coefficients(text: str):
    """U, V, W from the reference's coefficient-file format: three blocks of
    whitespace-separated integer rows (one row per block id, one column per
    product) separated by lines starting with '#'."""
    blocks, cur = [], []
    for line in text.splitlines():
        if line.strip().startswith("#"):
            if cur:
                blocks.append(cur)
            cur = []
            continue
        if line.strip():
            cur.append([int(x) for x in line.split()])
    if cur:
        blocks.append(cur)
    if len(blocks) != 3:
        raise ValueError(f"expected U, V and W blocks, found {len(blocks)}")
    return tuple(np.array(b, dtype=np.int64) for b in blocks)


def classical_coeffs(mb: int, kb: int, nb: int):
    """U, V, W of the classical <mb, kb, nb> product: one product per (row,
    summed slice, column)."""
    R = mb * kb * nb
    U = np.zeros((mb * kb, R), dtype=np.int64); V = np.zeros((kb * nb, R), dtype=np.int64)
    W = np.zeros((mb * nb, R), dtype=np.int64)
    r = 0
    for i in range(mb):
        for t in range(kb):
            for j in range(nb):
                U[i * kb + t, r] = V[t * nb + j, r] = W[i * nb + j, r] = 1
                r += 1
    return U, V, W


def strassen_plus_classical(axis: int):
    """<3,2,2> (axis 0), <2,3,2> (axis 1) or <2,2,3> (axis 2) with 11
    products: Strassen on the leading 2 x 2 x 2 blocks and the 4 classical
    products of the extra block row, summed slice or column."""
    mb, kb, nb = (3 if axis == 0 else 2), (3 if axis == 1 else 2), (3 if axis == 2 else 2)
    U = np.zeros((mb * kb, 11), dtype=np.int64); V = np.zeros((kb * nb, 11), dtype=np.int64)
    W = np.zeros((mb * nb, 11), dtype=np.int64)
    for r in range(7):
        for i in range(4):
            br, bc = divmod(i, 2)
            U[br * kb + bc, r] = globals()["U"][i, r]
            V[br * nb + bc, r] = globals()["V"][i, r]
            W[br * nb + bc, r] = globals()["W"][i, r]
    r = 7
    for x in range(2):
        for y in range(2):
            if axis == 0:
                a, b, c = (2, x), (x, y), (2, y)
            elif axis == 1:
                a, b, c = (x, 2), (2, y), (x, y)
            else:
                a, b, c = (x, y), (y, 2), (x, 2)
            U[a[0] * kb + a[1], r] = 1
            V[b[0] * nb + b[1], r] = 1
            W[c[0] * nb + c[1], r] = 1
            r += 1
    return U, V, W


def uniform(shape, seed: int, order: str = "F", dtype=np.float64) -> np.ndarray:
    """Seeded i.i.d. U[-1, 1] entries (numpy MT19937), column-major by default."""
    rng = np.random.Generator(np.random.MT19937(seed))
    x = rng.uniform(-1.0, 1.0, size=int(np.prod(shape))).astype(dtype)
    return np.asarray(x.reshape(shape, order=order), order=order)


def uniform_pair(shape_a, shape_b, seed: int = 0, order: str = "F"):
    """A then B drawn from ONE seeded stream (numpy MT19937), i.i.d.
    U[-1, 1], column-major by default: the config-1 inputs ("entries
    i.i.d. uniform[-1,1] from seed 0", A first, then B)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    out = []
    for shape in (shape_a, shape_b):
        x = rng.uniform(-1.0, 1.0, size=int(np.prod(shape)))
        out.append(np.asarray(x.reshape(shape, order=order), order=order))
    return out[0], out[1]


def exact_dots(Arows: np.ndarray, Bcols: np.ndarray) -> np.ndarray:
    """Per-sample dot products sum_p Arows[s, p] * Bcols[s, p] accumulated in
    long double (x87 80-bit on x86-64): the products of two doubles carry at
    most 2^-64 relative error there, so for the sums checked here (p up to
    2^14) the result is exact to far below the FP64 bound."""
    a = np.asarray(Arows, dtype=np.longdouble)
    b = np.asarray(Bcols, dtype=np.longdouble)
    return np.sum(a * b, axis=1)


def error_bound(level: int, npk: int, maxA: float, maxB: float) -> float:
    """max|C - Cref| <= 4 * 12^L * NPk * 2^-53 * max|A| * max|B| (FP64 bound)."""
    return 4.0 * (12.0 ** level) * npk * 2.0 ** -53 * maxA * maxB
