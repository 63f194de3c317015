"""Fast matrix-multiplication families beyond Strassen: the oracle's
restatement of the coefficient-driven product schedule (the reference
generates its product code from U/V/W coefficient files,
src/stra_internal/3t/strassen:1-14 and src/stra_internal/3m/my_stra_gen.py),
and the library's algorithm registry (tblis_stra_set_algorithm /
tblis_stra_register_algorithm) on the CPU.  GPU parity of the families lives
in tests/test_fmm_gpu.py."""
import numpy as np
import pytest

from oracle import oracle

FAMILIES = {
    1: ((2, 2, 2), oracle.classical_coeffs(2, 2, 2)),
    2: ((3, 2, 2), oracle.strassen_plus_classical(0)),
    3: ((2, 3, 2), oracle.strassen_plus_classical(1)),
    4: ((2, 2, 3), oracle.strassen_plus_classical(2)),
}


def coefficient_text(U, V, W):
    rows = lambda M: "\n".join(" ".join(str(int(x)) for x in r) for r in M)
    return "# U\n" + rows(U) + "\n#\n" + rows(V) + "\n#\n" + rows(W) + "\n"


@pytest.mark.parametrize("fid", sorted(FAMILIES))
@pytest.mark.parametrize("shape", [(12, 10, 9), (13, 7, 11), (1, 5, 3)])
def test_family_schedules_multiply_exactly(fid, shape):
    dims, (U, V, W) = FAMILIES[fid]
    m, k, n = shape
    rng = np.random.default_rng(fid)
    A, B = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
    for level in (1, 2):
        assert np.abs(oracle.fmm_matmul(A, B, dims, U, V, W, level) - A @ B).max() < 1e-13


def test_coefficient_text_round_trip():
    U, V, W = oracle.parse_coefficients(coefficient_text(oracle.U, oracle.V, oracle.W))
    assert np.array_equal(U, oracle.U) and np.array_equal(V, oracle.V) and np.array_equal(W, oracle.W)


def test_builtin_algorithm_info(tsb):
    want = {0: (2, 2, 2, 7, 2), 1: (2, 2, 2, 8, 1), 2: (3, 2, 2, 11, 1), 3: (2, 3, 2, 11, 1), 4: (2, 2, 3, 11, 1)}
    for aid, (mb, kb, nb, rank, levels) in want.items():
        info = tsb.algorithm_info(aid)
        assert (info["mb"], info["kb"], info["nb"], info["rank"], info["levels"]) == (mb, kb, nb, rank, levels)


def test_set_algorithm_knob(tsb):
    assert tsb.get_algorithm() == 0
    tsb.set_algorithm("strassen223")
    assert tsb.get_algorithm() == 4
    tsb.set_algorithm(0)
    with pytest.raises(tsb.TblisStraError):
        tsb.set_algorithm(999)
    assert tsb.get_algorithm() == 0


def test_register_algorithm_checks_exactness(tsb):
    # Strassen with its products in another order: valid, two levels
    perm = [3, 0, 6, 1, 5, 2, 4]
    U, V, W = (X[:, perm] for X in (oracle.U, oracle.V, oracle.W))
    aid = tsb.register_algorithm(2, 2, 2, U, V, W)
    assert aid >= 5 and tsb.algorithm_info(aid)["levels"] == 2
    # one coefficient changed: not a matrix multiplication
    Ub = U.copy()
    Ub[0, 0] = -Ub[0, 0] if Ub[0, 0] else 1
    with pytest.raises(tsb.TblisStraError) as ei:
        tsb.register_algorithm(2, 2, 2, Ub, V, W)
    assert ei.value.status == 5
    # parsed from the reference's file format
    aid2 = tsb.register_algorithm(2, 2, 2, *tsb.parse_coefficients(coefficient_text(oracle.U, oracle.V, oracle.W)))
    assert tsb.algorithm_info(aid2)["rank"] == 7
