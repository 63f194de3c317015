"""The C caller of INTEGRATION.md (tests/capi_example.c), compiled and linked
against the library with nothing but the public header, run on the GPU: the
reference-named drop-in symbols on host buffers at every level and variant,
checked against the oracle within the FP64 bound."""
import os

import numpy as np
import pytest

from oracle import oracle
from tests.test_capi import build_c_example

pytestmark = pytest.mark.gpu


def pattern(n, mul, add):
    i = np.arange(n, dtype=np.int64)
    return ((i * mul + add) % 2001 - 1000) / 1000.0


@pytest.mark.parametrize("level,impl", [(0, 1), (1, 1), (1, 2), (1, 3), (2, 1), (2, 2), (2, 3)])
def test_c_caller_matches_oracle(tsb, cuda, tmp_path, level, impl):
    import subprocess
    E = 10
    exe = build_c_example(tmp_path)
    out = tmp_path / "C.bin"
    r = subprocess.run([exe, str(level), str(impl), str(out), str(E)], capture_output=True)
    assert r.returncode == 0, r.stderr
    n = E ** 4
    A = pattern(n, 7919, 13).reshape((E,) * 4, order="F")
    B = pattern(n, 104729, 7).reshape((E,) * 4, order="F")
    C = pattern(n, 1299709, 3).reshape((E,) * 4, order="F")
    ref = np.array(C, order="F")
    oracle.contract(1.5, A, "efac", B, "fbde", 0.5, ref, "abcd")
    got = np.fromfile(out, dtype=np.float64).reshape((E,) * 4, order="F")
    bound = 1.5 * oracle.error_bound(level, E * E, np.abs(A).max(), np.abs(B).max()) + 4 * 2.0 ** -53 * 0.5
    assert float(np.abs(got - ref).max()) <= bound
