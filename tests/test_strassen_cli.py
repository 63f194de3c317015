"""The test_strassen command line of the library (tblis-strassen_b200/
test_strassen.py): the reference's -file format, its fallbacks and its output
row (test/test_strassen.cxx:45-66, 281, 409, 420-529), on the CPU; one GPU run
of the driver on a small file."""
import importlib.util
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "tblis-strassen_b200", "test_strassen.py")

spec = importlib.util.spec_from_file_location("ts_cli", CLI)
cli = importlib.util.module_from_spec(spec)
spec.loader.exec_module(cli)


def test_parse_lengths():
    assert cli.parse_lengths("a:4;b:8;cc:3;"[:8]) == {"a": 4, "b": 8}
    assert cli.parse_lengths("x:128;") == {"x": 128}
    with pytest.raises(ValueError):
        cli.parse_lengths("ab:4;")


def test_parse_file_comments_and_empty_line_end():
    text = ["# comment\n", "abcd efac fbde & a:6;b:5;c:4;d:3;e:2;f:7;\n", "ij ik kj & i:9;j:8;k:7;\n",
            "\n", "ij ik kj & i:1;j:1;k:1;\n"]
    cases = cli.parse_file(text)
    assert [c[:3] for c in cases] == [("abcd", "efac", "fbde"), ("ij", "ik", "kj")]
    assert cases[0][3]["f"] == 7
    with pytest.raises(ValueError):
        cli.parse_file(["ij ik kj a:1;\n"])
    with pytest.raises(ValueError):
        cli.parse_file(["ij ik kj & i:2;j:2;\n"])     # k has no extent


@pytest.mark.parametrize("m,n,k", [(256, 256, 256), (4096, 36, 7), (1, 2, 97)])
def test_random_contraction_bundle_products(m, n, k):
    rng = np.random.default_rng(3)
    for _ in range(5):
        idx_C, idx_A, idx_B, L = cli.random_contraction(m, n, k, rng)
        prod = lambda s: int(np.prod([L[c] for c in s])) if s else 1
        assert prod([c for c in idx_A if c in idx_C]) == m
        assert prod([c for c in idx_B if c in idx_C]) == n
        assert prod([c for c in idx_A if c in idx_B]) == k
        assert sorted(idx_C) == sorted(set(idx_C))


def test_row_format_matches_reference_printf():
    row = cli.format_row(4096, 4096, 4096, 1.5, 1.2, 3.0e-30)
    assert row == " 4096  4096  4096\t  1.500e+00  1.200e+00 1.374e+02\t   91.63  114.53\t  0.00"


@pytest.mark.gpu
def test_cli_file_mode_on_gpu(tmp_path, cuda):
    f = tmp_path / "cases.txt"
    f.write_text("# small cases\nabcd efac fbde & a:12;b:10;c:8;d:6;e:14;f:4;\nij ik kj & i:100;j:90;k:80;\n")
    for level, impl in ((1, 1), (2, 2), (1, 3), (0, 3)):
        out = subprocess.check_output([sys.executable, CLI, "-file", str(f), "-level", str(level),
                                       "-impl", str(impl), "-niter", "2", "-seed", "1"], text=True)
        rows = [r for r in out.splitlines() if r.strip()]
        assert len(rows) == 2
        for r in rows:
            fields = r.split()
            assert len(fields) == 9
            assert fields[-1] == "0.00"
        assert rows[1].split()[:3] == ["100", "90", "80"]


@pytest.mark.gpu
def test_cli_random_mode_on_gpu(cuda):
    out = subprocess.check_output([sys.executable, CLI, "-m", "300", "-n", "200", "-k", "500", "-niter", "1",
                                   "-seed", "5"], text=True)
    fields = out.split()
    assert fields[:3] == ["300", "200", "500"] and fields[-1] == "0.00"
