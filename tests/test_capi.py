"""The C-ABI library on a machine without a GPU: it loads, exports every
function include/tblis_stra_b200.h declares, has the reference's struct
layout, and reports errors as status codes instead of aborting."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tblis_stra_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "defined")))


def test_every_declared_symbol_is_exported(tsb):
    names = declared_functions()
    assert "tblis_tensor_mult" in names and "stra_tblis_tensor_mult_2level" in names
    for n in names:
        assert hasattr(tsb.lib, n), n
    # the data symbol too
    ctypes.c_void_p.in_dll(tsb.lib, "tblis_single")


def test_struct_layout_matches_header(tsb, tmp_path):
    prog = tmp_path / "layout.c"
    prog.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "tblis_stra_b200.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(tblis_tensor),'
        'offsetof(tblis_tensor,conj),offsetof(tblis_tensor,scalar),offsetof(tblis_tensor,data),'
        'offsetof(tblis_tensor,ndim),offsetof(tblis_tensor,len),offsetof(tblis_tensor,stride));return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    T = tsb.tblis_tensor
    want = [ctypes.sizeof(T), T.conj.offset, T.scalar.offset, T.data.offset, T.ndim.offset,
            T.len.offset, T.stride.offset]
    assert got == want


def test_struct_layout_matches_reference_header():
    """include/tblis_stra_b200.h against the reference's own
    src/util/basic_types.h, through the fixture tests/golden/make_layout.py
    compiled from the reference header: every offset, field size, struct size
    and alignment of tblis_tensor and tblis_matrix, the scalar typedefs and the
    type_t values."""
    import json
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_layout import layout
    with open(os.path.join(ROOT, "tests", "golden", "struct_layout.json")) as f:
        want = json.load(f)
    want.pop("_source")
    got = layout(["-I" + os.path.join(ROOT, "include")], HEADER)
    assert got == want


def build_c_example(tmp_path):
    """Compile and link tests/capi_example.c the way INTEGRATION.md says a C
    caller does: the public header and -ltblis_stra_b200, nothing else."""
    lib_dir = os.path.join(ROOT, "tblis-strassen_b200")
    exe = tmp_path / "capi_example"
    subprocess.check_call(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "capi_example.c"), "-o", str(exe),
                           "-L", lib_dir, "-ltblis_stra_b200", "-Wl,-rpath," + lib_dir])
    return str(exe)


def test_c_example_links_and_runs(tsb, tmp_path):
    """The linked C program runs; without a GPU the drop-in call reports
    TBLIS_STRA_ERR_NO_DEVICE as its status instead of aborting."""
    import torch
    exe = build_c_example(tmp_path)
    r = subprocess.run([exe, "1", "1", str(tmp_path / "C.bin"), "6"], capture_output=True)
    assert r.returncode == (0 if torch.cuda.is_available() else 10), r.stderr


def test_impl_knob(tsb):
    assert tsb.get_impl() == 1
    for impl in (2, 3, 1):
        tsb.set_impl(impl)
        assert tsb.get_impl() == impl
    with pytest.raises(tsb.TblisStraError):
        tsb.set_impl(4)
    assert tsb.get_impl() == 1


def test_product_parallel_knob(tsb):
    assert tsb.get_product_parallel() == -1
    for mode in (0, 1, -1):
        tsb.set_product_parallel(mode)
        assert tsb.get_product_parallel() == mode
    for bad in (2, -2):
        with pytest.raises(tsb.TblisStraError):
            tsb.set_product_parallel(bad)
    assert tsb.get_product_parallel() == -1


def test_failure_knobs(tsb):
    """Wait bound, wait injection and allocation ceiling: per-thread settings
    with their defaults restored (no GPU needed)."""
    assert tsb.get_wait_limit() == 0
    tsb.set_wait_limit(12345)
    assert tsb.get_wait_limit() == 12345
    with pytest.raises(tsb.TblisStraError):
        tsb.set_wait_limit(-1)
    tsb.set_wait_limit(0)
    lib = tsb.lib
    assert lib.tblis_stra_get_wait_injection() == 0
    tsb.set_wait_injection(True)
    assert lib.tblis_stra_get_wait_injection() == 1
    tsb.set_wait_injection(False)
    assert lib.tblis_stra_get_wait_injection() == 0
    tsb.set_alloc_limit(1 << 20)
    assert tsb.get_alloc_limit() == 1 << 20
    tsb.set_alloc_limit(None)


def test_status_strings(tsb):
    for s in range(12):
        assert tsb.status_string(s) != "unknown status"
    assert tsb.status_string(99) == "unknown status"


def test_threads_knob_is_kept(tsb):
    tsb.lib.tblis_set_num_threads(6)
    assert tsb.lib.tblis_get_num_threads() == 6
    tsb.lib.tblis_set_num_threads(1)


def test_no_device_is_a_status_not_a_crash(tsb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    A = np.ones((4, 4)); B = np.ones((4, 4)); C = np.zeros((4, 4))
    with pytest.raises(tsb.TblisStraError) as e:
        tsb.mult(1.0, A, "ik", B, "kj", 0.0, C, "ij")
    assert e.value.status in (6, 10)
    # drop-in void symbol: records the status instead
    with pytest.raises(tsb.TblisStraError):
        tsb.mult(1.0, A, "ik", B, "kj", 0.0, C, "ij", drop_in=True)
    assert tsb.lib.tblis_stra_last_status() in (6, 10)


def test_bad_level_is_rejected(tsb):
    A = np.ones((2, 2)); C = np.zeros((2, 2))
    with pytest.raises(tsb.TblisStraError) as e:
        tsb.contract(3, 1.0, A, "ik", A, "kj", 0.0, C, "ij")
    assert e.value.status == 5


def test_batch_schedule_mask(tsb):
    try:
        tsb.set_batch_schedules(["packed_grouped", "fused"])
        assert tsb.lib.tblis_stra_get_batch_schedules() == (1 << 2) | (1 << 0)
        with pytest.raises(tsb.TblisStraError):
            tsb.set_batch_schedules([])            # empty mask
        with pytest.raises(tsb.TblisStraError):
            tsb.set_batch_schedules(["scale"])     # not a schedule the tuner chooses
        assert tsb.lib.tblis_stra_get_batch_schedules() == (1 << 2) | (1 << 0)
        tsb.set_batch_schedules(["split_grouped"])
        assert tsb.lib.tblis_stra_get_batch_schedules() == 1 << 6
    finally:
        tsb.set_batch_schedules(None)
    assert tsb.lib.tblis_stra_get_batch_schedules() == 0b1011111


def test_matrix_struct_layout_matches_header(tsb, tmp_path):
    prog = tmp_path / "mlayout.c"
    prog.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "tblis_stra_b200.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(tblis_matrix),'
        'offsetof(tblis_matrix,conj),offsetof(tblis_matrix,scalar),offsetof(tblis_matrix,data),'
        'offsetof(tblis_matrix,m),offsetof(tblis_matrix,n),offsetof(tblis_matrix,rs),'
        'offsetof(tblis_matrix,cs));return 0;}\n')
    exe = tmp_path / "mlayout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    M = tsb.tblis_matrix
    want = [ctypes.sizeof(M), M.conj.offset, M.scalar.offset, M.data.offset, M.m.offset, M.n.offset,
            M.rs.offset, M.cs.offset]
    assert got == want


def test_matrix_shape_and_type_errors(tsb):
    """Mismatched matrix shapes or element types are statuses (checked before
    any device work, as src/stra_iface/3m/stra_mult.cxx:19-27 asserts them)."""
    import numpy as np
    A = np.zeros((4, 5)); B = np.zeros((6, 3)); C = np.zeros((4, 3))
    with pytest.raises(tsb.TblisStraError) as e:
        tsb.matrix_mult(1, 1.0, A, B, 0.0, C)
    assert e.value.status == 3                       # TBLIS_STRA_ERR_EXTENT
    with pytest.raises(tsb.TblisStraError) as e:
        tsb.matrix_mult(0, 1.0, np.zeros((4, 5), np.float32), np.zeros((5, 3)), 0.0, C)
    assert e.value.status == 2                       # TBLIS_STRA_ERR_TYPE
