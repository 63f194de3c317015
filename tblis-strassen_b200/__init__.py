"""tblis-strassen for NVIDIA B200 (sm_100a).

The library proper is ``libtblis_stra_b200.so`` (C ABI in
``include/tblis_stra_b200.h``).  This package re-exports the Python mirror of
the reference's contraction API (:mod:`.tblis_stra`).  The directory name
contains a hyphen, so load it by path, e.g.::

    import importlib.util, sys
    spec = importlib.util.spec_from_file_location(
        "tblis_strassen_b200", "tblis-strassen_b200/__init__.py",
        submodule_search_locations=["tblis-strassen_b200"])
    tsb = importlib.util.module_from_spec(spec); sys.modules[spec.name] = tsb
    spec.loader.exec_module(tsb)
"""
from .tblis_stra import (  # noqa: F401
    SCHEDULES, Batch, IMPL_AB, IMPL_ABC, IMPL_NAIVE, TYPE_DOUBLE, TYPE_FLOAT, TblisStraError,
    contract, get_fp32_terms, get_impl, get_product_parallel, get_workspace_limit, kernel_timing,
    launch_count, lib, matrix_mult, fused_pairs_query, measure_dmma_peak, noalloc_mult, mult, plan_query, set_batch_schedules, set_fp32_terms, set_impl,
    set_kernel_timing, set_product_parallel, set_workspace_limit, set_wait_limit, get_wait_limit, set_wait_injection,
    set_alloc_limit, get_alloc_limit, ALGORITHMS, set_algorithm, get_algorithm, algorithm_info,
    register_algorithm, parse_coefficients, load_algorithm_file, status_string, stra_mult, stra_mult_2level, tblis_matrix, tblis_tensor, version,
)
