"""Benchmark of the Strassen tensor-contraction path on B200.

Workload (one step = one contraction call):
    C(a,b,c,d) += A(e,f,a,c) * B(f,b,d,e)   FP64, column-major, U[-1,1] (seed 0)
    with every extent 128, i.e. NIm = NJn = NPk = 16384, through
    stra_tblis_tensor_mult (one-level Strassen, variant ABC).
Metric: effective TFLOP/s = 2*NIm*NJn*NPk / t  (the reference's GFLOPS
formula, test/test_strassen.cxx:228,355), for every Strassen level.

The timed region runs exactly --steps contractions on device-resident
operands, bracketed by barrier + synchronize, timed with CUDA events on the
launching stream (max over ranks).  The operands (3 x 2 GiB) are far larger than
the 126 MB L2, so no flush is needed between steps.  The same line also reports
the plain L=0 kernel on the same GPU, the end-to-end figure through the C ABI
with pinned host buffers (host<->device copies inside the timed region), the
roofline of the dominant kernel against a cuBLAS DGEMM measured in the same
run, clocks sampled during the timed region, the error of sampled entries
against exact (long-double) dot products of the same inputs, and the
reference's own CPU implementation timed on the same workload (one full-size
call on all host cores; rank 0, N=1).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "tblis-strassen_b200")
sys.path.insert(0, ROOT)

IDX_A, IDX_B, IDX_C = "efac", "fbde", "abcd"
METRIC = "effective TFLOPS (2mnk/t) Strassen L1/L2 vs plain L=0 TC on 1 B200 at stated error"

# DRAM traffic (read + write bytes) per launch of the dominant kernel at the
# default workload, from one full-size ncu capture (one pass of
# dram__bytes_read.sum + dram__bytes_write.sum; summary in
# profiles/packed_gemm_ws_kernel_fp64_L1_e128_dram.md): packed_gemm_ws_kernel,
# the launch of the L=1 product group at extents 128 (7 GEMMs of 8192^3 on
# packed S_q, T_q, run tile position by tile position): 263.06 GB read,
# 6.45 GB written.
NCU_TRAFFIC_BYTES = 263.06e9 + 6.45e9


def load_package():
    name = "tblis_strassen_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def colmajor(torch, shape, device, gen=None, fill=None, pin=False):
    """Column-major tensor of the given shape (U[-1,1] or constant)."""
    rev = tuple(reversed(shape))
    if device == "cpu":
        t = torch.empty(rev, dtype=torch.float64, pin_memory=pin)
    else:
        t = torch.empty(rev, dtype=torch.float64, device=device)
    if fill is None:
        t.uniform_(-1.0, 1.0, generator=gen)
    else:
        t.fill_(fill)
    return t.permute(*reversed(range(len(shape))))


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def dgemm_peak(torch, device, n=8192, reps=5):
    """cuBLAS DGEMM throughput (TFLOP/s) on this GPU: the FP64 roofline
    denominator (MEASURED_PEAKS.json carries no FP64 figure)."""
    a = torch.rand(n, n, dtype=torch.float64, device=device)
    b = torch.rand(n, n, dtype=torch.float64, device=device)
    c = torch.empty(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def cpu_reference(ext: int, min_seconds: float, level: int, impl: int):
    """The reference's own CPU implementation (oracle/_ref, compiled from its
    sources) on the benchmark workload itself: the same contraction at extent
    `ext` per index (NIm = NJn = NPk = ext^2), all host threads, the minimum
    over repetitions (the reference's run_kernel, test/test_strassen.cxx:74-95)
    run until `min_seconds` of CPU work have been spent (at least one).
    Returns (TFLOP/s, threads, sample description, kind)."""
    from oracle import oracle
    import numpy as np
    if not oracle.ref_available():
        return None
    threads = os.cpu_count() or 1
    oracle.ref_set_threads(threads)
    e = ext
    A, B = oracle.uniform_pair((e,) * 4, (e,) * 4, seed=0)
    C = np.zeros((e,) * 4, order="F")
    flops = 2.0 * float(e ** 2) ** 3
    best, spent, reps = float("inf"), 0.0, 0
    while spent < min_seconds or reps < 1:
        t0 = time.perf_counter()
        oracle.ref_mult(level, impl, 1.0, A, IDX_A, B, IDX_B, 1.0, C, IDX_C)
        dt = time.perf_counter() - t0
        best, spent, reps = min(best, dt), spent + dt, reps + 1
        if reps >= 20:
            break
    sample = (f"reference stra_tblis_tensor_mult{'_2level' if level == 2 else ''} "
              f"(L={level}, impl={impl}) on the benchmark workload itself, extent {e} "
              f"(NIm=NJn=NPk={e * e}), seed-0 U[-1,1] column-major, min of {reps} rep(s) "
              f"({spent:.1f} s CPU wall, {threads} threads)")
    if level == 0:
        sample = sample.replace("stra_tblis_tensor_mult", "tblis_tensor_mult")
    return flops / best / 1e12, threads, sample, "reference"


def sampled_exact_error(torch, A, B, C, nsamples=4096, seed=7):
    """Error of C(abcd) = A(efac) B(fbde) at `nsamples` random entries against
    exact dot products of the same inputs (long double on the host, the
    oracle's exact_dots): (max |C - exact|, sampled normwise error
    ||C_s - exact_s|| / ||exact_s||).  A, B, C are device tensors with every
    extent equal; FP32 values are promoted exactly."""
    from oracle import oracle
    import numpy as np
    rng = np.random.default_rng(seed)
    # (a, b, c, d): a, c from A(e,f,a,c); b, d from B(f,b,d,e)
    hi = (A.shape[2], B.shape[1], A.shape[3], B.shape[2])
    idx = np.stack([rng.integers(0, h, size=nsamples) for h in hi], axis=1)
    worst, num, den = 0.0, 0.0, 0.0
    for lo in range(0, nsamples, 512):
        part = torch.as_tensor(idx[lo:lo + 512], device=A.device)
        a, b, c, d = part[:, 0], part[:, 1], part[:, 2], part[:, 3]
        Ar = A[:, :, a, c].permute(2, 0, 1).reshape(len(a), -1).double().cpu().numpy()
        Bc = B[:, b, d, :].permute(1, 2, 0).reshape(len(a), -1).double().cpu().numpy()
        got = C[a, b, c, d].double().cpu().numpy().astype(np.longdouble)
        ex = oracle.exact_dots(Ar, Bc)
        diff = np.abs(got - ex)
        worst = max(worst, float(diff.max()))
        num += float(np.sum(diff * diff))
        den += float(np.sum(ex * ex))
    return worst, (num / den) ** 0.5 if den else 0.0


def batched_form(torch, tsb, device, stream, count, barrier_sync, max_over_ranks, dtypes=None):
    """The batched uneven workload: `count` contractions with 2-4 indices per
    bundle, extents uniform in 8..96, bundle products in [512, 8192], random
    index orders per operand (seed 0), U[-1,1]; one batch plan (grouped
    launches in one CUDA graph) with autotuned levels, timed against the same
    batch forced to L=0; FP64, then FP32 (split-BF16, 6 terms)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from batched_cases import draw_problem
    rng = np.random.default_rng(0)
    shapes = [draw_problem(rng) for _ in range(count)]
    flops = 0.0
    for ext, ia, ib, ic in shapes:
        m = np.prod([ext[c] for c in ia if c in ic]); n = np.prod([ext[c] for c in ib if c in ic])
        k = np.prod([ext[c] for c in ia if c in ib])
        flops += 2.0 * float(m) * float(n) * float(k)
    out = {"problems": count, "tflop_per_batch": flops / 1e12,
           "workload": "2-4 indices per bundle, extents U{8..96}, bundle products in [512, 8192], random orders"}
    for dtype, name in ((torch.float64, "fp64"), (torch.float32, "fp32_split6")):
        if dtypes is not None and dtype not in dtypes:
            continue
        g = torch.Generator(device=device).manual_seed(1)
        tens = []
        for ext, ia, ib, ic in shapes:
            A = torch.empty([ext[c] for c in ia], dtype=dtype, device=device).uniform_(-1, 1, generator=g)
            B = torch.empty([ext[c] for c in ib], dtype=dtype, device=device).uniform_(-1, 1, generator=g)
            C = torch.zeros([ext[c] for c in ic], dtype=dtype, device=device)
            tens.append((A, ia, B, ib, C, ic))
        res = {}
        # autotuned (level, variant, tile) vs the plain grouped fused launch at L=0
        # FP64: against the plain grouped fused launch; FP32: against the
        # split schedule problem by problem
        # against the plain one-launch fused kernel / problem-by-problem split
        # schedule, and against the best fixed L=0 schedule (the grouped packed
        # GEMM over chunks of problems, FP64; the grouped split GEMM, FP32)
        modes = [("autotuned", -1, None)]
        if dtype == torch.float64:
            modes += [("fused_L0", 0, ["fused"]), ("packed_grouped_L0", 0, ["packed_grouped"])]
        else:
            modes += [("split_L0", 0, ["split"]), ("split_grouped_L0", 0, ["split_grouped"])]
        for mode, lv, allowed in modes:
            probs = [(1.0, A, ia, B, ib, 0.0, C, ic, lv) for A, ia, B, ib, C, ic in tens]
            tsb.set_batch_schedules(allowed)
            try:
                batch = tsb.Batch(probs)
            finally:
                tsb.set_batch_schedules(None)
            create_s, tune_s, timings = batch.stats()
            levels, sched = batch.levels(), batch.schedule()
            batch.execute(stream)
            barrier_sync()
            n = 3
            tt = max_over_ranks(time_steps(torch, lambda: batch.execute(stream), n, stream))
            res[mode] = {"tflops_effective": flops * n / tt / 1e12, "ms_per_batch": tt / n * 1e3,
                         "create_s": create_s, "autotune_s": tune_s, "candidate_timings": timings,
                         "levels": {str(l): levels.count(l) for l in (0, 1, 2) if levels.count(l)},
                         "schedules": {k: sched.count(k) for k in sorted(set(sched))}}
            batch.close()
        # spot check: a few problems against the single-call L=0 path
        worst = 0.0
        for A, ia, B, ib, C, ic in tens[:: max(1, len(tens) // 8)]:
            R = torch.zeros_like(C, dtype=torch.float64)
            tsb.contract(0, 1.0, A.double(), ia, B.double(), ib, 0.0, R, ic, stream=stream)
            torch.cuda.synchronize()
            worst = max(worst, float(torch.linalg.norm((C.double() - R).flatten()) / torch.linalg.norm(R.flatten())))
        res["spot_normwise_err"] = worst
        for base in ("fused_L0", "split_L0", "packed_grouped_L0", "split_grouped_L0"):
            if base in res:
                res["autotuned_vs_" + base] = res["autotuned"]["tflops_effective"] / res[base]["tflops_effective"]
        out[name] = res
        del tens
        torch.cuda.empty_cache()
    return out


def precision_sweep(torch, tsb, device, stream, barrier_sync, max_over_ranks):
    """The precision form over its sizes and both input sets: C(abcd) +=
    A(efac) B(fbde) in FP32 at NIm = NJn = NPk in {4096, 8192, 16384}, entries
    U[-1,1] or sign * 10^U[-3,3] (log-uniform magnitudes in [1e-3, 1e3]),
    L = 0/1/2 with 6 and 3 split-BF16 terms; effective TFLOP/s (median of 3)
    and the normwise error of 1024 sampled entries against exact
    (long-double) dot products of the same FP32 values."""
    out = {}
    for dist in ("uniform", "loguniform"):
        for lo, hi in ((64, 64), (64, 128), (128, 128)):
            npk = lo * hi
            flops = 2.0 * float(npk) ** 3
            g = torch.Generator(device=device).manual_seed(7)
            ext = dict(a=lo, b=lo, e=lo, c=hi, d=hi, f=hi)

            def operand(idx):
                t = colmajor(torch, [ext[x] for x in idx], device, g).float()
                if dist == "loguniform":
                    mag = torch.empty_like(t).uniform_(-3.0, 3.0, generator=g)
                    t = torch.sign(t) * torch.pow(10.0, mag)
                return t

            A, B = operand(IDX_A), operand(IDX_B)
            C = colmajor(torch, [ext[x] for x in IDX_C], device, fill=0.0).float()
            for terms in (6, 3):
                tsb.set_fp32_terms(terms)
                for lv in (0, 1, 2):
                    def run():
                        tsb.contract(lv, 1.0, A, IDX_A, B, IDX_B, 0.0, C, IDX_C, stream=stream)
                    run()
                    barrier_sync()
                    ts = sorted(max_over_ranks(time_steps(torch, run, 1, stream)) for _ in range(3))
                    _, nw = sampled_exact_error(torch, A, B, C, nsamples=1024)
                    out[f"{dist}_N{npk}_L{lv}_{terms}terms"] = {"tflops": flops / ts[1] / 1e12,
                                                                 "sampled_normwise_err": nw}
            tsb.set_fp32_terms(6)
            del A, B, C
            torch.cuda.empty_cache()
    return out


def differentiation_form(torch, device, stream, barrier_sync, max_over_ranks, steps=3):
    """Forward plus backward of the two-contraction chain C(a,b,i,j) =
    sum_{e,f} A(a,b,e,f) B(e,f,i,j), D(a,b,k,l) = sum_{i,j} C E(i,j,k,l),
    loss = sum D*W (a,b,e,f = 128, i,j,k,l = 48; U[-1,1]) through the
    autograd binding: FP64 and FP32 (split-BF16, 6 terms) at L = 0 and 1.
    One step = forward + backward (6 contractions, 4.24 TFLOP by 2mnk)."""
    import importlib
    ag = importlib.import_module("tblis_strassen_b200.autograd")
    n, m = 128, 48
    # 2mnk of: C, D (forward); dL/dC, dA, dB, dE (backward)
    flops = 2.0 * (n * n * m * m * n * n + n * n * m * m * m * m
                   + n * n * m * m * m * m + n * n * n * n * m * m + n * n * m * m * n * n + m * m * m * m * n * n)
    out = {"workload": "C(abij)=A(abef)B(efij), D(abkl)=C(abij)E(ijkl), loss=sum D*W; a,b,e,f=128, i,j,k,l=48",
           "tflop_per_step": flops / 1e12}
    for dtype, name in ((torch.float64, "fp64"), (torch.float32, "fp32_split6")):
        g = torch.Generator(device=device).manual_seed(2)
        A = (torch.rand((n, n, n, n), dtype=dtype, device=device, generator=g) * 2 - 1).requires_grad_()
        B = (torch.rand((n, n, m, m), dtype=dtype, device=device, generator=g) * 2 - 1).requires_grad_()
        E = (torch.rand((m, m, m, m), dtype=dtype, device=device, generator=g) * 2 - 1).requires_grad_()
        W = torch.rand((n, n, m, m), dtype=dtype, device=device, generator=g) * 2 - 1
        for level in (0, 1):
            def step():
                for X in (A, B, E):
                    X.grad = None
                C = ag.contract(A, "abef", B, "efij", "abij", level=level)
                D = ag.contract(C, "abij", E, "ijkl", "abkl", level=level)
                (D * W).sum().backward()
            for _ in range(2):
                step()
            barrier_sync()
            t = max_over_ranks(time_steps(torch, step, steps, stream))
            out[f"{name}_L{level}"] = {"tflops_effective": flops * steps / t / 1e12, "ms_per_step": t / steps * 1e3}
        del A, B, E, W
        torch.cuda.empty_cache()
    return out


def time_steps(torch, fn, steps, stream):
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        fn()
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end) / 1e3


# The FP64 square and rank-k sweep: (NIm, NJn, NPk) as extent pairs of the
# bundles I = (a, c), J = (b, d), P = (e, f) of C(abcd) += A(efac) B(fbde).
SWEEP = [((32, 64), (32, 64), (32, 64)), ((64, 64), (64, 64), (64, 64)),
         ((64, 128), (64, 128), (64, 128)), ((128, 128), (128, 128), (128, 128)),
         ((128, 128), (128, 128), (16, 16)), ((128, 128), (128, 128), (16, 32)),
         ((128, 128), (128, 128), (32, 32)), ((128, 128), (128, 128), (32, 64))]


def sweep(args):
    """Effective TFLOP/s of every sweep shape at L = 0, 1, 2 and variants ABC,
    AB and Naive (one warm-up, then the median of 3 CUDA-event timed calls),
    and the largest error against L = 0 relative to the FP64 bound; one JSON
    line per shape."""
    import torch
    tsb = load_package()
    dev = torch.device("cuda:0")
    gen = torch.Generator(device=dev).manual_seed(0)
    for (a, c), (b, d), (e, f) in SWEEP:
        ext = dict(a=a, b=b, c=c, d=d, e=e, f=f)
        A = colmajor(torch, [ext[x] for x in IDX_A], dev, gen)
        B = colmajor(torch, [ext[x] for x in IDX_B], dev, gen)
        C0 = colmajor(torch, [ext[x] for x in IDX_C], dev, fill=0.0)
        m, n, k = a * c, b * d, e * f
        flops = 2.0 * m * n * k
        R = C0.clone()
        tsb.contract(0, 1.0, A, IDX_A, B, IDX_B, 0.0, R, IDX_C)
        line = {"NIm": m, "NJn": n, "NPk": k, "tflops": {}, "err_over_bound": {}}
        for impl, name in ((1, "ABC"), (2, "AB"), (3, "Naive")):
            for lv in (0, 1, 2):
                if lv == 0 and impl != 1:
                    continue
                C = C0.clone()
                tsb.contract(lv, 1.0, A, IDX_A, B, IDX_B, 0.0, C, IDX_C, impl=impl)
                ts = []
                for _ in range(3):
                    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    s0.record()
                    tsb.contract(lv, 1.0, A, IDX_A, B, IDX_B, 0.0, C, IDX_C, impl=impl)
                    s1.record()
                    s1.synchronize()
                    ts.append(s0.elapsed_time(s1))
                key = f"L{lv}" if lv == 0 else f"L{lv}_{name}"
                line["tflops"][key] = flops / statistics.median(ts) / 1e9
                err = float((C - R).abs().max())
                line["err_over_bound"][key] = err / (4.0 * 12.0 ** lv * k * 2.0 ** -53)
        print(json.dumps(line), flush=True)
        del A, B, C0, R, C
        torch.cuda.empty_cache()


def kernel_probe(args):
    """One warm-up and one timed contraction per requested level (the
    command the ncu captures under profiles/ run)."""
    import torch
    tsb = load_package()
    dev = torch.device("cuda:0")
    gen = torch.Generator(device=dev).manual_seed(0)
    e = args.extent
    ia, ib, ic = IDX_A, IDX_B, IDX_C
    if args.layout == "kmajor":
        # the GEMM C(i,j) = A(k,i) B(k,j) with m = n = k = extent^2, both
        # operands stored with k contiguous
        n = e * e
        A = torch.empty((n, n), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=gen).t()
        B = torch.empty((n, n), dtype=torch.float64, device=dev).uniform_(-1, 1, generator=gen).t()
        C = torch.zeros((n, n), dtype=torch.float64, device=dev).t()
        ia, ib, ic = "ki", "kj", "ij"
    else:
        shape = (e,) * 4
        A = colmajor(torch, shape, dev, gen)
        B = colmajor(torch, shape, dev, gen)
        C = colmajor(torch, shape, dev, fill=0.0)
    if args.dtype == "f32":
        A, B, C = A.float(), B.float(), C.float()
        tsb.set_fp32_terms(args.terms)
    if args.workspace is not None:
        tsb.set_workspace_limit(args.workspace)      # 0: the fully fused kernel
    tsb.set_product_parallel(args.product_parallel)
    if args.kernels == "batch":
        # a 64-problem batched form (FP64, or FP32 with --dtype f32), executed twice
        del A, B, C
        torch.cuda.empty_cache()
        out = batched_form(torch, tsb, dev, torch.cuda.current_stream(), 64, torch.cuda.synchronize,
                           lambda x: x, [torch.float32 if args.dtype == "f32" else torch.float64])
        print(json.dumps(out))
        return
    if args.kernels == "dgemm":
        # cuBLAS DGEMM at the same m = n = k, for side-by-side profiles
        n = e * e
        a = torch.rand(n, n, dtype=torch.float64, device=dev)
        b = torch.rand(n, n, dtype=torch.float64, device=dev)
        c = torch.empty(n, n, dtype=torch.float64, device=dev)
        torch.matmul(a, b, out=c)
        torch.cuda.synchronize()
        s, t = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b, out=c)
        t.record()
        t.synchronize()
        ms = s.elapsed_time(t)
        print(f"cuBLAS DGEMM {n}^3: {ms:.3f} ms  {2.0 * n ** 3 / ms / 1e9:.2f} TFLOP/s")
        return
    levels = [int(x) for x in args.kernels.split(",")]
    for lv in levels:
        tsb.contract(lv, 1.0, A, ia, B, ib, 1.0, C, ic, impl=args.variant)
    torch.cuda.synchronize()
    flops = 2.0 * float(e * e) ** 3
    for lv in levels:
        s, t = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tsb.set_kernel_timing(True)
        s.record()
        tsb.contract(lv, 1.0, A, ia, B, ib, 1.0, C, ic, impl=args.variant)
        t.record()
        t.synchronize()
        ms = s.elapsed_time(t)
        parts = {k: tsb.kernel_timing(k) for k in ("fused", "fused_pairs", "fused_tma", "pack", "packed_gemm", "aux",
                                                   "split_gemm")}
        tsb.set_kernel_timing(False)
        print("   kernels: " + ", ".join(f"{k} {n}x {v:.2f} ms" for k, (n, v) in parts.items() if n))
        print(f"L{lv} impl{args.variant} {args.dtype}{'/' + str(args.terms) + ' terms' if args.dtype == 'f32' else ''} "
              f"{args.layout} extent {e}: {ms:.3f} ms  {flops / ms / 1e9:.2f} TFLOP/s effective")


def rank_sync(torch, dist, device):
    """(barrier_sync, max_over_ranks) for this process: a barrier bracketed by
    device synchronisation (CPU ranks, device None, skip it), and the maximum
    of a per-rank float over all ranks (itself with one process)."""
    def sync():
        if device is not None:
            torch.cuda.synchronize(device)

    def barrier_sync():
        sync()
        if dist is not None:
            dist.barrier()
        sync()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier_sync, max_over_ranks


def aggregate_tflops(world, flops_per_step, steps, seconds):
    """Whole-job throughput: every rank runs its own replica of the step, so
    the job does world * steps steps in the slowest rank's time."""
    return world * flops_per_step * steps / seconds / 1e12


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--extent", type=int, default=128, help="extent of each of the six indices")
    ap.add_argument("--level", type=int, default=1)
    ap.add_argument("--variant", type=int, default=1, help="1 ABC, 2 AB, 3 Naive")
    ap.add_argument("--cpu-seconds", type=float, default=30.0,
                    help="CPU time budget of the reference's timed repetitions (at least one full-size call)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP32 split-BF16 lines")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-form lines")
    ap.add_argument("--no-autograd", action="store_true", help="skip the differentiation-form lines")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--dtype", choices=["f64", "f32"], default="f64",
                    help="operand type of the --kernels probe (f32 = split-BF16 tcgen05 path)")
    ap.add_argument("--terms", type=int, default=6, help="split-BF16 product terms for f32 (3 or 6)")
    ap.add_argument("--sweep", action="store_true",
                    help="FP64 square and rank-k sweep over L = 0/1/2 and ABC/AB/Naive (one JSON line per shape)")
    ap.add_argument("--workspace", type=int, default=None,
                    help="--kernels probe: device workspace limit in bytes (0 = fully fused kernel)")
    ap.add_argument("--product-parallel", type=int, default=-1, choices=[-1, 0, 1],
                    help="--kernels probe: product-parallel schedule (-1 automatic, 0 never, 1 when it fits)")
    ap.add_argument("--layout", choices=["config1", "kmajor"], default="config1",
                    help="--kernels probe: the headline contraction, or the GEMM A(k,i) B(k,j) of m=n=k=extent^2")
    ap.add_argument("--kernels", default=None,
                    help="comma-separated levels: run one warm-up and one timed call per level "
                         "and print per-level times (profiling driver; no JSON line)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.sweep:
        return sweep(args)
    if args.kernels is not None:
        return kernel_probe(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    e = args.extent
    npk = e * e
    flops = 2.0 * float(npk) ** 3
    config = {"workload": f"C(abcd)+=A(efac)*B(fbde) FP64 col-major, extents {e} "
                          f"(NIm=NJn=NPk={npk}), L={args.level} impl={args.variant}",
              "NIm": npk, "NJn": npk, "NPk": npk, "level": args.level, "impl": args.variant,
              "l2_flush": "inputs (3 x %.1f GiB) larger than L2" % (npk * npk * 8 / 2 ** 30),
              "parallelism": f"replicas{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        r = cpu_reference(e, args.cpu_seconds, args.level, args.variant)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
            return
        val, cores, sample, kind = r
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOP/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f64", "data": "synthetic U[-1,1]", "config": config,
                          "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": cores, "kind": kind,
                                           "sample": sample},
                          "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    tsb = load_package()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(device)
    stream = torch.cuda.current_stream(device)

    barrier_sync, max_over_ranks = rank_sync(torch, dist, device)

    gen = torch.Generator(device=device).manual_seed(0 + rank)
    shape = (e,) * 4
    A = colmajor(torch, shape, device, gen)
    B = colmajor(torch, shape, device, gen)
    C = colmajor(torch, shape, device, fill=0.0)

    def step(level=args.level, impl=args.variant):
        tsb.contract(level, 1.0, A, IDX_A, B, IDX_B, 1.0, C, IDX_C, impl=impl, stream=stream)

    # ---- headline: device-resident operands --------------------------------
    for _ in range(args.warmup):
        step()
    barrier_sync()
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
    launches0 = tsb.launch_count()
    tsb.set_kernel_timing(True)      # per-kernel CUDA events on the launch stream
    barrier_sync()
    t = time_steps(torch, step, args.steps, stream)
    barrier_sync()
    launches = tsb.launch_count() - launches0
    clocks = sampler.stop() if sampler else None
    t = max_over_ranks(t)
    ms_per_step = t / args.steps * 1e3
    value = aggregate_tflops(world, flops, args.steps, t)

    kinds_snapshot = {k: tsb.kernel_timing(k) for k in ("fused", "pack", "packed_gemm", "aux")}
    tsb.set_kernel_timing(False)

    # ---- same GPU, other levels (the plain L=0 kernel is the Strassen ratio's denominator)
    levels = {}
    for lv in sorted({0, 1, 2} - {args.level}) + [args.level]:
        if lv == args.level:
            levels[f"L{lv}"] = value / world
            continue
        for _ in range(2):
            step(lv, 1)
        barrier_sync()
        tl = max_over_ranks(time_steps(torch, lambda: step(lv, 1), max(2, args.steps // 2), stream))
        levels[f"L{lv}"] = flops * max(2, args.steps // 2) / tl / 1e12

    # ---- the no-workspace ABC kernel (all products in one persistent launch,
    #      operand sums formed in the consumers from the staged raw blocks),
    #      through the regular call with no workspace allowed (at this level,
    #      at L=0 and at L=2) and through the allocation-free entry point
    no_workspace = {}
    tsb.set_workspace_limit(0)
    try:
        nw = max(2, args.steps // 4)
        for lv in sorted({0, args.level, 2}):
            for _ in range(2):
                step(lv, 1)
            barrier_sync()
            tsb.set_kernel_timing(True)
            tf = max_over_ranks(time_steps(torch, lambda: step(lv, 1), nw, stream))
            ran = [k for k in ("fused", "fused_pairs", "fused_tma") if tsb.kernel_timing(k)[0] > 0]
            tsb.set_kernel_timing(False)
            no_workspace[f"L{lv}_workspace0"] = flops * nw / tf / 1e12
            no_workspace[f"L{lv}_kernel"] = {"fused": "stra_fused_kernel (gathers)",
                                              "fused_pairs": "stra_fused_pair_kernel (16-byte pair copies)",
                                              "fused_tma": "stra_fused_pair_kernel (tensor-map boxes)"}.get(
                                                  ran[0] if ran else "", "none")
    finally:
        tsb.set_workspace_limit(None)
    noalloc = tsb.noalloc_mult
    for _ in range(2):
        noalloc(args.level, 1.0, A, IDX_A, B, IDX_B, 1.0, C, IDX_C, stream=stream)
    barrier_sync()
    tf = max_over_ranks(time_steps(torch, lambda: noalloc(args.level, 1.0, A, IDX_A, B, IDX_B, 1.0, C, IDX_C,
                                                            stream=stream), nw, stream))
    no_workspace[f"L{args.level}_noalloc"] = flops * nw / tf / 1e12

    # ---- accuracy of this run's result: sampled entries against exact dots --
    C.zero_()
    step()
    torch.cuda.synchronize(device)
    exact_err, exact_nw = sampled_exact_error(torch, A, B, C)
    C0 = colmajor(torch, shape, device, fill=0.0)
    tsb.contract(0, 1.0, A, IDX_A, B, IDX_B, 0.0, C0, IDX_C, stream=stream)
    torch.cuda.synchronize(device)
    max_err = float((C - C0).abs().max())
    # FP64 bound: 4 * 12^L * NPk * 2^-53 * max|A| * max|B|
    bound = 4.0 * 12.0 ** args.level * npk * 2.0 ** -53 * float(A.abs().max()) * float(B.abs().max())
    del C0

    # ---- roofline of the dominant kernel ------------------------------------
    peak = dgemm_peak(torch, device)
    # the FP64 tensor-pipe ceiling itself: register-only DMMA loops, with the
    # SM clock sampled while they run (about 0.5 s per launch)
    psampler = ClockSampler(local_rank) if rank == 0 else None
    if psampler:
        psampler.start()
    dmma_ceiling, dmma_ms = tsb.measure_dmma_peak(500000, stream)
    pclocks = psampler.stop() if psampler else None
    kinds = kinds_snapshot
    dom = max(kinds, key=lambda k: kinds[k][1])
    n_launch, dom_ms = kinds[dom]
    # Algorithmic work of one launch of the dominant kernel: the contraction's
    # 2*NIm*NJn*NPk divided over the launches that carry it (one per Strassen
    # product for the packed GEMM; one per contraction for the fused kernel).
    per_launch_flops = flops * args.steps / max(n_launch, 1)
    achieved = per_launch_flops / (dom_ms / max(n_launch, 1) / 1e3) / 1e12
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak,
                "traffic": NCU_TRAFFIC_BYTES,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                "executed_frac": achieved * (7.0 / 8.0) ** args.level / peak,
                "peak_dmma": dmma_ceiling,
                "peak_dmma_source": ("register-only m16n8k4 DMMA loops on every SM (tblis_stra_measure_dmma_peak), "
                                     f"one {dmma_ms:.0f} ms launch, SM clock median "
                                     f"{(pclocks or {}).get('sm_mhz')} MHz"),
                "frac_of_dmma_ceiling": achieved / dmma_ceiling,
                "executed_frac_of_dmma_ceiling": achieved * (7.0 / 8.0) ** args.level / dmma_ceiling,
                "L0_frac_of_dmma_ceiling": None,
                "kernel": {"fused": "stra_dmma_kernel", "pack": "pack_kernel",
                           "packed_gemm": "packed_gemm_ws_kernel", "aux": "aux"}[dom],
                "launches_timed": n_launch, "kernel_ms_total": dom_ms,
                "share_of_step": dom_ms / (t * 1e3),
                "other_kernels_ms": {k: v[1] for k, v in kinds.items() if k != dom}}

    # ---- precision form: FP32 operands on the split-BF16 tcgen05 path -------
    precision = None
    if not args.no_precision:
        A32, B32 = A.float(), B.float()
        A64r, B64r = A32.double(), B32.double()      # the FP32 values, exactly, in FP64
        Cref = colmajor(torch, shape, device, fill=0.0)
        tsb.contract(0, 1.0, A64r, IDX_A, B64r, IDX_B, 0.0, Cref, IDX_C, stream=stream)
        del A64r, B64r
        precision = {"oracle": ("normwise_err: this library's FP64 L=0 contraction of the same FP32 values "
                               "(itself checked below against exact dots); sampled_*_vs_exact: 1024 entries "
                               "against long-double dot products of the same FP32 values"),
                     "tolerance_normwise": {"6": 1e-6, "3": 6e-5}}
        nref = float(torch.linalg.norm(Cref.flatten()))
        C32 = colmajor(torch, shape, device, fill=0.0).float()
        for terms in (6, 3):
            tsb.set_fp32_terms(terms)
            for lv in (0, 1, 2):
                def run32():
                    tsb.contract(lv, 1.0, A32, IDX_A, B32, IDX_B, 0.0, C32, IDX_C, stream=stream)
                for _ in range(2):
                    run32()
                barrier_sync()
                tt = max_over_ranks(time_steps(torch, run32, 3, stream))
                err = float(torch.linalg.norm((C32.double() - Cref).flatten())) / nref
                s_max, s_nw = sampled_exact_error(torch, A32, B32, C32, nsamples=1024)
                precision[f"L{lv}_{terms}terms"] = {"tflops": flops * 3 / tt / 1e12, "normwise_err": err,
                                                    "sampled_normwise_err_vs_exact": s_nw,
                                                    "sampled_max_err_vs_exact": s_max}
        tsb.set_fp32_terms(6)
        best6 = max(v["tflops"] for k, v in precision.items() if k.endswith("_6terms"))
        precision["best_6terms_vs_fp64_L0"] = best6 / levels["L0"]
        del A32, B32, C32, Cref
        torch.cuda.empty_cache()
        precision["sweep"] = precision_sweep(torch, tsb, device, stream, barrier_sync, max_over_ranks)

    # ---- differentiation form: forward + backward through the autograd binding
    differentiation = None
    if not args.no_autograd:
        differentiation = differentiation_form(torch, device, stream, barrier_sync, max_over_ranks)

    # ---- end to end through the C ABI with pinned host buffers --------------
    e2e = None
    if not args.no_e2e:
        del A, B, C
        torch.cuda.empty_cache()
        hA = colmajor(torch, shape, "cpu", pin=True, fill=0.5)
        hB = colmajor(torch, shape, "cpu", pin=True, fill=0.25)
        hC = colmajor(torch, shape, "cpu", pin=True, fill=0.0)
        tsb.set_impl(args.variant)

        def e2e_step():
            tsb.contract(args.level, 1.0, hA, IDX_A, hB, IDX_B, 1.0, hC, IDX_C, drop_in=True)

        e2e_step()
        barrier_sync()
        n2 = max(2, args.steps // 2)
        t0 = time.perf_counter()
        te = time_steps(torch, e2e_step, n2, torch.cuda.current_stream(device))
        wall = time.perf_counter() - t0
        te = max_over_ranks(max(te, wall))
        tsb.set_impl(1)
        nbytes = npk * npk * 8
        e2e = {"value": world * flops * n2 / te / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": 3 * nbytes, "d2h_bytes_per_step": nbytes,
               "path": "stra_tblis_tensor_mult with pinned host tensors (copies inside the call, pipelined in 8 chunks: C's slowest B/C label in 4 x its A/C label c in 2)"}
        del hA, hB, hC

    batched = None
    if not args.no_batched:
        batched = batched_form(torch, tsb, device, stream, args.batch_count, barrier_sync, max_over_ranks)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        r = cpu_reference(e, 0.0, args.level, args.variant)
        if r is not None:
            cpu = {"value": r[0], "unit": "TFLOP/s", "cores": r[1], "kind": r[3], "sample": r[2]}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    if levels.get("L0"):
        roofline["L0_frac_of_dmma_ceiling"] = levels["L0"] / dmma_ceiling
    line = {"metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic U[-1,1] (seed 0)",
            "config": config, "levels_tflops": levels,
            "ratio_vs_L0": value / world / levels["L0"] if levels.get("L0") else None,
            "err_vs_exact_samples": {"max_abs": exact_err, "normwise": exact_nw, "samples": 4096,
                                     "bound": bound, "within_bound": exact_err <= bound,
                                     "exact": "long-double dot products of the same inputs on the host"},
            "max_err_vs_L0": max_err, "error_bound": bound,
            "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks,
            "precision_form": precision,
            "batched_form": batched,
            "differentiation_form": differentiation,
            "no_workspace_tflops": no_workspace,
            "gpu_launches": launches,
            "measured_peaks_file": {k: measured_peaks().get(k) for k in ("hbm_gbs", "bf16_tflops")}}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
