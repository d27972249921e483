#!/usr/bin/env python
"""Benchmark of the IFGF matvec at the headline configuration.

Workload: N = 1,000,000 points uniform on the ellipsoid with semi-axes
(1, 1, 0.5) (normalised Gaussian directions projected radially, seed 0),
sources = targets, Helmholtz kernel e^{ikr}/(4 pi r) with k = 100, complex
densities Re, Im ~ N(0, 1) (seed 1), leaf boxes <= 100 points, order p
(high-order cones (p-3, p, p), low-order cones (p-3, p-3, p-3) clamped at 2).
A step is one matvec u = A w.  The metric is milliseconds per matvec (lower
is better) at relative error <= 1e-4 against the FP64 direct sum at 1,000
sampled targets.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times whole matvecs of the CPU restatement of the
reference's mult (oracle/; the reference itself needs Eigen and oneTBB, which
this image lacks) on all host cores: init untimed, one warm-up matvec, then
timed matvecs until K are done or about REF_BUDGET_S seconds have been timed
(the line reports the steps actually timed).  That arm loads nothing of the
CUDA library.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def _load_by_path(path, name):
    import importlib.util

    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# the synthetic inputs, loaded by file path: importing them through the
# package would load the CUDA library, which the reference arm must not touch
W = _load_by_path(os.path.join(ROOT, "ifgf_b200", "workloads.py"), "_ifgf_bench_workloads")

METRIC = "IFGF matvec ms at N=1e6, k=100, rel err<=1e-4 vs FP64; mixed/batched vs FP64"
UNIT = "ms"
TOL = 1e-4
# seconds of whole oracle matvecs the reference arm times at most (about a
# minute each on 16 host cores at the headline size)
REF_BUDGET_S = 100.0
# DRAM bytes per unit and right-hand side of the dominant kernels (see the
# roofline section): upward FFMA / tensor-core kernels per padded
# geometry-table entry over the levels each runs at this workload, far field
# per (target, far box) pair; from the full-size launch list with
# dram__bytes_read.sum + dram__bytes_write.sum
# (profiles/launches_bench_1e6_mixed_batched.md)
UPWARD_FFMA_DRAM_B = 19.3
UPWARD_TC_DRAM_B = 22.2
FAR_DRAM_B = 26.7


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default=None)
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--k", type=float, default=100.0)
    ap.add_argument("--order", type=int, default=9)
    ap.add_argument("--leaf", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-freq-set", action="store_true",
                    help="skip the convolution-quadrature frequency-set measurement")
    ap.add_argument("--batch", type=int, default=8,
                    help="right-hand sides per step of the mixed pipeline (1: single matvec)")
    ap.add_argument("--upward", choices=["auto", "ffma", "tensor"], default="auto",
                    help="kernel of the mixed upward transfer (tensor cores / FP32 FMA)")
    return ap.parse_args()


def workload_config(a, precision):
    return {
        "workload": f"helmholtz k={a.k:g}, N={a.n} ellipsoid (1,1,0.5), sources=targets",
        "kernel": "helmholtz",
        "n_points": a.n,
        "wavenumber": a.k,
        "leaf_size": a.leaf,
        "order_p": a.order,
        "precision": precision,
        "l2": "inputs and per-matvec working set larger than L2 (126 MB)",
        "parallelism": (f"source subtrees sharded over {a.gpus} GPUs, NCCL all-reduce of the "
                        "target vector" if a.gpus > 1 else "single GPU"),
    }


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        # short, so that ranks waiting on a failed one end with an error
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(ws, x):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# flop model (per unit; transcendental = 1, FMA = 2, complex mul = 6)
# ---------------------------------------------------------------------------
def model(stats):
    lo = stats["order_low"]
    hi = stats["order_high"]
    plo = lo[0] * lo[1] * lo[2]
    cheb = 3 * (plo + lo[1] * lo[2] + lo[2]) * 2
    f_near, f_factor = 23, 25
    f_far = 15 + 6 + cheb + 10
    f_up = 15 + 6 + cheb + 12
    # coarse -> fine: three mode products (complex x real = 4 flops per MAC)
    f0, f1, f2 = 3, 3, 3
    F0, F1, F2 = f0 * lo[0], f1 * lo[1], f2 * lo[2]
    macs = F0 * hi[0] * hi[1] * hi[2] + F0 * F1 * hi[1] * hi[2] + F0 * F1 * F2 * hi[2]
    f_c2f = 4 * macs
    return {
        "leaf_sample": stats["leaf_factor_evals"] * f_factor,
        "upward": stats["upward_node_evals"] * f_up,
        "coarse_to_fine": stats["coarse_cones_total"] * f_c2f,
        "target_eval": stats["far_target_evals"] * f_far,
        "near": stats["near_point_pairs"] * f_near,
        "permute": 0.0,
    }


def measured_peak_tflops(dtype):
    """Dense GEMM throughput of this GPU in the given precision (cuBLAS via
    torch.matmul, 8192^3, best of 5): the measured peak of the FP64 / FP32 pipe."""
    import torch

    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192 if dtype == torch.float64 else 8192
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


# ---------------------------------------------------------------------------
# CPU side: whole matvecs of the oracle on all host threads
# ---------------------------------------------------------------------------
def oracle_matvecs(a, pts, w, warmup, steps, budget_s):
    """Whole FP64 oracle matvecs at the headline configuration on every host
    thread (OpenMP over the reference's parallel loops): init untimed, then
    `warmup` untimed matvecs, then timed ones until `steps` are done or
    `budget_s` seconds have been timed.  Returns (seconds per timed matvec,
    threads, init seconds)."""
    from oracle import oracle as O

    threads = O.max_threads()
    op = O.OracleOperator("helmholtz", a.k, a.leaf, a.order)
    t0 = time.perf_counter()
    op.init(pts, pts)
    init_s = time.perf_counter() - t0
    for _ in range(warmup):
        op.mult(w)
    times = []
    while len(times) < max(1, steps):
        t0 = time.perf_counter()
        op.mult(w)
        times.append(time.perf_counter() - t0)
        if sum(times) >= budget_s:
            break
    return times, threads, init_s


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def run_reference(a):
    # CPU only: rank 0 times whole oracle matvecs, the other ranks exit
    # without work (no process group: the arm has no collective)
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pts = W.ellipsoid_points(a.n, seed=0)
    w = W.densities(a.n, seed=1)
    warm = min(a.warmup, 1)  # the reference's own timing: one warm-up mult, then timed mults
    times, threads, init_s = oracle_matvecs(a, pts, w, warm, a.steps, REF_BUDGET_S)
    v = float(np.mean(times)) * 1e3
    sample = (f"{len(times)} whole FP64 matvecs timed on {threads} host threads after {warm} "
              f"warm-up matvec(s); oracle init {init_s:.1f} s untimed")
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": len(times),
        "warmup": warm, "steps_requested": a.steps, "warmup_requested": a.warmup,
        "ms_per_step": v, "higher_is_better": False, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(a, "fp64"), "impl": "reference",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "CPU restatement of the reference mult (oracle/), whole matvecs; the reference "
                "needs Eigen>=5 and oneTBB, absent from this image; timed steps are capped at "
                f"about {REF_BUDGET_S:.0f} s so the arm ends within minutes",
    }
    print(json.dumps(line), flush=True)


def frequency_set(a, dev):
    """Convolution-quadrature frequency set on one GPU: N = 1e5 points on the
    unit sphere, the modified Helmholtz kernel e^{-s r}/(4 pi r) at the 64
    wavenumbers s_l = (1 - 0.5 z_l)/dt, z_l = 0.9 e^{2 pi i l / 64}, dt = 0.01,
    one density each (leaf 100, order 8), and 16 right-hand sides of the
    Helmholtz kernel at k = 20 (leaf 100, order 9), in mixed precision.  The 64 wavenumbers run as
    one multi-wavenumber batch and, for comparison, as the per-frequency loop
    of set_wavenumber + matvec; errors against the FP64 direct sum at 1000
    sampled targets."""
    import torch

    import ifgf_b200 as G

    n, L, R = 100_000, 64, 16
    pts = W.sphere_points(n, seed=0)
    ks = (1.0 - 0.5 * 0.9 * np.exp(2j * np.pi * np.arange(L) / L)) / 0.01
    wl = np.stack([W.densities(n, seed=10 + l) for l in range(L)])
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def timed(fn, steps):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    op = G.ModifiedHelmholtzIfgfOperator(ks[0], 100, 8)
    op.init(pts, pts)
    op.set_precision("mixed")
    dW = torch.from_numpy(wl).to(dev)
    dU = torch.empty_like(dW)
    dU2 = torch.empty_like(dW)
    nb = n * 16  # bytes per complex128 plane

    def one_pass():
        op.mult_wavenumbers_device(ks, dW.data_ptr(), dU.data_ptr(), sp)

    ms_pass = timed(one_pass, a.steps)
    launches = op.stats()["launches_per_mult"]

    def per_frequency():
        for l in range(L):
            op.set_wavenumber(ks[l])
            op.mult_device(dW.data_ptr() + l * nb, dU2.data_ptr() + l * nb, sp)

    ms_loop = timed(per_frequency, 1)
    one_pass()
    torch.cuda.synchronize()
    u, u2 = dU.cpu().numpy(), dU2.cpu().numpy()
    idx = W.sample_targets(n, 1000, seed=2)
    errs = []
    for l in range(0, L, 4):
        op.set_wavenumber(ks[l])
        d = op.direct_eval(wl[l], idx)
        errs.append(float(np.linalg.norm(u[l][idx] - d) / np.linalg.norm(d)))
    loop_vs_pass = max(float(np.linalg.norm(u[l] - u2[l]) / np.linalg.norm(u2[l]))
                       for l in range(L))

    oph = G.HelmholtzIfgfOperator(20.0, 100, 9)
    oph.init(pts, pts)
    oph.set_precision("mixed")
    wr = np.stack([W.densities(n, seed=200 + r) for r in range(R)])
    dWr = torch.from_numpy(wr).to(dev)
    dUr = torch.empty_like(dWr)
    ms_rhs = timed(lambda: oph.mult_batch_device(dWr.data_ptr(), dUr.data_ptr(), R, sp), a.steps)
    torch.cuda.synchronize()
    d = oph.direct_eval(wr[0], idx)
    err_h = float(np.linalg.norm(dUr[0].cpu().numpy()[idx] - d) / np.linalg.norm(d))

    # all 80 solves captured into one CUDA graph (after the calls above built
    # every buffer and tuned the kernels): one launch runs the whole set
    op.set_wavenumber(ks[0])
    one_pass()
    torch.cuda.synchronize()
    dU3, dUr3 = torch.empty_like(dU), torch.empty_like(dUr)
    graph = torch.cuda.CUDAGraph()
    cs = torch.cuda.Stream()
    cs.wait_stream(stream)
    with torch.cuda.graph(graph, stream=cs, capture_error_mode="relaxed"):
        op.mult_wavenumbers_device(ks, dW.data_ptr(), dU3.data_ptr(), cs.cuda_stream)
        oph.mult_batch_device(dWr.data_ptr(), dUr3.data_ptr(), R, cs.cuda_stream)
    ms_graph = timed(graph.replay, a.steps)
    same = (float(torch.linalg.norm(dU3 - dU) / torch.linalg.norm(dU)),
            float(torch.linalg.norm(dUr3 - dUr) / torch.linalg.norm(dUr)))
    del graph
    return {
        "workload": "modified Helmholtz CQ set, 64 wavenumbers s_l = (1 - 0.45 e^{2 pi i l/64})"
                    "/0.01, N=100000 unit sphere, (order 8) + 16 Helmholtz k=20 right-hand "
                    "sides (order 9); leaf 100, mixed",
        "ms_64_wavenumbers_one_batch": ms_pass,
        "launches_per_batch": launches,
        "ms_64_wavenumbers_set_wavenumber_loop": ms_loop,
        "speedup_batch_vs_loop": ms_loop / ms_pass,
        "max_rel_err_vs_fp64_direct_every_4th": max(errs),
        "max_rel_diff_batch_vs_loop": loop_vs_pass,
        "ms_16_rhs_helmholtz_k20_one_batch": ms_rhs,
        "rel_err_helmholtz_k20_rhs0": err_h,
        "ms_all_80": ms_pass + ms_rhs,
        "ms_all_80_one_cuda_graph": ms_graph,
        "graph_rel_diff_vs_direct_calls": same,
        "graph_note": "the 64-wavenumber batch and the 16-right-hand-side batch captured into "
                      "one CUDA graph (one launch per stage and level for each, "
                      f"{launches} + {oph.stats()['launches_per_mult']} kernels), replayed",
    }


def run_ours(a):
    import torch

    import ifgf_b200 as G

    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    precision = a.precision or "mixed"
    batch = a.batch if precision == "mixed" else 1

    pts = W.ellipsoid_points(a.n, seed=0)
    w = W.densities(a.n, seed=1)
    op = G.HelmholtzIfgfOperator(a.k, a.leaf, a.order)
    op.set_precision(precision)
    op.set_upward_path(a.upward)
    if ws > 1:
        # each rank takes a share of the source subtrees; the partial target
        # vectors are summed by one NCCL all-reduce per matvec
        op.set_shard(rank, ws)
    # the CUDA context exists before init is timed (its creation is no part
    # of the operator's setup)
    torch.zeros(1, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    op.init(pts, pts)
    torch.cuda.synchronize()
    init_ms = (time.perf_counter() - t0) * 1e3

    # right-hand side 0 is w; the others are further seeded densities
    wb = np.stack([w] + [W.densities(a.n, seed=100 + b) for b in range(batch - 1)])
    dwb = torch.from_numpy(wb).to(dev)
    dub = torch.empty_like(dwb)
    dw, du = dwb[0], dub[0]
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def reduce(t):
        if ws > 1:
            from ifgf_b200.distributed import reduce_partial

            reduce_partial(t)

    def step1():
        op.mult_device(dw.data_ptr(), du.data_ptr(), sp)
        reduce(du)

    def step_batch():
        op.mult_batch_device(dwb.data_ptr(), dub.data_ptr(), batch, sp)
        reduce(dub)

    step = step_batch if batch > 1 else step1

    def timed(fn, steps):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        barrier(ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        return max_over_ranks(ws, e0.elapsed_time(e1) / steps)

    # ---- timed region (device events on the launching stream) ----
    # no per-kernel events here: the near field then runs on its own stream,
    # overlapping the level loop, as in production use
    clocks = Clocks(local)
    clocks.start()
    ms_step = timed(step, a.steps)
    clk = clocks.stop()
    ms = ms_step / batch  # per matvec
    single_ms = timed(step1, a.steps) if batch > 1 else ms

    # ---- per-kernel breakdown: a separate pass with CUDA events around every
    # launch (serialised on one stream), for the roofline of the top kernel ----
    op.set_profiling(True)
    for _ in range(a.steps):
        step()
    torch.cuda.synchronize()
    stats = op.stats()
    prof = stats["profile"]
    op.set_profiling(False)

    # ---- accuracy against the FP64 direct sum (GPU, Kahan) ----
    step()
    torch.cuda.synchronize()
    u = dub[0].cpu().numpy()
    idx = W.sample_targets(a.n, 1000, seed=2)
    d = op.direct_eval(w, idx)
    err = float(np.linalg.norm(u[idx] - d) / np.linalg.norm(d))

    # ---- the plain FP64 pipeline on the same operator, for the ratio ----
    fp64 = None
    if precision == "mixed":
        op.set_precision("fp64")
        ms64 = timed(step1, a.steps)
        u64 = du.cpu().numpy()
        err64 = float(np.linalg.norm(u64[idx] - d) / np.linalg.norm(d))
        fp64 = {"ms_per_matvec": ms64, "rel_err_vs_fp64_direct": err64,
                "speedup_mixed_batched_vs_fp64": ms64 / ms,
                "speedup_mixed_single_vs_fp64": ms64 / single_ms,
                "mixed_vs_fp64_rel_diff": float(np.linalg.norm(u - u64) / np.linalg.norm(u64))}
        op.set_precision("mixed")

    # ---- end to end through the public API, pinned host buffers ----
    wp = torch.from_numpy(wb).pin_memory()
    up = torch.empty(wb.shape, dtype=torch.complex128).pin_memory()
    wn, un = wp.numpy(), up.numpy()
    if ws == 1:
        # the reference-facing call: host arrays in, host arrays out
        def e2e_step():
            if batch > 1:
                op.mult_batch(wn, out=un)
            else:
                op.mult(wn[0], out=un[0])
        ds = torch.cuda.default_stream()
    else:
        # per rank: pinned host densities to the GPU, its share, the
        # all-reduce, the result back to pinned host memory
        def e2e_step():
            dwb.copy_(wp, non_blocking=True)
            step()
            up.copy_(dub, non_blocking=True)
        ds = stream
    e2e_step()
    torch.cuda.synchronize()
    barrier(ws)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(ds)
    for _ in range(a.steps):
        e2e_step()
    f1.record(ds)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(ws, f0.elapsed_time(f1) / a.steps) / batch

    # ---- roofline of the dominant kernel (per matvec) ----
    # Peaks: MEASURED_PEAKS.json (driver-measured on this pool's B200s): the
    # sustained bf16 tensor rate for a kernel timed inside a long step, the
    # HBM copy rate.  The flop figure is the algorithmic model (per unit:
    # transcendental = 1, FMA = 2), so `frac` is algorithmic work over the
    # measured peak of the pipe the kernel runs its contraction on.
    flops = model(stats)
    kernels = {k: v for k, v in prof.items() if isinstance(v, dict)}
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    per_mult_ms = kernels[dom]["ms"] / max(prof["mults"], 1)
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        peaks = {}
    hbm = peaks.get("hbm_gbs")
    bf16 = peaks.get("bf16_tflops_sustained")
    achieved = flops[dom] / (per_mult_ms * 1e-3) / 1e12
    # levels whose upward transfer ran on the tensor cores (the autotuner's
    # choice for this step's plane count)
    planes_per_pass = min(batch, max(stats.get("batch_planes", 4), 1)) if batch > 1 else 1
    tuner = (stats.get("upward_tuner") or {}).get(str(planes_per_pass), {})
    tc_levels = [i for i, c in enumerate(tuner.get("tensor", [])) if c == 1]
    levels = stats["upward_levels"]
    # DRAM bytes per padded geometry-table entry and right-hand side, per
    # upward kernel, and per (target, far box) pair and right-hand side of
    # the far field: one ncu capture of dram__bytes_read.sum +
    # dram__bytes_write.sum of this bench command at full size, summed over
    # the launches of each kernel and divided by the units they processed
    # (profiles/launches_bench_1e6_mixed_batched.md)
    bytes_per_unit = {"upward_ffma": UPWARD_FFMA_DRAM_B, "upward_tensor": UPWARD_TC_DRAM_B,
                      "target_eval": FAR_DRAM_B}
    traffic = None
    if precision == "mixed" and batch > 1:
        if dom == "upward":
            traffic = sum(u["padded_entries"] * (bytes_per_unit["upward_tensor"] if i in tc_levels
                                                 else bytes_per_unit["upward_ffma"])
                          for i, u in enumerate(levels))
        elif dom == "target_eval":
            traffic = bytes_per_unit["target_eval"] * stats["far_target_evals"]
    if precision == "mixed" and dom == "upward" and tc_levels and bf16:
        roof = {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": bf16,
                "unit": "TFLOP/s", "frac": achieved / bf16,
                "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)",
                "tensor_levels": tc_levels,
                "tensor_note": "upward transfer on the tensor cores (tcgen05 kind::tf32, split "
                               "TF32 pieces) on the listed levels, FP32 FMA elsewhere; per padded "
                               "entry and plane the tensor cores execute 4 lanes x 2 basis pieces "
                               "x 112 x 2 = 1792 flops for the model's 933"}
    else:
        sgemm = measured_peak_tflops(torch.float64 if precision == "fp64" else torch.float32)
        roof = {"kernel": dom, "bound": "fp64" if precision == "fp64" else "fp32",
                "achieved": achieved, "peak": sgemm, "unit": "TFLOP/s", "frac": achieved / sgemm,
                "peak_source": "builder's in-run cuBLAS GEMM via torch.matmul 8192^3 "
                               "(MEASURED_PEAKS.json has no FP32/FP64 figure)"}
    roof.update({
        "traffic": traffic,
        "traffic_note": "DRAM bytes per matvec of the kernel: ncu per-unit figures of this "
                        "command, scaled by the units of one matvec",
        "launches_per_step": kernels[dom]["launches"] / max(prof["mults"], 1) * batch,
        "ms_per_matvec": per_mult_ms,
        "ms_note": "per-kernel times come from a pass with CUDA events around every launch "
                   "(serialised on one stream); the timed step overlaps the near field",
        "model": "survey flop model: transcendental = 1 flop, FMA = 2; per matvec; the FFMA "
                 "upward kernel executes 600 flops per unit (basis-vector FMAs) for the "
                 "model's 933"})
    if traffic is not None and hbm:
        bw = traffic / (per_mult_ms * 1e-3) / 1e9
        roof["hbm"] = {"achieved": bw, "peak": hbm, "unit": "GB/s", "frac": bw / hbm,
                       "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}
    breakdown = {k: v["ms"] / max(prof["mults"], 1) for k, v in kernels.items()}
    breakdown["serialised_total"] = sum(breakdown.values())
    per_level = {k: [round(x / max(prof["mults"], 1), 3) for x in v["level_ms"]]
                 for k, v in kernels.items() if any(v.get("level_ms", []))}
    # passes per step: one launch sequence covers up to batch_planes
    # right-hand sides
    passes = -(-batch // max(stats.get("batch_planes", 4), 1)) if batch > 1 else 1

    cfg = workload_config(a, precision)
    cfg["batch"] = batch
    line = {
        "metric": METRIC, "value": ms, "unit": UNIT, "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if precision == "fp64" else "f32+f64",
        "data": "synthetic", "config": cfg,
        "value_note": (f"ms per matvec; a step is one batch of {batch} right-hand sides "
                       "through the batched mixed pipeline" if batch > 1 else "ms per matvec"),
        "single_rhs_ms": single_ms,
        "rel_err_vs_fp64_direct": err, "tol": TOL, "meets_tol": err <= TOL,
        "fp64_pipeline": fp64,
        "init_ms": init_ms,
        "init_phases_ms": {"octrees_gpu": stats["init_tree_ms"],
                           "interaction_lists_gpu": stats["init_lists_ms"],
                           "host_plan": stats["init_target_lists_ms"],
                           "device_tables": stats["init_device_phases_ms"]},
        "kernel_ms_per_matvec": breakdown, "kernel_ms_per_level": per_level,
        "gpu_launches": int(stats["launches_per_mult"] * passes * a.steps),
        "e2e": {"value": e2e_ms, "unit": UNIT, "h2d_bytes_per_step": int(wb.nbytes),
                "d2h_bytes_per_step": int(wb.nbytes), "note": "ms per matvec"},
        "roofline": roof, "clocks": clk,
        "upward_tuner": stats.get("upward_tuner"),
        "work": {k: stats[k] for k in ("near_point_pairs", "far_target_evals",
                                       "leaf_factor_evals", "upward_node_evals",
                                       "coarse_cones_total", "fine_cones_total",
                                       "upward_runs_max", "upward_levels")},
    }
    if ws == 1 and not a.no_freq_set:
        line["frequency_set"] = frequency_set(a, dev)
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        # one whole oracle matvec (its first matvec is no slower than later
        # ones: measured 72.1 / 73.8 s for a first and a second at N=2e5)
        times, threads, init_s = oracle_matvecs(a, pts, w, 0, 1, 0.0)
        v = float(times[0]) * 1e3
        line["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one whole FP64 oracle matvec of this workload on {threads} host threads "
                      f"(init {init_s:.1f} s untimed); ms per matvec"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
