"""Headline benchmark: mixed-precision refined SPD solve vs plain FP64, n = 32768, 64 RHS.

One step = one solve of A X = B through the library's C-ABI (rc_spd_solve_mixed): FP32
working copy with TF32 (default) or BF16 tensor-core trailing updates and FP64 diagonal
blocks, then FP64 conjugate-gradient refinement to a normwise backward error <= 1e-15.
Inputs: A = Q diag(lambda) Q^T, Q from the QR of a seeded N(0,1) matrix, lambda
log-spaced from 1 to 1/kappa; B ~ N(0,1), 64 columns (synthetic, seeded; generated on the
GPU by torch -- input generation only, outside every timed region).

metric unit: TFLOP/s counted as n^3/3 + 2 n^2 nrhs per solve (refinement flops are not
credited), for the mixed solve and the plain FP64 solve alike.

Beside the headline (single GPU): the same solve at kappa = 1e10 with the emulated-FP64
factor (--precision emu64: FP64 working copy, int8 digit-product trailing updates) against
cuSOLVER on that system ("kappa_1e10"), and the roofline of the digit-product kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 32768] [--nrhs 64] [--kappa 1e2] [--precision tf32|bf16|emu64]
                    [--no-e2e] [--no-kappa10] [--no-cpu]

--impl reference times the reference's own CPU path (Remora's cholesky_decomposition +
solve, compiled from its headers into oracle/_ref) on the host cores, on a bounded
sample of the workload (n = 4096 by default), in the same metric. For N > 1 GPUs each rank
runs an independent replica (the path does not shard: replicas only); the time is the
max over ranks and value counts all ranks' solves.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SPD solve TFLOP/s n=32768 mixed+refine vs plain FP64, equal backward error"
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one rc_syrk_tc launch (TF32, CTA
# pairs) at C = 8192 x 8192, depth 1024: `bench.py --case syrk_tc`.
SYRK_TC_DRAM_BYTES_8192 = 253.5e6


def flops(n: int, nrhs: int) -> float:
    return n ** 3 / 3.0 + 2.0 * n * n * nrhs


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        d["source"] = "measured"
        return d
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = open(f"/tmp/rc_clocks_{os.getpid()}.csv", "w+")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if self.out is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.count(",") >= 8]
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_spd(n: int, kappa: float, seed: int, device):
    """A = Q diag(lambda) Q^T (column-major FP64), Q from the QR of a seeded Gaussian."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    G = torch.randn((n, n), generator=g, device=device, dtype=torch.float64)
    Q, _ = torch.linalg.qr(G)
    del G
    lam = torch.logspace(0.0, -math.log10(kappa), n, device=device, dtype=torch.float64)
    A = (Q * lam) @ Q.T
    del Q
    A = (A + A.T) * 0.5  # exactly symmetric
    torch.cuda.synchronize()
    return A  # symmetric, so its row-major storage is also its column-major storage


def backward_error(A, X, B) -> float:
    import torch
    R = B - A @ X
    normA = A.abs().sum(dim=0).max()
    eta = R.abs().amax(dim=0) / (normA * X.abs().amax(dim=0) + B.abs().amax(dim=0))
    return float(eta.max().item())


def cpu_reference(n: int, nrhs: int, steps: int, warmup: int, seed: int = 1) -> dict:
    """The reference's CPU path (oracle/_ref: Remora's cholesky_decomposition + solve),
    single-threaded as the reference is, on an n x n SPD sample of the workload."""
    import numpy as np
    import oracle
    ref = oracle.Reference()
    g = ref.rng(seed)
    G = g.normal(n, n)
    A = np.asfortranarray(G @ G.T / n + 1e-2 * np.eye(n))
    B = g.normal(n, nrhs, row_major=False)
    times = []
    for i in range(warmup + steps):
        X = np.array(B, order="F")
        t0 = time.perf_counter()
        status = ref.cholesky_solve(A, X)
        dt = time.perf_counter() - t0
        assert status == 0
        if i >= warmup:
            times.append(dt)
    t = min(times)
    return {"value": flops(n, nrhs) / t / 1e12, "seconds": t, "times": times}


def workload_config(args, world: int) -> dict:
    """The config of this build's arm: the headline workload it is measured on."""
    return {"workload": f"mixed-precision refined SPD solve n={args.n} nrhs={args.nrhs} kappa={args.kappa:g}",
            "n": args.n, "nrhs": args.nrhs, "kappa": args.kappa, "precision": args.precision,
            "tol": 1e-15, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (A is n^2 x 8 bytes)"}


def reference_config(args) -> dict:
    """The config of the reference arm: the work its timer actually measures -- an FP64 CPU
    solve at the sample size, a bounded stand-in for the n x n headline solve, counted in
    the same metric unit (n^3/3 + 2 n^2 nrhs of the sample's own n)."""
    return {"workload": f"Remora CPU cholesky_decomposition + solve, FP64, n={args.ref_n} nrhs={args.nrhs} "
                        f"(bounded sample of the n={args.n} headline solve; the CPU rate is flat in n "
                        f"above ~2048)",
            "n": args.ref_n, "nrhs": args.nrhs, "kappa": None, "precision": None, "arithmetic": "fp64 (CPU)",
            "headline_n": args.n, "parallelism": "1 host thread (the reference is single-threaded)",
            "l2": "n/a (CPU)"}


def run_reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.ref_n
    r = cpu_reference(n, args.nrhs, args.steps, args.warmup)
    line = {
        "metric": METRIC, "value": r["value"], "unit": "TFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (G G^T / n + 1e-2 I from Remora's mt19937 "
                                                        "generator, N(0,1) right-hand sides)",
        "config": reference_config(args),
        "impl": "reference",
        "cpu_baseline": {"value": r["value"], "unit": "TFLOP/s", "cores": 1, "kind": "reference",
                         "sample": f"Remora's CPU cholesky_decomposition + solve (FP64), one n={n}, "
                                   f"nrhs={args.nrhs} solve per step ({flops(n, args.nrhs):.3e} flops by the metric's "
                                   f"n^3/3 + 2 n^2 nrhs count), min of {args.steps}",
                         "host_cores": os.cpu_count()},
        "e2e": {"value": r["value"], "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def max_over_ranks(value: float, device=None) -> float:
    """The largest of the ranks' values (the job's time is its slowest replica's); with no
    process group, the value itself. Every rank must call it, in the same order."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


_T0 = time.perf_counter()
_PHASE = ["start"]


def phase(name: str) -> None:
    """Progress of the default run on stderr (the JSON result line is the only stdout)."""
    _PHASE[0] = name
    print(f"[bench {time.perf_counter() - _T0:7.1f} s] {name}", file=sys.stderr, flush=True)


def start_watchdog(seconds: float) -> None:
    """End the process (exit status 3, with the phase it was in) if the run outlives
    `seconds`: a stalled run then fails in minutes instead of holding the GPU until an
    outer limit kills it. Every device wait of the library is bounded, so this is the last
    line, not the first."""
    import threading

    def fire():
        import faulthandler
        print(json.dumps({"metric": METRIC, "error": f"watchdog: no result after {seconds:.0f} s",
                          "phase": _PHASE[0]}), flush=True)
        print(f"[bench] watchdog fired in phase '{_PHASE[0]}'; thread stacks:", file=sys.stderr, flush=True)
        faulthandler.dump_traceback(file=sys.stderr, all_threads=True)
        os._exit(3)

    t = threading.Timer(seconds, fire)
    t.daemon = True
    t.start()


def fail_on_status(lib, status: int, info: dict, where: str) -> None:
    """A solve that did not succeed ends the run with its status and, for a device
    timeout, the site of the wait that ran out."""
    if status == 0:
        return
    site = ctypes.c_int(0)
    dev_status = lib.rc_device_error_site(None, ctypes.byref(site))
    print(json.dumps({"metric": METRIC, "error": f"{where}: rc_spd_solve_mixed returned {status}",
                      "device_status": dev_status, "timeout_site": site.value, "info": info}), flush=True)
    sys.exit(4)


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist
    from remora_b200 import _lib, ops

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    lib = _lib.lib()
    n, nrhs = args.n, args.nrhs
    phase("test matrix")
    A = make_spd(n, args.kappa, seed=1234 + rank, device=dev)
    gB = torch.Generator(device=dev).manual_seed(99 + rank)
    B = torch.randn((nrhs, n), generator=gB, device=dev, dtype=torch.float64).t()  # column-major
    X = torch.empty((nrhs, n), device=dev, dtype=torch.float64).t()
    stream = torch.cuda.current_stream()

    def step():
        _, info, status = ops.spd_solve_mixed(A, B, args.precision, tol=1e-15, max_iter=args.max_iter, X=X)
        return info, status

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    phase("warm-up")
    for i in range(args.warmup):
        info, status = step()
        fail_on_status(lib, status, info, f"warm-up step {i}")
    barrier()
    phase("timed steps")
    launches0 = lib.rc_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    infos = []
    with Clocks(local) as clk:
        e0.record(stream)
        for i in range(args.steps):
            infos.append(step())
            _PHASE[0] = f"timed step {i + 1} of {args.steps} done"
        e1.record(stream)
        barrier()
    launches = lib.rc_launch_count() - launches0
    for i, (info_i, status_i) in enumerate(infos):
        fail_on_status(lib, status_i, info_i, f"timed step {i}")
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3, dev)
    mixed_bwd = backward_error(A, X, B)
    status_ok = all(s == 0 for _, s in infos)
    last = infos[-1][0]

    phase("FP64 comparators")
    # Plain FP64 solve (this library) and the cuSOLVER comparator, same inputs.
    X64 = B.clone()
    torch.cuda.synchronize()
    e0.record(stream)
    st64 = ops.cholesky_solve(A, X64)
    e1.record(stream)
    torch.cuda.synchronize()
    t64 = e0.elapsed_time(e1) / 1e3
    fp64_bwd = backward_error(A, X64, B)
    del X64
    torch.cuda.empty_cache()
    e0.record(stream)
    L, _ = torch.linalg.cholesky_ex(A)
    Xc = torch.cholesky_solve(B, L)
    e1.record(stream)
    torch.cuda.synchronize()
    tcus = e0.elapsed_time(e1) / 1e3
    cus_bwd = backward_error(A, Xc, B)
    del L, Xc
    torch.cuda.empty_cache()

    # End to end through the C-ABI from pinned host buffers: H2D of A and B, the solve,
    # D2H of X, every step.
    e2e = None
    if not args.no_e2e:
        phase("end to end from pinned host buffers")
        Ah = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        Ah.copy_(A)
        Bh = B.cpu().pin_memory()
        Xh = torch.empty((nrhs, n), dtype=torch.float64, pin_memory=True).t()
        Ad = torch.empty_like(A)
        Bd = torch.empty((nrhs, n), device=dev, dtype=torch.float64).t()
        del A
        torch.cuda.empty_cache()
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        statuses = []
        for _ in range(args.steps):
            Ad.copy_(Ah, non_blocking=True)
            Bd.copy_(Bh, non_blocking=True)
            statuses.append(ops.spd_solve_mixed(Ad, Bd, args.precision, tol=1e-15, max_iter=args.max_iter, X=X)[1:])
            Xh.copy_(X, non_blocking=True)
        e1.record(stream)
        barrier()
        for i, (info_i, status_i) in enumerate(statuses):
            fail_on_status(lib, status_i, info_i, f"end-to-end step {i}")
        te = max_over_ranks(e0.elapsed_time(e1) / 1e3, dev)
        e2e = {"value": world * args.steps * flops(n, nrhs) / te / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": n * n * 8 + n * nrhs * 8, "d2h_bytes_per_step": n * nrhs * 8,
               "ms_per_step": te / args.steps * 1e3}
        del Ah, Ad
        torch.cuda.empty_cache()
    else:
        del A

    # kappa = 1e10 beside the headline: a TF32/BF16 factor cannot precondition it to FP64
    # accuracy, so the solve runs with the emulated-FP64 factor ("emu64": int8 digit-product
    # trailing updates), against cuSOLVER's FP64 Cholesky solve on the same system.
    k10 = None
    if not args.no_kappa10 and world == 1:
        phase("kappa 1e10 (emu64 factor)")
        A10 = make_spd(n, 1e10, seed=4321, device=dev)
        X10 = torch.empty((nrhs, n), device=dev, dtype=torch.float64).t()
        st10, info10 = 0, {}
        for i in range(2):  # one warm-up solve, one timed
            torch.cuda.synchronize()
            e0.record(stream)
            _, info10, st10 = ops.spd_solve_mixed(A10, B, "emu64", tol=1e-15, max_iter=args.max_iter, X=X10)
            e1.record(stream)
            torch.cuda.synchronize()
            fail_on_status(lib, st10, info10, f"kappa 1e10 solve {i}")
        t10 = e0.elapsed_time(e1) / 1e3
        bwd10 = backward_error(A10, X10, B)
        del X10
        e0.record(stream)
        L, _ = torch.linalg.cholesky_ex(A10)
        Xc = torch.cholesky_solve(B, L)
        e1.record(stream)
        torch.cuda.synchronize()
        tc10 = e0.elapsed_time(e1) / 1e3
        cbwd10 = backward_error(A10, Xc, B)
        del L, Xc, A10
        torch.cuda.empty_cache()
        k10 = {"kappa": 1e10, "precision": "emu64", "ms": t10 * 1e3, "tflops": flops(n, nrhs) / t10 / 1e12,
               "backward_error": bwd10, "converged": info10.get("converged"), "cg_iterations": info10.get("iterations"),
               "factor_ms": info10.get("factor_ms"), "refine_ms": info10.get("refine_ms"),
               "cusolver_ms": tc10 * 1e3, "cusolver_backward_error": cbwd10,
               "speedup_vs_cusolver": tc10 / t10, "speedup_vs_fp64_plain": t64 / t10}

    phase("roofline kernel")
    # Roofline: the dominant kernel, the tcgen05 trailing update (lower SYRK C -= P P^T)
    # at the largest trailing shape of the factorisation, timed with CUDA events on its own
    # stream: first in the configuration the factorisation runs (RC_SYRK_BESIDE, room for a
    # look-ahead CTA on every SM), then in the deeper-ring configuration of a lone call.
    outer = 1024
    rows = n - outer
    peaks = load_peaks()
    prec = 1 if args.precision == "bf16" else 0
    P = torch.randn((rows, outer), device=dev, dtype=torch.float32)
    if prec:
        P = P.bfloat16()
    C = torch.zeros((rows, rows), device=dev, dtype=torch.float32)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    syrk_flops = float(rows) * (rows + 1) * outer

    def time_syrk(flags: int) -> float:
        def syrk():
            _lib.call("rc_syrk_tc_ex", prec, rows, outer, -1.0, ctypes.c_void_p(P.data_ptr()), outer, 1.0,
                      ctypes.c_void_p(C.data_ptr()), rows, flags, sptr)
        for _ in range(3):
            syrk()
        torch.cuda.synchronize()
        reps = 10
        e0.record(stream)
        for _ in range(reps):
            syrk()
        e1.record(stream)
        torch.cuda.synchronize()
        return syrk_flops / (e0.elapsed_time(e1) / 1e3 / reps) / 1e12

    achieved = time_syrk(1)  # RC_SYRK_BESIDE
    achieved_alone = time_syrk(0)
    peak = peaks["bf16_tflops"] if prec else peaks["bf16_tflops"] / 2.0
    # DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from one ncu
    # capture of the TF32 kernel at C = 8192 x 8192, depth 1024, scaled to this shape by
    # the C area it reads and writes ((rows / 8192)^2); not captured for BF16.
    traffic = None if prec else SYRK_TC_DRAM_BYTES_8192 * (rows / 8192.0) ** 2
    del P, C
    torch.cuda.empty_cache()

    # The emulated-FP64 trailing update (the kappa = 1e10 path's dominant kernel) at the same
    # shape: FP64 P and C, 28 int8 digit-pair products per FP64 product.
    P64 = torch.randn((rows, outer), device=dev, dtype=torch.float64)
    C64 = torch.zeros((rows, rows), device=dev, dtype=torch.float64)

    def syrk_emu():
        _lib.call("rc_syrk_emu64", rows, outer, -1.0, ctypes.c_void_p(P64.data_ptr()), outer, 1.0,
                  ctypes.c_void_p(C64.data_ptr()), rows, sptr)
    for _ in range(2):
        syrk_emu()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(5):
        syrk_emu()
    e1.record(stream)
    torch.cuda.synchronize()
    t_emu = e0.elapsed_time(e1) / 1e3 / 5
    del P64, C64
    torch.cuda.empty_cache()
    int8_peak = 2.0 * peaks["bf16_tflops"]
    emu_roof = {"kernel": f"emu_update_kernel (tcgen05 kind::i8, lower SYRK {rows}x{rows}x{outer} in emulated FP64, "
                          "7 digits, 28 digit-pair products)",
                "bound": "tensor", "achieved": 28 * syrk_flops / t_emu / 1e12, "peak": int8_peak, "unit": "TOPS (int8)",
                "frac": 28 * syrk_flops / t_emu / 1e12 / int8_peak, "traffic": None,
                "fp64_equivalent_tflops": syrk_flops / t_emu / 1e12, "ms": t_emu * 1e3,
                "peak_source": "2 x bf16_tflops (the int8 rate is twice the bf16 rate) of "
                               + peaks.get("source", "?") + " peaks",
                "algorithmic": "28 n(n+1)k int8 operations per launch"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        phase("CPU reference sample")
        try:
            r = cpu_reference(args.ref_n, nrhs, steps=1, warmup=0)
            cpu = {"value": r["value"], "unit": "TFLOP/s", "cores": 1, "kind": "reference",
                   "sample": f"Remora CPU cholesky_decomposition + solve, n={args.ref_n}, nrhs={nrhs}, one run",
                   "host_cores": os.cpu_count()}
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": "TFLOP/s", "cores": 1, "kind": "reference", "sample": f"failed: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": world * args.steps * flops(n, nrhs) / t / 1e12,
            "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": ("f64 (factor: fp64 storage, int8 digit-product trailing updates)" if args.precision == "emu64"
                      else "f64 (factor: fp32 storage, " + args.precision + " tensor products)"),
            "data": "synthetic (seeded Q diag(lambda) Q^T, N(0,1) right-hand sides)",
            "config": workload_config(args, world),
            "mixed": {"converged": status_ok, "backward_error": mixed_bwd, "cg_iterations": last["iterations"],
                      "factor_ms": last["factor_ms"], "refine_ms": last["refine_ms"], "shift": last["shift"]},
            "fp64_plain": {"ms": t64 * 1e3, "tflops": flops(n, nrhs) / t64 / 1e12, "backward_error": fp64_bwd,
                           "status": st64},
            "fp64_cusolver": {"ms": tcus * 1e3, "tflops": flops(n, nrhs) / tcus / 1e12, "backward_error": cus_bwd},
            "speedup_vs_fp64_plain": t64 / (t / args.steps),
            "speedup_vs_cusolver": tcus / (t / args.steps),
            "roofline": {"kernel": f"tc_gemm_pair_kernel (tcgen05 cta_group::2, lower SYRK {rows}x{rows}x{outer}, "
                                   f"{args.precision}; the configuration the factorisation runs, RC_SYRK_BESIDE)",
                         "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": "ncu DRAM bytes of the 8192 x 8192 x 1024 launch scaled by C area"
                         if traffic else None,
                         "peak_source": ("bf16_tflops of " if prec else "bf16_tflops/2 (TF32 rate) of ")
                         + peaks.get("source", "?") + " peaks",
                         "algorithmic": "n(n+1)k flops per launch"},
            "roofline_emu64": emu_roof,
            "roofline_alone": {"kernel": "the same kernel in the deeper-ring configuration of a lone rc_syrk_tc call",
                               "achieved": achieved_alone, "peak": peak, "unit": "TFLOP/s",
                               "frac": achieved_alone / peak},
            "kappa_1e10": k10,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        if args.precision == "emu64":  # the headline's dominant kernel is then the digit-product update
            line["roofline_tf32_pair"] = line["roofline"]
            line["roofline"] = emu_roof
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_case(args) -> None:
    """One small case of one kernel, repeated (warm-up + steps): the command the ncu
    captures under profiles/ run. Inputs are larger than L2 where the kernel streams."""
    import torch
    from remora_b200 import _lib, ops
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    sptr = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    reps = args.warmup + args.steps
    if args.case == "syrk_tc":  # the mixed factorisation's trailing update, n x n lower, depth 1024
        n, k = 8192, 1024
        P = torch.randn((n, k), device=dev, dtype=torch.float32)
        if args.precision == "bf16":
            P = P.bfloat16()
        C = torch.zeros((n, n), device=dev, dtype=torch.float32)
        for _ in range(reps):
            _lib.call("rc_syrk_tc", 1 if args.precision == "bf16" else 0, n, k, -1.0, ctypes.c_void_p(P.data_ptr()),
                      k, 1.0, ctypes.c_void_p(C.data_ptr()), n, sptr)
    elif args.case == "syrk_emu":  # the emulated-FP64 trailing update, n x n lower, depth 1024
        n, k = 8192, 1024
        P = torch.randn((n, k), device=dev, dtype=torch.float64)
        C = torch.zeros((n, n), device=dev, dtype=torch.float64)
        for _ in range(reps):
            _lib.call("rc_syrk_emu64", n, k, -1.0, ctypes.c_void_p(P.data_ptr()), k, 1.0,
                      ctypes.c_void_p(C.data_ptr()), n, sptr)
    elif args.case == "dgemm":  # FP64 DMMA GEMM 4096^3
        n = 4096
        A = torch.rand((n, n), device=dev, dtype=torch.float64)
        B = torch.rand((n, n), device=dev, dtype=torch.float64)
        C = torch.zeros((n, n), device=dev, dtype=torch.float64)
        for _ in range(reps):
            ops.gemm(A, B, C, 1.0, 0.0)
    elif args.case == "potrf":  # FP64 blocked Cholesky n = 8192 (diagonal blocks, panels, updates)
        n = 8192
        G = torch.randn((n, n), device=dev, dtype=torch.float64)
        S = G @ G.T / n + torch.eye(n, device=dev, dtype=torch.float64)
        W = torch.empty_like(S)
        for _ in range(reps):
            W.copy_(S)
            ops.potrf(W, sync=False)
    elif args.case == "rng":  # normal fill of 2^28 floats, 16384 x 16384 row-major
        X = torch.empty((16384, 16384), device=dev, dtype=torch.float32)
        for _ in range(reps):
            ops.generate_normal(X, [1, 2, 3, 4], 0.0, 1.0)
    elif args.case == "mixed":  # the headline solve at a reduced size
        A = make_spd(args.n, args.kappa, seed=1234, device=dev)
        B = torch.randn((args.nrhs, args.n), device=dev, dtype=torch.float64).t()
        for _ in range(reps):
            ops.spd_solve_mixed(A, B, args.precision, tol=1e-15, max_iter=args.max_iter)
    elif args.case == "sliced":  # FP64 product on the int8 digit split, 8192 x 8192 times 8192 x 64
        n = 8192
        A = torch.randn((n, n), device=dev, dtype=torch.float64).t()
        P = torch.randn((64, n), device=dev, dtype=torch.float64).t()
        C = torch.zeros((64, n), device=dev, dtype=torch.float64).t()
        for _ in range(reps):
            ops.gemm_sliced(A, P, C, 1.0, 0.0)
    elif args.case == "batched":  # 4096 uneven RBF systems, n ~ U{16..512}
        import numpy as np
        rs = np.random.default_rng(1)
        mats, rhs = [], []
        for n in rs.integers(16, 513, 4096):
            X = rs.standard_normal((n, 8))
            d2 = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
            mats.append(np.exp(-0.5 * d2) + 1e-2 * np.eye(n))
            rhs.append(rs.standard_normal(n))
        sysb = ops.BatchedSystems(mats, rhs)
        a0, b0 = sysb.A.clone(), sysb.b.clone()
        for _ in range(reps):
            sysb.A.copy_(a0)
            sysb.b.copy_(b0)
            sysb.solve()
    torch.cuda.synchronize()
    print(json.dumps({"case": args.case, "reps": reps, "ok": True}))


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=32768)
    ap.add_argument("--nrhs", type=int, default=64)
    ap.add_argument("--kappa", type=float, default=1e2)
    ap.add_argument("--precision", choices=["tf32", "bf16", "emu64"], default="tf32")
    ap.add_argument("--max-iter", type=int, default=200)
    ap.add_argument("--ref-n", type=int, default=4096, help="CPU reference sample size")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-kappa10", action="store_true", help="skip the kappa = 1e10 emu64 solve beside the headline")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--case", choices=["syrk_tc", "syrk_emu", "dgemm", "potrf", "rng", "mixed", "batched", "sliced"],
                    help="run one small kernel case (for ncu captures) instead of the benchmark")
    ap.add_argument("--watchdog", type=float, default=600.0,
                    help="seconds after which a run that has not finished exits with status 3")
    args = ap.parse_args()
    if args.watchdog > 0:
        start_watchdog(args.watchdog)
    if args.case:
        run_case(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
