#!/usr/bin/env python
"""Benchmark of the B^T D A / SpGEMM hot path on B200.

Workload (one "step"): a value refill of C = B^T diag(d) A with a cached pattern,
A 100000 x 50000 and B 100000 x 40000 CSR FP64 with 8 distinct uniform columns per
row (N(0,1) values), d ~ U[0.1, 10]; C is 40000 x 50000 with ~6.39M entries. This is
the configuration the headline metric is quoted on; SparseDiffEngine re-evaluates
the same pattern with new values, so every step brings new A, B and d values.

  value   algorithmic HBM GB/s of the device-resident refill (inputs in HBM),
          L2 flushed between timed steps, CUDA events on the launching stream,
          max over ranks (N > 1 runs one independent product per rank: weak scaling)
  e2e     the same metric through the upstream C ABI with host buffers
          (BTDA_matrices_fill_values on sparse matrix handles: the host->device
          copies of A.x, B.x and d and the device->host copy of C.x are inside the
          timed region)
  roofline / cpu_baseline / clocks / gpu_launches: see the JSON keys.

``--impl reference`` times the upstream CPU implementation (compiled from its own
sources by oracle/Makefile) on the same workload on the host cores (rank 0 only).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="budget of the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-conversions", action="store_true")
    ap.add_argument("--no-dense", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--small-tiles", action="store_true",
                    help="plan the headline product for the small-tile refill (128-thread CTAs, "
                         "512-term tiles) instead of autotuning it (reproducible profiles)")
    ap.add_argument("--refill", choices=["auto", "pipelined", "staged", "direct"], default="auto",
                    help="with --small-tiles: force the pipelined, the staged direct or the plain direct "
                         "tile refill of the headline product (auto: the library's default / the autotuner's "
                         "choice)")
    ap.add_argument("--split-rows", action="store_true",
                    help="N > 1: one headline product split by output rows across the ranks "
                         "(strong scaling) instead of one product per rank (weak scaling)")
    ap.add_argument("--dense-blocks", type=int, default=64,
                    help="blocks of the stacked_pd x CSC case (64 is the configuration; fewer for profiling)")
    ap.add_argument("--learned-matrices", type=int, default=200)
    ap.add_argument("--learned-runs", type=int, default=5,
                    help="new-pattern builds per path in the skewed case (median and spread reported)")
    ap.add_argument("--learned-size", type=int, nargs=2, default=[1_000_000, 20_000_000],
                    metavar=("ROWS", "NNZ"),
                    help="skewed case: rows (= columns) of A and B and their target nonzeros "
                         "(the configuration is 1000000 20000000; smaller for profiling)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the CPU leg's comparison of every sub-result with the oracle")
    ap.add_argument("--stub", action="store_true",
                    help="no GPU: exercise the rank launcher, barrier and max-over-ranks reduction "
                         "on gloo with a placeholder timed region (for CPU tests of the launcher)")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def algorithmic_bytes_refill(nnzA, mA, nnzL, nL, len_d, nnzC):
    """Bytes a refill must move at least once (int32 = 4 B, FP64 = 8 B): A (x, i,
    p), L = CSC of B (row indices, values, column offsets), d, and C (read C.i,
    write C.x): 12 nnz(A) + 4 (m_A + 1) + 12 nnz(L) + 4 (n_L + 1) + 8 len(d) +
    12 nnz(C)."""
    return (12 * nnzA + 4 * (mA + 1) + 12 * nnzL + 4 * (nL + 1) + 8 * len_d + 12 * nnzC)


def design_bytes_refill(nnzL, terms):
    """Bytes this design moves beyond the algorithmic ones, per refill: the CSR
    position of every L entry (B's values are read through it, 4 B), the entry
    values V (written and read, 16 B per entry), the entry records (8 B per entry)
    and the compiled schedule (one 4-byte word per term)."""
    return 4 * nnzL + 16 * nnzL + 8 * nnzL + 4 * terms


class Clocks:
    """nvidia-smi sampler running while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.dev)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but the launcher started {world} rank(s)")
    return world, rank, local


def launch_ranks(args):
    """--gpus N without a torchrun environment: start N ranks of this script, one
    process per GPU, under torch.distributed.run on 127.0.0.1, and return their
    exit status. A hard limit well above the process group's own timeout ends a
    launch whose ranks wait on one another."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           str(Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.call(cmd)


def make_barrier(world, backend="nccl"):
    import torch
    import torch.distributed as dist
    if world <= 1:
        return (lambda: None), (lambda v: v)
    import datetime
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    dev = "cuda" if backend == "nccl" else "cpu"

    def barrier():
        dist.barrier()

    def allmax(v):
        t = torch.tensor([float(v)], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return barrier, allmax


def allsum(v):
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t)
    return float(t.item())


def run_stub(args, world, rank):
    """The launcher and the rank plumbing without a GPU (gloo): every rank takes the
    same barrier / timed region / max-over-ranks steps as the GPU arm; rank 0 prints
    one JSON line whose n_gpus is the number of ranks that ran."""
    barrier, allmax = make_barrier(world, backend="gloo")
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        time.sleep(0.001 * (1 + rank))
    t = allmax((time.perf_counter() - t0) / args.steps)
    seen = int(allmax(rank)) + 1
    barrier()
    if rank == 0:
        print(json.dumps({"metric": "stub", "value": round(world / t, 3), "unit": "steps/s", "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3),
                          "stub": True, "ranks_seen": seen}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------- reference arm
def reference_btda_times(A, B, d, A2x, B2x, d2, reps):
    from oracle import oracle
    lib_path = oracle.REF_DIR / "libsdl_reftime.so"
    if not lib_path.exists():
        raise RuntimeError("upstream timing library not built")
    L = C.CDLL(str(lib_path))
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.ref_time_btda.argtypes = [ip, ip, dp, dp, C.c_int, C.c_int, ip, ip, dp, dp, C.c_int, dp, dp,
                                C.c_int, dp]
    L.ref_time_btda.restype = None
    c = lambda a, t: np.ascontiguousarray(a).ctypes.data_as(C.POINTER(t))  # noqa: E731
    keep = [np.ascontiguousarray(a) for a in (A[0], A[1], A[2], A2x, B[0], B[1], B[2], B2x, d, d2)]
    out = np.zeros(3)
    L.ref_time_btda(c(keep[0], C.c_int), c(keep[1], C.c_int), c(keep[2], C.c_double),
                    c(keep[3], C.c_double), A[3], A[4], c(keep[4], C.c_int), c(keep[5], C.c_int),
                    c(keep[6], C.c_double), c(keep[7], C.c_double), B[4], c(keep[8], C.c_double),
                    c(keep[9], C.c_double), reps, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out  # alloc s, refill s, nnz


def reference_spgemm_times(A, B, reps):
    from oracle import oracle
    L = C.CDLL(str(oracle.REF_DIR / "libsdl_reftime.so"))
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.ref_time_spgemm.argtypes = [ip, ip, dp, C.c_int, C.c_int, ip, ip, dp, C.c_int, C.c_int, dp]
    L.ref_time_spgemm.restype = None
    keep = [np.ascontiguousarray(a) for a in (A[0], A[1], A[2], B[0], B[1], B[2])]
    c = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    out = np.zeros(3)
    L.ref_time_spgemm(c(keep[0], C.c_int), c(keep[1], C.c_int), c(keep[2], C.c_double), A[3], A[4],
                      c(keep[3], C.c_int), c(keep[4], C.c_int), c(keep[5], C.c_double), B[4], reps,
                      out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def reference_csr_to_csc_times(A, reps):
    from oracle import oracle
    L = C.CDLL(str(oracle.REF_DIR / "libsdl_reftime.so"))
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.ref_time_csr_to_csc.argtypes = [ip, ip, dp, C.c_int, C.c_int, C.c_int, dp]
    L.ref_time_csr_to_csc.restype = None
    keep = [np.ascontiguousarray(a) for a in (A[0], A[1], A[2])]
    c = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    out = np.zeros(3)
    L.ref_time_csr_to_csc(c(keep[0], C.c_int), c(keep[1], C.c_int), c(keep[2], C.c_double), A[3], A[4],
                          reps, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out  # alloc s, fill s, nnz


def workload():
    from sparsediff_linalg_b200 import workloads as wl
    A, B, d = wl.btda(seed=1)
    rng = np.random.default_rng(2)
    A2x = rng.standard_normal(len(A[1]))
    B2x = rng.standard_normal(len(B[1]))
    d2 = rng.uniform(0.1, 10.0, A[3])
    return A, B, d, A2x, B2x, d2


WORKLOAD_NAME = ("btda_refill: C = B^T diag(d) A, A 100000x50000, B 100000x40000 CSR FP64, "
                 "8 nnz/row uniform, values N(0,1), d U[0.1,10], new A/B/d values every step")


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    A, B, d, A2x, B2x, d2 = workload()
    nnzC_est = None
    # one step = one upstream refill (CSC mirror refresh + planned fill); warmup first
    t_alloc = None
    times = []
    for phase, reps in (("warmup", max(1, args.warmup)), ("timed", args.steps)):
        out = reference_btda_times(A, B, d, A2x, B2x, d2, reps)
        t_alloc, t_step, nnzC_est = out
        if phase == "timed":
            times.append(t_step)
    t_step = times[0]
    nnzC = int(nnzC_est)
    B_alg = algorithmic_bytes_refill(len(A[1]), A[3], len(B[1]), B[4], A[3], nnzC)
    gbs = B_alg / t_step / 1e9
    line = {
        "impl": "reference", "metric": "btda_refill_hbm_gbs", "value": round(gbs, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_step * 1e3, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": bench_config(nnzC),
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": 1, "kind": "reference",
                         "sample": f"{args.steps} upstream BTDA_matrices_fill_values refills "
                                   f"(A, B, d changed each time) on one host core"},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_alloc_ms": round(t_alloc * 1e3, 3),
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- parity (CPU leg)
def parity_of(got, want_fn, target):
    """Compare a GPU result (p, i, x host arrays) with the oracle's (computed by
    want_fn on the host cores): structure_equal, bit_identical, max_rel_err."""
    from oracle import parallel
    t0 = time.perf_counter()
    want = want_fn()
    cpu_s = time.perf_counter() - t0
    r = parallel.compare_csr(got, want)
    r.update(oracle=target, oracle_s=round(cpu_s, 2), threads=parallel.threads_default())
    return r


def _h(t, n=None):
    a = t.cpu().numpy()
    return a if n is None else a[:n]


L2_NOTE = ("device arm: L2 flushed between timed steps (256 MiB write); "
           "host arm: upstream's CPU refill, no device cache involved")


def bench_config(nnz_C):
    """The workload keys both arms print (the same on the device and host arms)."""
    return {"workload": WORKLOAD_NAME, "nnz_C": int(nnz_C), "l2": L2_NOTE}


# ---------------------------------------------------------------- b200 arm
def run_b200(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    barrier, allmax = make_barrier(world)
    from sparsediff_linalg_b200 import lib, nvtx
    from sparsediff_linalg_b200.device import btda_product, Product
    L = lib()
    assert L.sdl_device_available() == 1, "CUDA library cannot use the device"
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    check = rank == 0 and world == 1 and not args.no_cpu_baseline and not args.no_parity

    A, B, d, A2x, B2x, d2 = workload()
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)  # noqa: E731
    Ap, Ai, Bp, Bi = T(A[0]), T(A[1]), T(B[0]), T(B[1])
    sets = [(T(A[2]), T(B[2]), T(d)), (T(A2x), T(B2x), T(d2))]

    split = args.split_rows and world > 1
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with nvtx.range("bench: headline symbolic"):
        if split:
            # rows r0..r1 of C on this rank (balanced by terms, the same ranges on every
            # rank); A, B and d are read whole, C stays row-partitioned
            from sparsediff_linalg_b200.device import btda_product_rows
            from sparsediff_linalg_b200.sharding import btda_row_weights, row_ranges
            r0, r1 = row_ranges(btda_row_weights(A[0], B[0], B[1], B[4]), world)[rank]
            P, Tr = btda_product_rows(Ap, Ai, A[4], Bp, Bi, B[4], r0, r1)
        else:
            P, Tr = btda_product(Ap, Ai, A[4], Bp, Bi, B[4])
        torch.cuda.synchronize()
    symbolic_ms = (time.perf_counter() - t0) * 1e3
    # the product's plan picked by the autotuner on this pattern (timed refills
    # below run with it); it reports the as-given plan's refill time beside its own
    tune = None
    if args.small_tiles:
        P.replan(tile_budget=512, tile_max_terms=512, refill_threads=128, stream=stream)
        if args.refill != "auto":
            P.set_refill_pipe(args.refill == "pipelined")
            P.set_refill_staged(args.refill == "staged")
        tune = P.tuning()
        torch.cuda.synchronize()
    elif not args.no_autotune:
        tune = P.autotune(reps=5, stream=stream)
        torch.cuda.synchronize()
    Cx = torch.empty(max(1, P.nnz), dtype=torch.float64, device=dev)
    nnz_C = P.nnz
    if split:
        nnz_C = int(round(allsum(P.nnz)))
    B_alg = algorithmic_bytes_refill(len(A[1]), A[3], len(B[1]), B[4], A[3], nnz_C)
    B_design = design_bytes_refill(len(B[1]), P.terms)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    for w in range(args.warmup):
        ax, bx, dd = sets[w % 2]
        P.fill(bx, dd, ax, Cx, stream=stream)
    torch.cuda.synchronize()

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    clk = Clocks(local)
    clk.start()
    launches0 = L.sdl_kernel_launch_count()
    barrier()
    torch.cuda.synchronize()
    with nvtx.range("bench: headline timed refills"):
        for k in range(args.steps):
            ax, bx, dd = sets[k % 2]
            flush.zero_()
            evs[k][0].record(stream)
            P.fill(bx, dd, ax, Cx, stream=stream)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = L.sdl_kernel_launch_count() - launches0
    clocks = clk.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    mean_ms = sum(step_ms) / len(step_ms)
    mean_ms_max = allmax(mean_ms)
    # weak: every rank refills a whole product; split: the ranks share one product
    value = (1 if split else world) * B_alg / (mean_ms_max * 1e-3) / 1e9

    peak, peak_kind = peaks()
    achieved = (B_alg / world if split else B_alg) / (mean_ms * 1e-3) / 1e9
    traffic = None
    tj = ROOT / "profiles" / "btda_refill_traffic.json"
    if tj.exists():
        tr = json.loads(tj.read_text())
        # the capture of the refill this run uses (the autotuner's choice when it ran)
        kind = (tune or {}).get("refill", "direct")
        entry = tr if kind == "direct" else tr.get(kind)
        traffic = entry.get("dram_bytes_per_launch") if isinstance(entry, dict) else None
    headline_parity = None
    if check:
        from oracle import parallel
        last = (args.steps - 1) % 2
        vA = (A[0], A[1], (A[2], A2x)[last], A[3], A[4])
        vB = (B[0], B[1], (B[2], B2x)[last], B[3], B[4])
        headline_parity = parity_of((_h(P.Cp), _h(P.Ci), _h(Cx, P.nnz)),
                                    lambda: parallel.btda(vA, vB, (d, d2)[last]),
                                    "oracle port (oracle/sdl_oracle.c), B^T D A with the last timed step's values")

    # ---- SpGEMM 2000x2000, 5 per row (launch-bound case): symbolic + numeric times
    from sparsediff_linalg_b200 import workloads as wl
    SA, SB = wl.spgemm_small(seed=0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    SP = Product(T(SA[0]), T(SA[1]), T(SB[0]), T(SB[1]), SB[4])
    torch.cuda.synchronize()
    sp_sym_ms = (time.perf_counter() - t0) * 1e3
    SCx = torch.empty(max(1, SP.nnz), dtype=torch.float64, device=dev)
    sax, sbx = T(SA[2]), T(SB[2])
    for _ in range(3):
        SP.fill(sax, None, sbx, SCx, stream=stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(50):
        SP.fill(sax, None, sbx, SCx, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    sp_num_us = e0.elapsed_time(e1) / 50 * 1e3
    spgemm = {"symbolic_ms": round(sp_sym_ms, 3), "numeric_us": round(sp_num_us, 2), "nnz_C": SP.nnz}
    if check:
        from oracle import parallel
        spgemm["parity"] = parity_of((_h(SP.Cp), _h(SP.Ci), _h(SCx, SP.nnz)), lambda: parallel.spgemm(SA, SB),
                                     "oracle port (oracle/sdl_oracle.c)")

    batched = None
    if not args.no_batched:
        with nvtx.range("bench: batched_512"):
            batched = run_batched(args, dev, world, rank, barrier, allmax, check)
    learned = None
    if not args.no_learned and world == 1:
        with nvtx.range("bench: learned_skewed"):
            learned = run_learned(args, dev, check)
    conversions = None
    if not args.no_conversions and world == 1:
        with nvtx.range("bench: conversions"):
            conversions = run_conversions(args, dev, peaks()[0], check)
    dense = None
    if not args.no_dense and world == 1:
        with nvtx.range("bench: stacked_pd"):
            dense = run_dense(args, dev, peaks()[0], check)

    # ---- e2e through the upstream C ABI with host buffers
    e2e = None
    if not args.no_e2e and not split:
        with nvtx.range("bench: e2e"):
            e2e = run_e2e(args, A, B, d, A2x, B2x, d2, B_alg, allmax, barrier, world, check)

    line = {
        "metric": "btda_refill_hbm_gbs", "value": round(value, 3), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(mean_ms_max, 5), "higher_is_better": True,
        "scaling": "strong" if split else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": bench_config(nnz_C),
        "parallelism": (f"one product split by output rows over {world} GPUs" if split else
                        f"{world} independent products (one per GPU)") if world > 1 else "1 GPU",
        "terms": P.terms,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_kind": f"{peak_kind} (copy bandwidth)",
                     "algorithmic_bytes": B_alg,
                     "algorithmic_formula": "12 nnz(A) + 4 (m_A + 1) + 12 nnz(L) + 4 (n_L + 1) + 8 len(d) + 12 nnz(C)",
                     "design_bytes": B_design,
                     "design_bytes_note": "moved beyond the algorithmic bytes: CSR positions of L (4 B/entry), "
                                          "entry values V written + read (16 B/entry), entry records (8 B/entry), "
                                          "schedule words (4 B/term)",
                     "kernel": "numeric refill (all launches of one step)"},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "symbolic_ms": round(symbolic_ms, 3),
        "autotune": tune,
        "spgemm_2000": spgemm,
    }
    if headline_parity is not None:
        line["parity"] = headline_parity
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the same product by the upstream library on one host core (alloc, then fills)
        try:
            r = reference_spgemm_times(SA, SB, 50)
            line["spgemm_2000"]["upstream_cpu"] = {"alloc_ms": round(r[0] * 1e3, 3),
                                                   "fill_us": round(r[1] * 1e6, 2), "nnz_C": int(r[2])}
        except Exception as e:  # the timing library is built with the oracle
            line["spgemm_2000"]["upstream_cpu"] = {"unavailable": str(e)[:200]}
    if e2e is not None:
        line["e2e"] = e2e
    if batched is not None:
        line["batched_512"] = batched
    if learned is not None:
        line["learned_skewed"] = learned
    if conversions is not None:
        line.update(conversions)
    if dense is not None:
        line["stacked_pd_x_csc"] = dense
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, A, B, d, A2x, B2x, d2, B_alg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_e2e(args, A, B, d, A2x, B2x, d2, B_alg, allmax, barrier, world, check=False):
    """The metric through BTDA_matrices_fill_values on sparse matrix handles with
    host value buffers (upstream API, what SparseDiffEngine calls)."""
    import torch
    from sparsediff_linalg_b200.matrices import SparseMatrix
    Am = SparseMatrix.from_csr(*A)
    Bm = SparseMatrix.from_csr(*B)
    Cm = Am.BTA_alloc_with(Bm)
    vals = [(A[2], B[2], np.ascontiguousarray(d)), (A2x, B2x, np.ascontiguousarray(d2))]
    for w in range(args.warmup):
        ax, bx, dd = vals[w % 2]
        Am.set_values(ax)
        Bm.set_values(bx)
        Cm.BTDA_fill(Am, dd, Bm)
    torch.cuda.synchronize()
    barrier()
    t_set, t_fill = [], []
    t0 = time.perf_counter()
    for k in range(args.steps):
        ax, bx, dd = vals[k % 2]
        ta = time.perf_counter()
        Am.set_values(ax)       # host write + matrix_values_changed, as a caller does
        Bm.set_values(bx)
        tb = time.perf_counter()
        Cm.BTDA_fill(Am, dd, Bm)  # returns with C.x current on the host
        t_set.append(tb - ta)
        t_fill.append(time.perf_counter() - tb)
    t = (time.perf_counter() - t0) / args.steps
    t = allmax(t)
    h2d = 8 * (len(A[1]) + len(B[1]) + A[3])
    d2h = 8 * Cm.nnz
    # the host link on this box: page-locked copies of the step's byte counts
    link = {}
    hb = torch.empty(max(h2d, d2h) // 8, dtype=torch.float64).pin_memory()
    db = torch.empty_like(hb, device="cuda")
    for name, nbytes, fn in (("h2d", h2d, lambda n: db[:n].copy_(hb[:n], non_blocking=True)),
                             ("d2h", d2h, lambda n: hb[:n].copy_(db[:n], non_blocking=True))):
        n = nbytes // 8
        fn(n)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            fn(n)
        e1.record()
        torch.cuda.synchronize()
        link[name] = e0.elapsed_time(e1) / 5
    del hb, db
    out = {"value": round(world * B_alg / t / 1e9, 3), "unit": "GB/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "ms_per_step": round(t * 1e3, 4),
           "phases_ms": {"caller_host_writes": round(statistics.median(t_set) * 1e3, 3),
                         "library_fill": round(statistics.median(t_fill) * 1e3, 3),
                         "link_floor": round(link["h2d"] + link["d2h"], 3),
                         "link_gbs": {"h2d": round(h2d / link["h2d"] / 1e6, 1),
                                      "d2h": round(d2h / link["d2h"] / 1e6, 1)}},
           "phases_note": "library_fill = operand uploads + refill + C.x download inside one call; link_floor = "
                          "the same bytes copied between page-locked host memory and the device on this box",
           "api": "BTDA_matrices_fill_values (host value arrays from the library's constructors, "
                  "page-locked in place on their first transfer; d a caller-owned host array)"}
    if check:
        from oracle import parallel
        last = (args.steps - 1) % 2
        ax, bx, dd = vals[last]
        out["parity"] = parity_of(Cm.csr()[:3], lambda: parallel.btda((A[0], A[1], ax, A[3], A[4]),
                                                                        (B[0], B[1], bx, B[3], B[4]), dd),
                                  "oracle port (oracle/sdl_oracle.c), host C after the last e2e step")
    return out


def batch_weights(inst):
    """Terms of every B^T D A instance (its refill cost): sum over rows k of
    nnz(B row k) * nnz(A row k), from the device row offsets."""
    w = []
    for k in inst:
        la = (k["Ap"][1:] - k["Ap"][:-1]).long()
        lb = (k["Bp"][1:] - k["Bp"][:-1]).long()
        w.append(int((la * lb).sum()))
    return w


def run_batched(args, dev, world=1, rank=0, barrier=lambda: None, allmax=lambda v: v, check=False,
                refills=20):
    """512 uneven B^T D A instances (rows log-uniform 1k..64k, cols = rows / 2, 4..16
    nnz per row), fixed patterns, `refills` value refills: batched (grouped
    persistent launches per refill, replayed from a CUDA graph) vs plain (one
    refill per product). Inputs total several GB, far above L2, so no flush is needed.
    With N ranks the products are partitioned by their term counts (LPT, no
    communication) and every rank refills its share; the time is the max over ranks."""
    import torch
    from sparsediff_linalg_b200 import workloads as wl
    from sparsediff_linalg_b200.device import Batch, btda_product
    from sparsediff_linalg_b200.sharding import shard_products
    t0 = time.perf_counter()
    inst_all = wl.batched_device(seed=3, count=512)
    mine = shard_products(batch_weights(inst_all), world)[rank] if world > 1 else list(range(len(inst_all)))
    inst = [inst_all[i] for i in mine]
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    prods, outs = [], []
    B_alg = 0
    for k in inst:
        P, T = btda_product(k["Ap"], k["Ai"], k["n"], k["Bp"], k["Bi"], k["n"])
        prods.append((P, T))
        outs.append(torch.empty(max(1, P.nnz), dtype=torch.float64, device=dev))
        B_alg += algorithmic_bytes_refill(k["Ai"].numel(), k["m"], k["Bi"].numel(), k["n"], k["m"], P.nnz)
    torch.cuda.synchronize()
    sym_s = time.perf_counter() - t0
    Bt = Batch([p for p, _ in prods])
    # two value sets per instance, alternated across refills
    vals = []
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    for k in inst:
        sets = []
        for _ in range(2):
            sets.append((torch.randn(k["Ai"].numel(), generator=g, device=dev, dtype=torch.float64),
                         torch.randn(k["Bi"].numel(), generator=g, device=dev, dtype=torch.float64),
                         torch.rand(k["m"], generator=g, device=dev, dtype=torch.float64) * 9.9 + 0.1))
        vals.append(sets)
    s = torch.cuda.Stream()

    def bind(which):
        for i, k in enumerate(inst):
            ax, bx, d = vals[i][which]
            Bt.bind(i, bx, d, ax, outs[i])

    def timed(fn):
        evs = []
        barrier()
        for r in range(refills):
            bind(r % 2)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                e0.record(s)
                fn(s)
                e1.record(s)
            evs.append((e0, e1))
        s.synchronize()
        return allmax(sum(a.elapsed_time(b) for a, b in evs) / refills)

    tuned = None
    if not args.no_autotune:
        # the group size picked by timing the candidates before the graph exists
        bind(0)
        t0 = time.perf_counter()
        gb, ms_t = Bt.autotune(reps=3, stream=s)
        s.synchronize()
        tuned = {"group_bytes": gb, "refill_ms": round(ms_t, 4), "candidates_mib": [16, 32, 64, 128, 256, "one group"],
                 "tune_s": round(time.perf_counter() - t0, 2)}
    for w in range(3):
        bind(w % 2)
        with torch.cuda.stream(s):
            Bt.refill(stream=s)
            Bt.refill_unbatched(stream=s)
    s.synchronize()
    ms_batched = timed(lambda st: Bt.refill(stream=st))
    ms_plain = timed(lambda st: Bt.refill_unbatched(stream=st))
    terms = sum(p.terms for p, _ in prods)
    B_all = B_alg
    if world > 1:
        B_all = int(round(allsum(B_alg)))
        terms = int(round(allsum(terms)))
    out = {"instances": len(inst_all), "refills": refills, "tiles": Bt.tiles, "groups": Bt.groups,
           "rows": int(sum(k["m"] for k in inst)),
           "nnz_A": int(sum(k["Ai"].numel() for k in inst)), "terms": int(terms),
           "nnz_C": int(sum(p.nnz for p, _ in prods)), "algorithmic_bytes": int(B_all),
           "batched_ms_per_refill": round(ms_batched, 4), "plain_ms_per_refill": round(ms_plain, 4),
           "batched_gbs": round(B_all / (ms_batched * 1e-3) / 1e9, 2),
           "plain_gbs": round(B_all / (ms_plain * 1e-3) / 1e9, 2),
           "speedup_vs_plain": round(ms_plain / ms_batched, 3),
           "generate_s": round(gen_s, 2), "symbolic_s": round(sym_s, 2)}
    if tuned is not None:
        out["autotune"] = tuned
    if world > 1:
        out["ranks"] = world
        out["partition"] = "products by term count (LPT), no collective on the data path; time = max over ranks"
        out["products_this_rank"] = len(inst)
    if check:
        # the batched path once more with the second value set, every product
        # against the oracle
        from oracle import parallel
        bind(1)
        with torch.cuda.stream(s):
            Bt.refill(stream=s)
        s.synchronize()
        t0 = time.perf_counter()

        def one(i):
            k, (P, _) = inst[i], prods[i]
            ax, bx, d = (v.cpu().numpy() for v in vals[i][1])
            got = (_h(P.Cp), _h(P.Ci), _h(outs[i], P.nnz))
            want = parallel.oracle.btda((_h(k["Ap"]), _h(k["Ai"]), ax, k["m"], k["n"]),
                                        (_h(k["Bp"]), _h(k["Bi"]), bx, k["m"], k["n"]), d)
            return parallel.compare_csr(got, want)

        res = parallel.map_threads(one, range(len(inst)))
        bad = [i for i, r in enumerate(res) if not (r["structure_equal"] and r["bit_identical"])]
        errs = [r["max_rel_err"] for r in res]
        out["parity"] = {"structure_equal": all(r["structure_equal"] for r in res),
                         "bit_identical": not bad,
                         "max_rel_err": None if any(e is None for e in errs) else max(errs, default=0.0),
                         "products_checked": len(res), "products_differing": bad[:20],
                         "oracle": "oracle port (oracle/sdl_oracle.c), every product, batched refill output",
                         "oracle_s": round(time.perf_counter() - t0, 2),
                         "threads": parallel.threads_default()}
    return out


def _event_ms(fn, stream, steps, flush=None):
    """Mean device ms of fn(stream) over `steps` runs (CUDA events on `stream`), with
    an L2 flush (256 MiB write) before each run when `flush` is given."""
    import torch
    evs = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn(stream)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs) / steps


_BUILD_NOTE = ("structure_ms: median wall time of 3 builds (structure + first value fill, each build's "
               "device memory freed before the next: returned to the library's block cache, which the "
               "next build allocates from); first_build_ms: the first of them, which also loads the kernels "
               "(CUDA loads modules on first launch) and allocates from the driver")


def _builds(build, runs=3):
    """(last result, median ms, first ms) of `runs` timed builds; the results of the
    earlier builds are released before the next one starts."""
    import torch
    times, res = [], None
    for _ in range(runs):
        res = None
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = build()
        torch.cuda.synchronize()
        times.append((time.perf_counter() - t0) * 1e3)
    return res, float(np.median(times)), times[0]


def run_conversions(args, dev, peak, check=False):
    """CSR -> CSC of a 1M x 1M matrix with 10 distinct uniform columns per row, and
    coalescing of 50M COO triplets over 1M x 1M (35M distinct pairs plus 15M repeats,
    shuffled) into CSR with duplicates summed in input order. Structure (once per
    pattern) and value refill are timed separately; the refill is the recurring cost.
    Algorithmic bytes (int32 = 4 B, FP64 = 8 B): conversion 24 nnz + 4 (m + 1) +
    4 (n + 1); its value refill 20 nnz (x read, CSC values written, position map
    read); coalescing 16 N_in + 12 nnz_out + 4 (m + 1); its value refill 12 N_in +
    8 nnz_out."""
    import torch
    from sparsediff_linalg_b200 import workloads as wl
    from sparsediff_linalg_b200.device import Coalesce, Transpose
    s = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    out = {}
    # ---- 4b: CSR -> CSC
    A = wl.transpose_big(seed=4)
    m, n, nnz = A[3], A[4], len(A[1])
    Ap = torch.as_tensor(A[0], device=dev)
    Ai = torch.as_tensor(A[1], device=dev)
    Ax = torch.as_tensor(A[2], device=dev)
    Tx = torch.empty(nnz, dtype=torch.float64, device=dev)

    def build_t():
        T = Transpose(Ap, Ai, m, n, stream=s)
        T.fill(Ax, Tx, stream=s)
        return T

    T, struct_ms, first_ms = _builds(build_t)
    for _ in range(3):
        T.fill(Ax, Tx, stream=s)
    fill_ms = _event_ms(lambda st: T.fill(Ax, Tx, stream=st), s, args.steps, flush)
    b_fill = 20 * nnz
    b_full = 24 * nnz + 4 * (m + 1) + 4 * (n + 1)
    out["csr_to_csc_1M"] = {
        "workload": "CSR -> CSC, 1M x 1M, 10 distinct uniform columns per row, FP64",
        "nnz": nnz, "structure_ms": round(struct_ms, 3), "first_build_ms": round(first_ms, 3),
        "structure_what": _BUILD_NOTE, "fill_us": round(fill_ms * 1e3, 2),
        "fill_gbs": round(b_fill / (fill_ms * 1e-3) / 1e9, 1),
        "fill_frac_of_hbm": round(b_fill / (fill_ms * 1e-3) / 1e9 / peak, 4),
        "conversion_ms": round(struct_ms, 3),
        "conversion_gbs": round(b_full / (struct_ms * 1e-3) / 1e9, 1),
        "algorithmic_bytes_fill": b_fill, "algorithmic_bytes_conversion": b_full}
    if check:
        from oracle import oracle
        out["csr_to_csc_1M"]["parity"] = parity_of(
            (_h(T.Tp), _h(T.Ti), _h(Tx)), lambda: oracle.transpose(A[0], A[1], A[2], m, n),
            "oracle port (oracle/sdl_oracle.c), whole matrix")
    if not args.no_cpu_baseline:
        try:
            r = reference_csr_to_csc_times(A, 3)
            out["csr_to_csc_1M"]["upstream_cpu"] = {"alloc_ms": round(r[0] * 1e3, 1),
                                                    "fill_ms": round(r[1] * 1e3, 2), "cores": 1}
        except Exception as e:  # noqa: BLE001
            out["csr_to_csc_1M"]["upstream_cpu"] = {"unavailable": str(e)[:200]}
    del T, Ap, Ai, Ax, Tx, A
    torch.cuda.empty_cache()
    # ---- 4c: COO coalescing (the triplets are drawn on the GPU)
    R, Cc, X, m, n = wl.coalesce_device(seed=5, device=dev)
    N = R.numel()

    def build_c():
        CO = Coalesce(R, Cc, m, n, stream=s)
        Cx = torch.empty(max(1, CO.nnz), dtype=torch.float64, device=dev)
        CO.fill(X, Cx, stream=s)
        return CO, Cx

    (CO, Cx), struct_ms, first_ms = _builds(build_c)
    for _ in range(3):
        CO.fill(X, Cx, stream=s)
    fill_ms = _event_ms(lambda st: CO.fill(X, Cx, stream=st), s, args.steps, flush)
    b_fill = 12 * N + 8 * CO.nnz
    b_full = 16 * N + 12 * CO.nnz + 4 * (m + 1)
    out["coo_coalesce_50M"] = {
        "workload": "COO -> CSR with duplicates summed, 50M triplets (35M distinct pairs + 15M "
                    "repeats, shuffled) over 1M x 1M, FP64",
        "triplets": N, "nnz_out": CO.nnz, "structure_ms": round(struct_ms, 3),
        "first_build_ms": round(first_ms, 3), "structure_what": _BUILD_NOTE,
        "fill_us": round(fill_ms * 1e3, 2), "fill_gbs": round(b_fill / (fill_ms * 1e-3) / 1e9, 1),
        "fill_frac_of_hbm": round(b_fill / (fill_ms * 1e-3) / 1e9 / peak, 4),
        "coalesce_gbs": round(b_full / ((struct_ms) * 1e-3) / 1e9, 1),
        "algorithmic_bytes_fill": b_fill, "algorithmic_bytes_coalesce": b_full}
    if check:
        from oracle import parallel
        hr, hc, hx = _h(R), _h(Cc), _h(X)
        out["coo_coalesce_50M"]["parity"] = parity_of(
            (_h(CO.Cp), _h(CO.Ci), _h(Cx, CO.nnz)), lambda: parallel.coalesce(hr, hc, hx, m, n),
            "oracle port (oracle/sdl_oracle.c; equal to upstream row_reduce of the one-triplet-per-row "
            "CSR), all 50M triplets")
    del CO, R, Cc, X, Cx
    torch.cuda.empty_cache()
    return out


def stacked_pd_S(rng, S_n, n0, per_col):
    """S (n0 x S_n CSR) with `per_col` distinct uniform rows in every column: drawn as
    the rows of S^T and transposed with numpy (a stable sort by column)."""
    from sparsediff_linalg_b200 import workloads as wl
    St = wl.fixed_rowlen_csr(S_n, n0, per_col, rng)
    rows_of = np.repeat(np.arange(S_n, dtype=np.int64), np.diff(St[0]))   # column of S
    order = np.argsort(St[1], kind="stable")
    Sp = np.zeros(n0 + 1, np.int32)
    Sp[1:] = np.cumsum(np.bincount(St[1], minlength=n0))
    return Sp, rows_of[order].astype(np.int32), St[2][order]


def reference_ba_spd_csr_times(m, blocks_rows, cperm, X, S, reps):
    from oracle import oracle
    L = C.CDLL(str(oracle.REF_DIR / "libsdl_reftime.so"))
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.ref_time_ba_spd_csr.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, dp, ip, ip, dp, C.c_int,
                                      C.c_int, C.c_int, dp]
    L.ref_time_ba_spd_csr.restype = None
    nb, m0, n0 = X.shape
    keep = [np.ascontiguousarray(a) for a in (blocks_rows, cperm, X, S[0], S[1], S[2])]
    c = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    out = np.zeros(2)
    L.ref_time_ba_spd_csr(m, nb, m0, n0, c(keep[0], C.c_int), c(keep[1], C.c_int), c(keep[2], C.c_double),
                          c(keep[3], C.c_int), c(keep[4], C.c_int), c(keep[5], C.c_double), S[3], S[4], reps,
                          out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def run_dense(args, dev, peak, check=False):
    """stacked_pd x CSC: 64 permuted-dense blocks of 64 x 256 (N(0,1)) whose 4096
    rows are a random permutation, col_perm 0..255, times S 256 x 100000 with 6
    distinct uniform rows per column (upstream BA_spd_csr_*): 64 output blocks of
    64 x 100000, 3.28 GB of FP64 -- bound by writing C. Algorithmic bytes:
    8 sum(m0 n0) + 12 nnz(S) + 4 (n_S + 1) + 8 nnz(C) + 4 sum(n0_C)."""
    import torch
    from sparsediff_linalg_b200.device import BlocksCsr
    rng = np.random.default_rng(6)
    nb, m0, n0, S_n = args.dense_blocks, 64, 256, 100_000
    rows = rng.permutation(nb * m0).astype(np.int32)
    blocks_rows = np.concatenate([np.sort(rows[k * m0:(k + 1) * m0]) for k in range(nb)]).astype(np.int32)
    cperm = np.arange(n0, dtype=np.int32)
    X = rng.standard_normal((nb, m0, n0))
    Sp, Si, Sx = stacked_pd_S(rng, S_n, n0, 6)
    S = (Sp, Si, Sx, n0, S_n)
    t0 = time.perf_counter()
    P = BlocksCsr([m0] * nb, [n0] * nb, [cperm] * nb, Sp, Si, n0, S_n)
    alloc_ms = (time.perf_counter() - t0) * 1e3
    Bv = torch.as_tensor(X.ravel(), device=dev)
    Sx_d = torch.as_tensor(Sx, device=dev)
    Cv = torch.empty(P.c_values, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(3):
        P.fill(Bv, Sx_d, Cv, stream=s)
    steps = max(3, min(args.steps, 10))
    ms = _event_ms(lambda st: P.fill(Bv, Sx_d, Cv, stream=st), s, steps, flush)
    nnzC = P.c_values
    sum_n0C = sum(b[2] for b in P.blocks)
    B_alg = 8 * nb * m0 * n0 + 12 * len(Si) + 4 * (S_n + 1) + 8 * nnzC + 4 * sum_n0C
    out = {"workload": f"stacked_pd ({nb} blocks of 64 x 256, rows permuted) x CSC 256 x 100000 with 6 "
                       "entries per column, FP64", "out_blocks": P.out_blocks, "nnz_C": int(nnzC),
           "alloc_ms": round(alloc_ms, 2), "fill_ms": round(ms, 4),
           "fill_gbs": round(B_alg / (ms * 1e-3) / 1e9, 1),
           "fill_frac_of_hbm": round(B_alg / (ms * 1e-3) / 1e9 / peak, 4), "algorithmic_bytes": int(B_alg),
           "l2": "flushed before each timed fill (256 MiB write); C (3.28 GB) exceeds L2"}
    if check:
        from oracle import oracle, parallel
        got = Cv.cpu().numpy()
        offs = np.concatenate([[0], np.cumsum([b[1] * b[2] for b in P.blocks])])
        t0 = time.perf_counter()

        def one(k):
            src, mk, n0c, perm = P.blocks[k]
            (cols, Cw), = oracle.blocks_csr([(X[src], cperm)], Sp, Si, Sx, S_n)
            Cg = got[offs[k]:offs[k + 1]].reshape(mk, n0c)
            ok = src == k and np.array_equal(perm, cols)
            bits = ok and np.array_equal(Cg.view(np.int64), Cw.view(np.int64))
            err = float(np.max(np.abs(Cg - Cw) / np.maximum(np.abs(Cw), 1e-300))) if ok and not bits else 0.0
            return ok, bits, err

        res = parallel.map_threads(one, range(P.out_blocks))
        out["parity"] = {"structure_equal": all(r[0] for r in res), "bit_identical": all(r[1] for r in res),
                         "max_rel_err": max((r[2] for r in res), default=0.0), "blocks_checked": len(res),
                         "oracle": "oracle restatement of BA_pd_csr (oracle/oracle.py blocks_csr), every block",
                         "oracle_s": round(time.perf_counter() - t0, 2), "threads": parallel.threads_default()}
        del got
    if not args.no_cpu_baseline:
        try:
            r = reference_ba_spd_csr_times(nb * m0, blocks_rows, cperm, X, S, 1)
            out["upstream_cpu"] = {"alloc_ms": round(r[0] * 1e3, 1), "fill_ms": round(r[1] * 1e3, 1),
                                   "cores": 1}
        except Exception as e:  # noqa: BLE001
            out["upstream_cpu"] = {"unavailable": str(e)[:200]}
    del P, Bv, Sx_d, Cv
    torch.cuda.empty_cache()
    out["ata_dmma"] = run_dense_ata(args, dev, X, blocks_rows, cperm, check)
    return out


def reference_atda_spd_times(m, n, blocks_rows, cperm, X, d, reps):
    from oracle import oracle
    L = C.CDLL(str(oracle.REF_DIR / "libsdl_reftime.so"))
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.ref_time_atda_spd.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, dp, dp, C.c_int, dp]
    L.ref_time_atda_spd.restype = None
    nb, m0, n0 = X.shape
    keep = [np.ascontiguousarray(a) for a in (blocks_rows, cperm, X, d)]
    c = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    out = np.zeros(2)
    L.ref_time_atda_spd(m, n, nb, m0, n0, c(keep[0], C.c_int), c(keep[1], C.c_int), c(keep[2], C.c_double),
                        c(keep[3], C.c_double), reps, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def run_dense_ata(args, dev, X, blocks_rows, cperm, check=False):
    """A^T diag(d) A of the same stacked_pd (64 blocks of 64 x 256, col_perm 0..255):
    64 partials of 256 x 256 on the FP64 tensor cores (mma.sync m8n8k4), summed in
    block order into one 256 x 256 block. 2 * 64 * 64 * 256 * 256 flops."""
    import torch
    from sparsediff_linalg_b200.device import BlocksAta
    nb, m0, n0 = X.shape
    m = nb * m0
    rng = np.random.default_rng(7)
    d = rng.uniform(0.1, 10.0, m)
    P = BlocksAta([m0] * nb, [n0] * nb, [blocks_rows[k * m0:(k + 1) * m0] for k in range(nb)], [cperm] * nb,
                  m, n0)
    Xv = torch.as_tensor(X.ravel(), device=dev)
    dd = torch.as_tensor(d, device=dev)
    Cv = torch.empty(P.c_values, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream()
    for _ in range(3):
        P.fill(Xv, dd, Cv, stream=s)
    ms = _event_ms(lambda st: P.fill(Xv, dd, Cv, stream=st), s, max(3, min(args.steps, 10)))
    flops = 2.0 * nb * m0 * n0 * n0
    out = {"workload": "A^T diag(d) A, A the stacked_pd above (64 blocks of 64 x 256), FP64 tensor cores",
           "out_blocks": P.out_blocks, "fill_us": round(ms * 1e3, 2),
           "fp64_tflops": round(flops / (ms * 1e-3) / 1e12, 2), "flops": int(flops)}
    if check:
        from oracle import oracle
        t0 = time.perf_counter()
        want = oracle.blocks_ata([(X[k], blocks_rows[k * m0:(k + 1) * m0], cperm) for k in range(nb)], d, n0)
        got = Cv.cpu().numpy()
        ok, worst, off = len(want) == P.out_blocks, 0.0, 0
        for (rows_g, cols_g), (rows_o, cols_o, Cw, Ca) in zip(P.blocks, want):
            ok = ok and np.array_equal(rows_g, rows_o) and np.array_equal(cols_g, cols_o)
            Cg = got[off:off + Cw.size].reshape(Cw.shape)
            off += Cw.size
            worst = max(worst, float(np.max(np.abs(Cg - Cw) / (Ca + 1e-300))))
        out["parity"] = {"structure_equal": bool(ok), "max_err_over_sum_abs_terms": worst,
                         "within_tol": bool(ok and worst <= 1e-12),
                         "oracle": "numpy A^T diag(d) A per block + upstream's coalescing order "
                                   "(oracle/oracle.py blocks_ata); upstream uses dgemm, so values agree "
                                   "within rounding, bounded by 1e-12 of the sum of |terms|",
                         "oracle_s": round(time.perf_counter() - t0, 2)}
    if not args.no_cpu_baseline:
        try:
            r = reference_atda_spd_times(m, n0, blocks_rows, cperm, X, d, 3)
            out["upstream_cpu"] = {"alloc_ms": round(r[0] * 1e3, 2), "fill_ms": round(r[1] * 1e3, 2),
                                   "blas": "OpenBLAS 0.3.15 (its own threading)"}
        except Exception as e:  # noqa: BLE001
            out["upstream_cpu"] = {"unavailable": str(e)[:200]}
    return out


def run_learned(args, dev, check=False):
    """Skewed SpGEMM C = A B, A and B 1M x 1M with Zipf(1.5) row lengths (~20M nnz
    each, rows capped at 50k), the pattern met for the first time: plain = the exact
    symbolic pass with its refill plan, then the first fill; learned = the one-shot
    pass (rows up to 8192 terms sorted with their values into the network's
    predicted capacity, overflowing rows redone exactly, larger rows by the bitmap
    pass and an accumulating kernel; no refill plan). Each is timed `learned_runs`
    times (median and range reported), each build's device memory freed before the
    next (into the library's block cache, which both paths then allocate from; an
    untimed build of each path runs first). The
    network is trained first on the row statistics of 200 seeded smaller matrices
    of the same recipe. Outputs are compared bit for bit."""
    import torch
    from sparsediff_linalg_b200 import workloads as wl
    from sparsediff_linalg_b200.device import Product
    from sparsediff_linalg_b200.learned import LearnedFilledProduct, LearnedProduct, scratch_bytes
    from sparsediff_linalg_b200.train_scheduler import train
    net, info = train(matrices=args.learned_matrices, epochs=8)
    t0 = time.perf_counter()
    rows, target = args.learned_size
    (Ap, Ai, Ax), (Bp, Bi, Bx), scales = wl.skewed_device(seed=0, m=rows, n=rows, target=target)
    gen_s = time.perf_counter() - t0
    m = Ap.numel() - 1

    def plain():
        P = Product(Ap, Ai, Bp, Bi, m)
        Cx = torch.empty(max(1, P.nnz), dtype=torch.float64, device=dev)
        P.fill(Ax, None, Bx, Cx)
        return P, Cx

    def learned():
        Q = LearnedFilledProduct(Ap, Ai, Bp, Bi, m, net, Ax, None, Bx, margin=0.25)
        return Q, Q.values

    def timed(make, runs):
        ms = []
        out = None
        for _ in range(runs):
            out = None
            torch.cuda.empty_cache()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = make()
            torch.cuda.synchronize()
            ms.append((time.perf_counter() - t0) * 1e3)
        return out, ms

    # one untimed pass of each first (first large allocations and kernel loads)
    for make in (plain, learned):
        w = make()
        torch.cuda.synchronize()
        del w
    runs = max(1, args.learned_runs)
    (P, cx_plain), plain_ms = timed(plain, runs)
    plain_cp, plain_ci = P.Cp.clone(), P.Ci.clone()
    plain_scratch = scratch_bytes(P)
    # the refill of the planned product (a recurring pattern), for reference
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    P.fill(Ax, None, Bx, cx_plain)
    e1.record()
    torch.cuda.synchronize()
    refill_ms = e0.elapsed_time(e1)
    del P
    (Q, cx_learned), learned_ms = timed(learned, runs)
    same = bool(torch.equal(plain_cp, Q.Cp) and torch.equal(plain_ci, Q.Ci) and
                torch.equal(cx_plain[:Q.nnz].view(torch.int64), cx_learned.view(torch.int64)))
    st = Q.stats
    med = lambda v: round(statistics.median(v), 2)  # noqa: E731
    short = lambda v: f"{v // 10**6}M" if v % 10**6 == 0 else f"{v // 1000}k" if v % 1000 == 0 else str(v)  # noqa: E731
    res = {"workload": f"C = A B, A and B {short(rows)} x {short(rows)}, Zipf(1.5) row lengths scaled to "
                       f"~{short(target)} nnz, cap 50k; the pattern met for the first time (structure + first values)",
           "nnz_A": int(Ai.numel()), "nnz_B": int(Bi.numel()), "terms": int(Q.terms),
           "nnz_C": int(Q.nnz), "zipf_scale": [round(x, 6) for x in scales], "runs": runs,
           "plain": {"new_pattern_ms_median": med(plain_ms), "new_pattern_ms_range": [round(min(plain_ms), 2),
                                                                                      round(max(plain_ms), 2)],
                     "what": "exact symbolic pass + refill plan + first fill", "scratch_bytes": int(plain_scratch),
                     "later_refill_ms": round(refill_ms, 3)},
           "learned": {"new_pattern_ms_median": med(learned_ms),
                       "new_pattern_ms_range": [round(min(learned_ms), 2), round(max(learned_ms), 2)],
                       "what": "learned one-shot pass (structure + values, no refill plan)",
                       "scratch_bytes": int(st["scratch_bytes"]), "fallback_rows": st["fallback_rows"],
                       "fallback_terms": st["fallback_terms"],
                       "class_accuracy": round(st["class_hits"] / max(1, st["rows"]), 4),
                       "capacity_over_nnz": round(st["capacity"] / max(1, Q.nnz), 4),
                       "term_bound_over_nnz": round(st["term_bound"] / max(1, Q.nnz), 4)},
           "speedup_new_pattern": round(statistics.median(plain_ms) / statistics.median(learned_ms), 3),
           "identical_structure_and_values": same, "training": info, "generate_s": round(gen_s, 2)}
    if check:
        from oracle import parallel
        hA = (_h(Ap), _h(Ai), _h(Ax), m, m)
        hB = (_h(Bp), _h(Bi), _h(Bx), m, m)
        res["parity"] = parity_of((_h(Q.Cp), _h(Q.Ci), _h(cx_learned)), lambda: parallel.spgemm(hA, hB),
                                  "oracle port (oracle/sdl_oracle.c), whole product, learned one-shot output")
    del Q, cx_learned, cx_plain
    torch.cuda.empty_cache()
    _ = LearnedProduct  # the scratch-sizing learned symbolic pass stays available
    return res


def cpu_baseline(args, A, B, d, A2x, B2x, d2, B_alg):
    try:
        # estimate the refill time with a couple of reps, then size the sample
        est = reference_btda_times(A, B, d, A2x, B2x, d2, 2)[1]
        reps = int(max(3, min(500, args.cpu_seconds / max(est, 1e-4))))
        out = reference_btda_times(A, B, d, A2x, B2x, d2, reps)
        return {"value": round(B_alg / out[1] / 1e9, 4), "unit": "GB/s", "cores": 1,
                "kind": "reference", "ms_per_step": round(out[1] * 1e3, 3),
                "alloc_ms": round(out[0] * 1e3, 2), "host_cores": os.cpu_count(),
                "sample": f"{reps} refills of the same workload by the upstream library "
                          f"(BTDA_matrices_fill_values), single-threaded"}
    except Exception as e:  # the port is the fallback checker
        return {"value": None, "unit": "GB/s", "cores": 1, "kind": "reference",
                "sample": f"unavailable: {e}"}


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args)
    world, rank, local = dist_setup(args)
    if args.stub:
        return run_stub(args, world, rank)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_b200(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
