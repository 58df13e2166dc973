#!/usr/bin/env python
"""Benchmark: KPM moments/s of the B200 engine on the TMD-lattice KPM workload.

Workload ("kpm_tmd_200x200"): TMD-like triangular-lattice tight-binding
Hamiltonian, 200 x 200 periodic supercell, one 5-orbital metal and two
3-orbital chalcogen sites per cell (N = 440,000 scalar rows, 1.4 M blocks,
nnz = 2.0e7), hopping blocks ~N(0, 0.5), on-site ~N(0, 0.2), rescaled into
[-0.95, 0.95]; 1024 Chebyshev moments of 64 random +-1 vectors held as one
multivector.  One step = one full moment computation (the fused two-moment
recurrence: 512 SpMM + moment-dot passes), inputs resident in HBM; the
working set (160 MB of values + 3 x 225 MB of vectors) exceeds the 126 MB L2,
so no flush is needed between steps.

Reported: ``value`` = moment-vectors/s of the plain FP64 drop-in path
(whole job, all ranks), ``fp32_bulk`` = the FP32-storage / FP64-sum path and
its DOS error, ``roofline`` of the fused Chebyshev SpMM kernel against the
measured HBM copy bandwidth, ``e2e`` = the same metric through the host-buffer
C-ABI call (random vectors copied in, moments copied out every step),
``spmv`` = the 5000-block FP64 SpMV (100 repeats) in GB/s, ``cpu_baseline`` =
the reference's own OpenMP C++ core on the host cores.

Multi-GPU (torchrun): every rank computes the moments of its own 64 vectors
with H replicated (weak scaling) and the moments are summed with one NCCL
all-reduce per step.  ``--impl reference`` times the reference's CPU core on
the same workload (rank 0 only).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "kpm_tmd_200x200"
METRIC = "KPM moments/s (moment x random-vector per second)"
UNIT = "moment-vectors/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--L", type=int, default=200)
    p.add_argument("--R", type=int, default=64)
    p.add_argument("--M", type=int, default=1024)
    p.add_argument("--cpu-moments", type=int, default=24, help="moments in the bounded CPU sample")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-spmv", action="store_true")
    p.add_argument("--only", default="all", choices=["all", "cheb", "spmv"],
                   help="profile one kernel: 'cheb' runs only the fused Chebyshev step (steps launches after "
                        "warmup), 'spmv' only the 5000-block SpMV; prints a short JSON line")
    return p.parse_args()


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxs.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxs), "reasons": sorted(reasons),
                "samples": len(sms)}


def build_workload(L):
    from vbcsr_b200 import workloads as W

    H, g = W.tmd_lattice(L, seed=2)
    return H, g


def rademacher(N, R, seed):
    rng = np.random.default_rng(seed)
    return np.where(rng.random((N, R)) < 0.5, -1.0, 1.0)


def algorithmic_bytes_cheb(H, ld, es):
    """Compulsory bytes of one fused Chebyshev step Y = 2 A X - Xprev (+ dots):
    values + column indices + row pointers once, X, Xprev read and Y written once."""
    return es * H.nnz + 4 * H.nnzb + 4 * (H.n + 1) + 3 * es * H.N * ld


def spmv_bench(args, torch, _capi, stream, sp, timed, hbm):
    """FP64 SpMV y = A x on the 5000-block-row random symmetric matrix (block
    sizes 4..8, ~12 mirrored neighbours per row), 100 repeated mults: L2
    flushed before each (the 19 MB working set fits in L2) and warm."""
    from vbcsr_b200 import workloads as W

    vp = C.c_void_p
    A = W.random_symmetric_blocks(5000, seed=1)
    da = _capi.DeviceMatrix.create(A.block_sizes, A.row_ptr, A.col_ind, A.values)
    x = torch.from_numpy(np.random.default_rng(1).normal(size=A.N)).cuda()
    y = torch.zeros_like(x)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def mv():
        _capi.call("vbg_spmv", da.h, vp(x.data_ptr()), vp(y.data_ptr()), sp)

    ms_warm = timed(mv, 100, 5)
    tot = 0.0
    for _ in range(100):
        flush.zero_()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        mv()
        a1.record(stream)
        a1.synchronize()
        tot += a0.elapsed_time(a1)
    ms_cold = tot / 100
    b = 8 * A.nnz + 4 * A.nnzb + 4 * (A.n + 1) + 16 * A.N
    return {"workload": "random_symmetric_5000_blocks_4to8", "N": A.N, "nnz": A.nnz,
            "algorithmic_bytes": b, "ms_l2_flushed": ms_cold, "gbs_l2_flushed": b / (ms_cold / 1e3) / 1e9,
            "frac_l2_flushed": b / (ms_cold / 1e3) / 1e9 / hbm, "ms_warm": ms_warm,
            "gbs_warm": b / (ms_warm / 1e3) / 1e9}


def cpu_reference_kpm(H, V, M, threads):
    from oracle.oracle import Reference

    ref = Reference(threads=threads)
    t0 = time.perf_counter()
    R = ref.matrix(H)
    t_build = time.perf_counter() - t0
    R.kpm_moments(V, 2)  # warm
    t0 = time.perf_counter()
    mu = R.kpm_moments(V, M)
    dt = time.perf_counter() - t0
    return dt, mu, t_build, ref.threads()


def run_reference(args, rank):
    if rank != 0:
        return
    from oracle.oracle import reference_available

    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvbcsr_ref.so was not built"}))
        return
    H, _ = build_workload(args.L)
    V = rademacher(H.N, args.R, 1234)
    threads = os.cpu_count() or 1
    from oracle.oracle import Reference

    ref = Reference(threads=threads)
    R = ref.matrix(H)
    Ms = max(4, args.cpu_moments)
    for _ in range(args.warmup):
        R.kpm_moments(V, 3)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        R.kpm_moments(V, Ms)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    value = args.R * Ms / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": f"{args.L}x{args.L}", "N": H.N, "nnz": H.nnz,
                   "nnzb": H.nnzb, "random_vectors": args.R, "moments_per_step": Ms,
                   "recurrence": "ex08 three-term (one SpMM per moment)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.threads(), "kind": "reference",
                         "sample": f"{Ms} moments x {args.R} vectors of the full workload per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    from vbcsr_b200 import _capi
    from vbcsr_b200 import kpm as K

    vp = C.c_void_p
    H, g = build_workload(args.L)
    dm = _capi.DeviceMatrix.create(H.block_sizes, H.row_ptr, H.col_ind, H.values)
    R, M = args.R, args.M
    ld = ((R * 8 + 63) // 64) * 8 if R > 1 else 1
    V = rademacher(H.N, R, 1234 + rank)
    V0 = torch.zeros((H.N, ld), dtype=torch.float64, device="cuda")
    V0[:, :R] = torch.from_numpy(V).cuda()
    mu64 = torch.zeros(M, dtype=torch.float64, device="cuda")
    mu32 = torch.zeros(M, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    sp = vp(stream.cuda_stream)

    def kpm(prec, out):
        _capi.call("vbg_kpm_moments", dm.h, R, ld, vp(V0.data_ptr()), M, prec, 1, 1, vp(out.data_ptr()), sp)
        if dist is not None:
            dist.all_reduce(out)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        if dist is not None:
            t = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    hbm, peak_kind = peaks()
    if args.only == "cheb":
        X1 = torch.zeros_like(V0)
        X2 = torch.zeros_like(V0)
        dots = torch.zeros(2, dtype=torch.float64, device="cuda")
        ms = timed(lambda: _capi.call("vbg_cheb_step", dm.h, R, ld, 2.0, 0.0, -1.0, vp(V0.data_ptr()),
                                      vp(X1.data_ptr()), vp(X2.data_ptr()), None, vp(dots.data_ptr()), None,
                                      0.0, 0.0, sp), args.steps, args.warmup)
        b = algorithmic_bytes_cheb(H, ld, 8)
        if rank == 0:
            print(json.dumps({"only": "cheb", "ms": ms, "algorithmic_bytes": b, "gbs": b / (ms / 1e3) / 1e9,
                              "frac": b / (ms / 1e3) / 1e9 / hbm}))
        return
    if args.only == "spmv":
        if rank == 0:
            print(json.dumps({"only": "spmv", **spmv_bench(args, torch, _capi, stream, sp, timed, hbm)}))
        return

    # launches per moment computation: sumsq + 1 + (M-2)//2 applies + finalize (one pipelined launch per apply)
    launches_per_step = 1 + (1 + (M - 2) // 2) + 1

    with ClockSampler(local_rank) as clk:
        ms64 = timed(lambda: kpm(0, mu64), args.steps, args.warmup)
    clocks = clk.summary()
    ms32 = timed(lambda: kpm(1, mu32), args.steps, args.warmup)
    value64 = world * R * M / (ms64 / 1e3)
    value32 = world * R * M / (ms32 / 1e3)

    # DOS error of the FP32 path against FP64 on the same vectors
    n_norm = world * R * H.N
    _, d64 = K.dos_from_moments(mu64.cpu().numpy() / n_norm, 2000)
    _, d32 = K.dos_from_moments(mu32.cpu().numpy() / n_norm, 2000)
    dos_err = float(np.abs(d32 - d64).max() / np.abs(d64).max())

    # roofline of the fused Chebyshev step (one launch of the pipelined kernel)
    X1 = torch.zeros_like(V0)
    X2 = torch.zeros_like(V0)
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")

    def cheb():
        _capi.call("vbg_cheb_step", dm.h, R, ld, 2.0, 0.0, -1.0, vp(V0.data_ptr()), vp(X1.data_ptr()),
                   vp(X2.data_ptr()), None, vp(dots.data_ptr()), None, 0.0, 0.0, sp)

    n_cheb = 50
    ms_cheb = timed(cheb, n_cheb, 3)
    bytes_cheb = algorithmic_bytes_cheb(H, ld, 8)
    achieved = bytes_cheb / (ms_cheb / 1e3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic_cheb_step_fp64.txt"
    if tf.exists():
        for ln in tf.read_text().splitlines():
            if ln.startswith("bytes_per_step="):
                traffic = float(ln.split("=", 1)[1])

    # end to end through the host-buffer C ABI: V0 host (pinned) -> moments host
    Vh = torch.from_numpy(V).pin_memory()
    muh = np.zeros(M)

    def e2e():
        _capi.call("vbg_kpm_moments_host", dm.h, R, vp(Vh.data_ptr()), M, 0, 1,
                   muh.ctypes.data_as(vp), sp)

    ms_e2e = timed(e2e, max(2, args.steps // 2), 1)
    e2e_value = world * R * M / (ms_e2e / 1e3)

    # FP64 SpMV, 5000 random symmetric blocks, 100 repeated mults
    spmv = None if args.no_spmv else spmv_bench(args, torch, _capi, stream, sp, timed, hbm)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle.oracle import reference_available

        if reference_available():
            Ms = max(4, args.cpu_moments)
            dt, _, _, thr = cpu_reference_kpm(H, V, Ms, os.cpu_count())
            cpu = {"value": R * Ms / dt, "unit": UNIT, "cores": thr, "kind": "reference",
                   "sample": f"{Ms} moments x {R} vectors of the same workload (ex08 three-term recurrence "
                             f"on the reference DistMultiVector ops), {dt:.1f} s"}

    line = {
        "metric": METRIC, "value": value64, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": f"{args.L}x{args.L}", "N": H.N, "nnz": H.nnz, "nnzb": H.nnzb,
                   "random_vectors_per_gpu": R, "moments": M, "recurrence": "two moments per SpMM (512 SpMMs)",
                   "cuda_graph": True, "l2": "inputs larger than L2 (no flush)"},
        "fp32_bulk": {"value": value32, "ms_per_step": ms32, "speedup_vs_fp64": value32 / value64,
                      "dos_err_vs_fp64": dos_err},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "kernel": "apply_pipe_kernel (fused Chebyshev step, FP64, k=64)",
                     "algorithmic_bytes_per_step": bytes_cheb, "ms_per_step": ms_cheb, "peak_kind": peak_kind},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(V.nbytes), "d2h_bytes_per_step": 8 * M,
                "ms_per_step": ms_e2e},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "spmv": spmv,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
