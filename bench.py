"""Benchmark: µs per exact negacyclic product at N = 65536, W = 2048 (q a seeded
random odd 2048-bit modulus, 64 limbs, K = 139 primes below 2^30), on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload N65536_W2048|N65536_W1747|N32768_W868|N4096_W256]

A step is one product c = a b mod (X^N + 1, q) on one GPU.  Multi-GPU runs
(torchrun, one process per GPU) are replicas: each rank multiplies its own
operands, with no collective on the data path ("scaling": "weak"); the value is
the whole job's time per product, max over ranks of the device time divided by
all ranks' products.

value  : device-only, operands resident in HBM; four operand sets rotate so the
         inputs of consecutive steps (4 x 50 MB) are larger than L2 (126 MB).
e2e    : the same product through the public C API with host buffers
         (fpm_run: host->device copies of a and b, device->host copy of c,
         inside the timed region), wall clock.
roofline: the dominant kernel's algorithmic bytes per launch over its CUDA-event
         duration, against the measured HBM copy bandwidth.
cpu_baseline: the reference's own CPU implementation (solve_cpu.cpp, OpenMP,
         built into oracle/_ref/) on a bounded sample, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "fherma-polymult_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOADS = {
    "N65536_W2048": (65536, 2048),
    "N65536_W1747": (65536, 1747),
    "N32768_W868": (32768, 868),
    "N4096_W256": (4096, 256),
}
METRIC = "µs per N=65536 2048-bit exact product"
ROTATE = 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="N65536_W2048")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def metric_name(workload):
    N, W = WORKLOADS[workload]
    return METRIC if (N, W) == (65536, 2048) else f"µs per N={N} {W}-bit exact product"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = max(smax, float(f[2]))
                except ValueError:
                    continue
                for name, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        finally:
            os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(N, L, K):
    """Per product and per stage launch, from the six-pass RNS schedule with
    twiddles cache-resident: decompose reads N L and writes K N words per
    operand; the column pass reads and writes both operands' residues (4 K N);
    the fused row pass reads 2 K N and writes K N; the inverse column pass reads
    and writes K N each; the CRT reads K N and writes N L."""
    w = 4
    return {
        "decompose": w * (N * L + K * N),
        "ntt_col_fwd": w * 4 * K * N,
        "ntt_row": w * 3 * K * N,
        "ntt_col_inv": w * 2 * K * N,
        "crt": w * (K * N + N * L),
        "product": w * (3 * N * L + 12 * K * N),
    }


def run_reference(args):
    """The reference's own CPU implementation (solve_cpu.cpp via the shim in
    oracle/_ref/libref_cpu.so), all host threads, same workload and metric."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    N, W = WORKLOADS[args.workload]
    import oracle
    from polymul import workload
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_cpu.so was not built "
                                                                "(reference tree absent when building)"}))
        return
    q, a, b = workload.case(N, W, "uniform", seed=1000 * 3 + 1)
    cores = os.cpu_count() or 1
    _, secs = oracle.ref_polymul(N, W, q, a, b, reps=args.warmup + args.steps)
    t = secs[args.warmup:]
    us = 1e6 * sum(t) / len(t)
    line = {
        "metric": metric_name(args.workload), "value": us, "unit": "us/product", "impl": "reference",
        "n_gpus": args.gpus, "steps": len(t), "warmup": args.warmup, "ms_per_step": us / 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded PCG64: random odd W-bit q, operands uniform in [0, q))",
        "config": {"workload": args.workload, "N": N, "W": W, "L": q.shape[0], "parallelism": "none (CPU)"},
        "cpu_baseline": {"value": us, "unit": "us/product", "cores": cores, "kind": "reference",
                         "sample": f"{len(t)} products at N={N} W={W}, reference solve_cpu.cpp (OpenMP, "
                                   f"{cores} threads), steady_clock around fherma_run"},
        "e2e": {"value": us, "unit": "us/product", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch

    import polymul
    from polymul import workload

    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    N, W = WORKLOADS[args.workload]
    L = (W + 31) // 32

    # Operand sets (same q; rank-dependent seeds).
    q, _, _ = workload.case(2, W, "zero", seed=3000 + 1)
    rng = np.random.Generator(np.random.PCG64(4000 + rank))
    sets_h = [(workload.uniform_below(q, N, rng), workload.uniform_below(q, N, rng)) for _ in range(ROTATE)]

    def todev(x):
        return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda()

    sets_d = [(todev(a), todev(b), torch.empty((N, L), dtype=torch.int32, device="cuda")) for a, b in sets_h]
    ctx = polymul.Context(N, W, q)
    K = ctx.K
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    launches_per_product = 4 if ctx.info.logN <= 10 else (5 if ctx.info.logR == 0 else 6)

    def step(i):
        da, db, dc = sets_d[i % ROTATE]
        ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sp)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
    stream.synchronize()

    # Per-stage timing (dominant kernel for the roofline), outside the main region.
    A = torch.empty((K, N), dtype=torch.int32, device="cuda")
    B = torch.empty((K, N), dtype=torch.int32, device="cuda")
    stages = {}

    def time_stage(fn, reps=10):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        fn()
        stream.synchronize()
        ev[0].record(stream)
        for _ in range(reps):
            fn()
        ev[1].record(stream)
        ev[1].synchronize()
        return ev[0].elapsed_time(ev[1]) / reps * 1e3   # us

    da, db, dc = sets_d[0]
    stages["decompose"] = time_stage(lambda: ctx.stage_decompose(da.data_ptr(), A.data_ptr(), 0, sp))
    ctx.stage_decompose(db.data_ptr(), B.data_ptr(), 1, sp)
    stages["transform"] = time_stage(lambda: ctx.stage_transform(A.data_ptr(), B.data_ptr(), 0, sp))
    stages["crt"] = time_stage(lambda: ctx.stage_crt(A.data_ptr(), dc.data_ptr(), sp))
    # One kernel at a time (the transform's passes alone: modes 2, 3, 4).
    kernels = {"k_decompose_tc": stages["decompose"], "k_crt_tc": stages["crt"]}
    if ctx.info.logR:
        kernels["k_ntt_col_fwd"] = time_stage(lambda: ctx.stage_transform(A.data_ptr(), B.data_ptr(), 2, sp))
        kernels["k_ntt_col_inv"] = time_stage(lambda: ctx.stage_transform(A.data_ptr(), B.data_ptr(), 4, sp))
    kernels["k_ntt_row"] = time_stage(lambda: ctx.stage_transform(A.data_ptr(), B.data_ptr(), 3, sp))

    # Timed region.
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        start.record(stream)
        for i in range(args.steps):
            step(i)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms = start.elapsed_time(end)
    clocks = clk.summary()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    products = args.steps * world
    us_per_product = ms * 1e3 / products

    # End to end through the C API with host buffers (fpm_run): pinned buffers
    # (the headline: host->device copies of a and b and the device->host copy of
    # c inside every timed step), and the same with pageable numpy buffers.
    a_h, b_h = sets_h[0]

    def pinned(x):
        t = torch.empty(x.shape, dtype=torch.int32, pin_memory=True)
        v = t.numpy().view(np.uint32)
        v[...] = x
        return t, v

    a_pt, a_p = pinned(a_h)
    b_pt, b_p = pinned(b_h)
    c_pt, c_p = pinned(np.zeros((N, L), np.uint32))

    def e2e(a_, b_, c_, n):
        ctx.run(a_, b_, c_)
        t0 = time.perf_counter()
        for _ in range(n):
            ctx.run(a_, b_, c_)
        return (time.perf_counter() - t0) * 1e6 / n

    e2e_us = e2e(a_p, b_p, c_p, args.e2e_steps)
    c_h = np.empty((N, L), np.uint32)
    e2e_pageable_us = e2e(a_h, b_h, c_h, args.e2e_steps)

    hbm, peak_kind = peaks()
    ab = algorithmic_bytes(N, L, K)
    kernel_bytes = {"k_decompose_tc": ab["decompose"], "k_ntt_col_fwd": ab["ntt_col_fwd"], "k_ntt_row": ab["ntt_row"],
                    "k_ntt_col_inv": ab["ntt_col_inv"], "k_crt_tc": ab["crt"]}
    # launches per product: the dominant kernel's time share in one product
    per_product = {"k_decompose_tc": 2, "k_ntt_col_fwd": 1, "k_ntt_row": 1, "k_ntt_col_inv": 1, "k_crt_tc": 1}
    dom = max(kernels, key=lambda k: kernels[k] * per_product[k])
    achieved = kernel_bytes[dom] / (kernels[dom] * 1e-6) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f)
        entry = tr.get(args.workload, {}).get(dom)
        if entry:
            traffic = entry["dram_bytes_per_launch"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            if oracle.ref_available():
                reps = 3
                _, secs = oracle.ref_polymul(N, W, q, a_h, b_h, reps=reps)
                cores = os.cpu_count() or 1
                cpu = {"value": 1e6 * statistics.median(secs), "unit": "us/product", "cores": cores,
                       "kind": "reference",
                       "sample": f"{reps} products at N={N} W={W} (median), the reference's solve_cpu.cpp "
                                 f"(OpenMP, {cores} threads)"}
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "unit": "us/product", "cores": None, "kind": "reference",
                   "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": metric_name(args.workload),
            "value": us_per_product,
            "unit": "us/product",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u32",
            "data": "synthetic (seeded PCG64: random odd W-bit q, operands uniform in [0, q))",
            "config": {"workload": args.workload, "N": N, "W": W, "L": L, "K": K,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": f"{ROTATE} operand sets rotate ({ROTATE * 3 * N * L * 4 / 1e6:.0f} MB > 126 MB L2)"},
            "products_per_s": 1e6 / us_per_product,
            "e2e": {"value": e2e_us, "unit": "us/product", "h2d_bytes_per_step": 2 * N * L * 4,
                    "d2h_bytes_per_step": N * L * 4, "host_buffers": "pinned (fpm_run, wall clock)"},
            "e2e_pageable": {"value": e2e_pageable_us, "unit": "us/product",
                             "host_buffers": "pageable numpy (fpm_run stages through pinned memory)"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes": kernel_bytes[dom],
                         "note": "algorithmic bytes per launch / CUDA-event launch time; traffic = ncu dram "
                                 "read+write per launch from profiles/ncu_traffic.json"},
            "stages_us": stages,
            "kernels_us": kernels,
            "product_algorithmic_bytes": ab["product"],
            "product_hbm_frac": ab["product"] / (us_per_product * world * 1e-6) / 1e9 / hbm,
            "gpu_launches": args.steps * launches_per_product,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
