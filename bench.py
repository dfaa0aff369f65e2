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
         inside the timed region), wall clock per call, median of 50 calls.
roofline: the dominant kernel's algorithmic bytes per launch over its CUDA-event
         duration, against the measured HBM copy bandwidth.
cpu_baseline: the reference's own CPU implementation (solve_cpu.cpp, OpenMP,
         built into oracle/_ref/) on a bounded sample, rank 0 only.
batched: 64 products of the uneven mix (N 4096 .. 65536, W 128 .. 2048) as one
         autotuned graph of grouped launches, against 64 sequential plain calls
         (device against device, host against host); stage_launch_layout is
         the five-launch schedule (one grouped launch per stage) timed alike;
         batched_n65536: the same for 16 products at N = 65536 (W 1747 / 2048).
serving: a seeded Poisson stream (10,000 requests at 2000/s) through the
         serving loop; p50 / p99 latency and products/s.
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
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="N65536_W2048")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--no-configs", action="store_true", help="skip timing the other benchmark points")
    ap.add_argument("--sustained-s", type=float, default=1.0,
                    help="seconds of back-to-back products for the sustained figure (0: skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (64-product mix) measurement")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving (Poisson stream) measurement")
    ap.add_argument("--serve-requests", type=int, default=10000)
    ap.add_argument("--serve-rate", type=float, default=2000.0)
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
    """SM clocks and clock-event (throttle) reasons, read through NVML back to
    back (about every 0.2 ms) on a background thread while the timed region
    runs (the same data as nvidia-smi's clocks.sm and clocks_event_reasons.*
    queries)."""

    NAMES = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
             "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
             "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
             "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, index: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        self.index = int(ids[index]) if index < len(ids) and ids[index].isdigit() else index
        self.sm, self.smax, self.reasons = [], 0.0, set()
        self.error = None
        self._stop = None
        self._thread = None

    def _run(self):
        import pynvml
        h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        bits = {name: getattr(pynvml, const) for name, const in self.NAMES.items()}
        while not self._stop.is_set():
            self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
            r = get_reasons(h)
            for name, bit in bits.items():
                if r & bit:
                    self.reasons.add(name)
            self._stop.wait(0.0002)

    def __enter__(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
        except Exception as e:   # the record is reported, not required
            self.error = str(e)
            return self
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._guarded, daemon=True)
        self._thread.start()
        while not self.sm and not self.error and self._thread.is_alive():
            time.sleep(0.001)   # the first sample is in before the region starts
        return self

    def _guarded(self):
        try:
            self._run()
        except Exception as e:
            self.error = str(e)

    def __exit__(self, *exc):
        if self._thread:
            self._stop.set()
            self._thread.join()

    def summary(self):
        out = {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.smax or None,
               "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "NVML, back to back"}
        if self.error:
            out["error"] = self.error
        return out


def algorithmic_bytes(N, L, K):
    """Per product and per stage launch, from the six-pass RNS schedule with
    twiddles cache-resident (B_alg = 4 (3 N L + 12 K N)): decompose reads N L
    and writes K N words per operand; the column pass reads and writes both
    operands' residues (4 K N); the fused row pass reads 2 K N and writes K N;
    the inverse column pass reads and writes K N each; the CRT reads K N and
    writes N L.  The row pass's prebuilt twiddle tables (K N Shoup pairs) are
    this design's own extra traffic, reported beside the algorithmic bytes."""
    w = 4
    return {
        "decompose": w * (N * L + K * N),
        "ntt_col_fwd": w * 4 * K * N,
        "ntt_row": w * 3 * K * N,
        "ntt_col_inv": w * 2 * K * N,
        "crt": w * (K * N + N * L),
        "product": w * (3 * N * L + 12 * K * N),
        "row_tables": 8 * K * N,
    }


def job_time(ms_local: float, steps: int, world: int, reduce_max):
    """Whole-job time of a replica run: every rank multiplies `steps` products
    of its own, so the job takes as long as the slowest rank (max over ranks of
    the device time) and the value is that time over all ranks' products.
    Returns (ms, us per product)."""
    ms = float(reduce_max(ms_local)) if world > 1 else float(ms_local)
    return ms, ms * 1e3 / (steps * world)


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


def pinned_like(torch, x):
    """A pinned host copy of x (u32), kept alive by the returned tensor."""
    t = torch.empty(x.shape, dtype=torch.int32, pin_memory=True)
    v = t.numpy().view(np.uint32)
    v[...] = x
    return t, v


def n65536_points(count, seed):
    """N = 65536 with a 1747-bit or a 2048-bit modulus (alternating), each q
    seeded: the large single products as a batch."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [(65536, (1747, 2048)[i % 2], None) for i in range(count)], rng


# The other benchmark points (N, W) and their value distributions.
CONFIG_POINTS = [
    ("N4096_W256", "uniform"),
    ("N32768_W868", "uniform"), ("N32768_W868", "max"), ("N32768_W868", "sparse"),
    ("N65536_W1747", "uniform"), ("N65536_W1747", "max"),
    ("N65536_W2048", "uniform"), ("N65536_W2048", "max"),
]


def measure_point(torch, polymul, workload, name, dist, stream, hbm, steps=30, e2e_steps=20):
    """One benchmark point: device time per product (CUDA events around each
    product, L2 flushed by a 256 MB write before each, outside the events), its
    fraction of the HBM roofline on the algorithmic bytes, and the end-to-end
    time through fpm_run with pinned host buffers (wall clock)."""
    N, W = WORKLOADS[name]
    seed = {"N4096_W256": 1, "N32768_W868": 2, "N65536_W1747": 3, "N65536_W2048": 4}[name]
    q, a, b = workload.case(N, W, dist, seed=1000 * seed + ["uniform", "max", "sparse"].index(dist))
    ctx = polymul.Context(N, W, q)
    L, K = ctx.L, ctx.K
    sp = stream.cuda_stream

    def todev(x):
        return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to("cuda")

    da, db = todev(a), todev(b)
    dc = torch.empty_like(da)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for _ in range(3):
            ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sp)
        for e0, e1 in evs:
            flush.zero_()
            e0.record(stream)
            ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sp)
            e1.record(stream)
    stream.synchronize()
    err = ctx.get_error(sp)
    t = sorted(e0.elapsed_time(e1) * 1e3 for e0, e1 in evs)
    dev_us = statistics.median(t)

    def pinned(x):
        tt = torch.empty(x.shape, dtype=torch.int32, pin_memory=True)
        v = tt.numpy().view(np.uint32)
        v[...] = x
        return tt, v

    (ta, pa), (tb, pb), (tc, pc) = pinned(a), pinned(b), pinned(np.zeros_like(a))
    ctx.run(pa, pb, pc)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.run(pa, pb, pc)
    e2e_us = (time.perf_counter() - t0) * 1e6 / e2e_steps
    got = dc.cpu().numpy().view(np.uint32)
    ab = algorithmic_bytes(N, L, K)
    res = {"workload": name, "dist": dist, "N": N, "W": W, "L": L, "K": K,
           "device_us": dev_us, "device_us_min": t[0], "e2e_us": e2e_us,
           "product_algorithmic_bytes": ab["product"],
           "hbm_frac": ab["product"] / (dev_us * 1e-6) / 1e9 / hbm,
           "device_equals_host_path": bool(np.array_equal(got, pc)), "error_word_clear": err == 0,
           "timing": f"median of {steps} products, L2 flushed before each; e2e {e2e_steps} fpm_run calls, "
                     "pinned buffers, wall clock"}
    del ta, tb, tc
    ctx.close()
    return res


def measure_sustained(torch, ctx, sets_d, stream, seconds=1.0):
    """Products back to back for about `seconds`, with the clocks sampled
    throughout: the same step as the timed region, long enough for the clock
    record to show the clocks under sustained load."""
    sp = stream.cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 0
    dev = torch.cuda.current_device()
    with ClockSampler(dev) as clk:
        t_end = time.perf_counter() + seconds
        e0.record(stream)
        while time.perf_counter() < t_end:
            for _ in range(200):
                da, db, dc = sets_d[n % ROTATE]
                ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sp)
                n += 1
            stream.synchronize()
        e1.record(stream)
        e1.synchronize()
    return {"products": n, "us_per_product": e0.elapsed_time(e1) * 1e3 / n, "clocks": clk.summary()}


def measure_batched(torch, polymul, workload, stream, count=64, reps=20, mix="uneven"):
    """Batched mix: `count` products, one graph of grouped launches after the
    autotuner, against `count` sequential plain calls on the same GPU (device
    buffers, and host buffers through fpm_run, the reference's fherma_run form).
    mix "uneven": N from {4096 .. 65536} and W from {128 .. 2048} (seeded);
    mix "n65536": N = 65536, W alternating 1747 and 2048."""
    sp = stream.cuda_stream
    if mix == "n65536":
        shells, rng = n65536_points(count, seed=3300)
        pts = [(N, W, workload.random_modulus(W, rng)) for N, W, _ in shells]
    else:
        pts = workload.mix_points(count, seed=4000)
    ops = workload.mix_operands(pts, seed=4001)
    ctxs = [polymul.Context(N, W, q) for N, W, q in pts]
    bt = polymul.Batch(ctxs)
    keep = []
    pa, pb, pc = [], [], []
    for (a, b), c in zip(ops, ctxs):
        (ta, va), (tb, vb) = pinned_like(torch, a), pinned_like(torch, b)
        tc, vc = pinned_like(torch, np.zeros_like(a))
        keep += [ta, tb, tc]
        pa.append(va)
        pb.append(vb)
        pc.append(vc)
    got = [x.copy() for x in bt.run(pa, pb)]
    info = bt.tune(reps=3)

    def timed(fn, n):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        fn()
        stream.synchronize()
        ev[0].record(stream)
        for _ in range(n):
            fn()
        ev[1].record(stream)
        ev[1].synchronize()
        return ev[0].elapsed_time(ev[1]) / n * 1e3   # us per call

    bufs = [bt.buffers(i) for i in range(count)]
    batch_us = timed(lambda: bt.run_device(sp), reps)

    def seq():
        for c, (da, db, dc) in zip(ctxs, bufs):
            c.run_device(da, db, dc, sp)

    seq_us = timed(seq, 5)
    # End to end: host (pinned) buffers in and out, wall clock.
    bt.run(pa, pb, pc)
    t0 = time.perf_counter()
    for _ in range(3):
        bt.run(pa, pb, pc)
    batch_e2e_us = (time.perf_counter() - t0) * 1e6 / 3
    outs = []
    for a, _ in ops:
        to, vo = pinned_like(torch, np.zeros_like(a))
        keep.append(to)
        outs.append(vo)
    for c, a, b, o in zip(ctxs, pa, pb, outs):   # each context's host path set up, untimed
        c.run(a, b, o)
    t0 = time.perf_counter()
    for c, a, b, o in zip(ctxs, pa, pb, outs):
        c.run(a, b, o)
    seq_e2e_us = (time.perf_counter() - t0) * 1e6
    exact = all(np.array_equal(g, o) for g, o in zip(got, outs)) and all(
        np.array_equal(x, o) for x, o in zip(pc, outs))
    # The one-launch-per-stage layout (3, every product in grouped launches:
    # decompose, the three transform passes over all products, CRT), timed
    # the same way, with its best grid, whether or not the tuner chose it.
    stage_layout = None
    for grid in (0, 1):
        bt.set_schedule(layout=3, order=1, prime_group=0, grid=grid, pipe_min_log_n=0)
        us3 = timed(lambda: bt.run_device(sp), reps)
        if stage_layout is None or us3 < stage_layout["batch_us"]:
            stage_layout = {"layout": 3, "grid": grid, "batch_us": us3, "launches_per_batch": bt.info.launches,
                            "speedup_vs_sequential": seq_us / us3}
    bt.set_schedule(layout=3, order=1, prime_group=0, grid=stage_layout["grid"], pipe_min_log_n=0)
    c3 = [x.copy() for x in bt.run(pa, pb)]
    stage_layout["bit_exact_vs_plain"] = bool(all(np.array_equal(x, o) for x, o in zip(c3, outs)))
    res = {
        "products": count,
        "mix": ("N = 65536, W alternating 1747 / 2048, seed 3300" if mix == "n65536" else
                "N in {4096,8192,16384,32768,65536} x W in {128,512,868,1747,2048}, seed 4000"),
        "batch_us": batch_us, "products_per_s": count / (batch_us * 1e-6),
        "sequential_us": seq_us, "sequential_products_per_s": count / (seq_us * 1e-6),
        "speedup_vs_sequential": seq_us / batch_us,
        "e2e_batch_us": batch_e2e_us, "e2e_sequential_us": seq_e2e_us,
        "e2e_speedup": seq_e2e_us / batch_e2e_us,
        "device_batch_vs_plain_e2e": seq_e2e_us / batch_us,
        "schedule": {"layout": info.layout, "order": info.order, "prime_group": info.prime_group,
                     "grid": info.grid, "pipe_min_log_n": info.pipe_min_log_n, "tuned_us": info.tuned_us},
        "launches_per_batch": info.launches, "device_bytes": info.device_bytes, "bit_exact_vs_plain": bool(exact),
        "stage_launch_layout": stage_layout,
    }
    bt.close()
    for c in ctxs:
        c.close()
    return res


def measure_serving(torch, polymul, workload, n=10000, rate=2000.0, lanes=4, max_batch=16):
    """Serving: a seeded Poisson stream of n requests at `rate`/s over 25
    resident points (the batched mix's N x W grid), pinned host buffers;
    latency from submit to the result written.  Operands come from two sets per
    point and results go to a ring of four buffers per point; every ring slot is
    checked against the product computed alone at the end.  Also the saturated
    rate (2000 requests at once) against the same requests as sequential plain
    fpm_run calls."""
    rng = np.random.Generator(np.random.PCG64(5000))
    cat = [(N, W) for N in workload.MIX_N for W in workload.MIX_W]
    ctxs, qs = [], []
    for N, W in cat:
        q = workload.random_modulus(W, rng)
        ctxs.append(polymul.Context(N, W, q))
        qs.append(q)
    keep, ops, outs, expect = [], [], [], []
    SETS, RING = 2, 4
    for p, (N, W) in enumerate(cat):
        ps, es, ring = [], [], []
        for s in range(SETS):
            a, b = workload.operands(qs[p], N, "uniform", rng)
            (ta, va), (tb, vb) = pinned_like(torch, a), pinned_like(torch, b)
            keep += [ta, tb]
            ps.append((va, vb))
            es.append(ctxs[p].run(a, b))
        for _ in range(RING):
            tc, vc = pinned_like(torch, np.zeros((N, ctxs[p].L), np.uint32))
            keep.append(tc)
            ring.append(vc)
        ops.append(ps)
        expect.append(es)
        outs.append(ring)
    pts = rng.integers(0, len(cat), size=n)
    arrivals = workload.poisson_arrivals(n, rate, seed=5001)
    a_l, b_l, c_l, last = [], [], [], {}
    cnt = np.zeros(len(cat), int)
    for i, p in enumerate(pts):
        s = i % SETS
        slot = cnt[p] % RING
        cnt[p] += 1
        a_l.append(ops[p][s][0])
        b_l.append(ops[p][s][1])
        c_l.append(outs[p][slot])
        last[(p, slot)] = s
    srv = polymul.Server(ctxs, budget_bytes=16 << 30, lanes=lanes, max_batch=max_batch)
    srv.replay(pts[:50], np.zeros(50), a_l[:50], b_l[:50], c_l[:50])    # warm-up
    b0 = srv.stats.batches
    t0 = time.perf_counter()
    lat = srv.replay(pts, arrivals, a_l, b_l, c_l)
    wall = time.perf_counter() - t0
    st = srv.stats
    verified = sum(np.array_equal(outs[p][slot], expect[p][s]) for (p, slot), s in last.items())
    m = min(2000, n)
    t0 = time.perf_counter()
    srv.replay(pts[:m], np.zeros(m), a_l[:m], b_l[:m], c_l[:m])
    sat = m / (time.perf_counter() - t0)
    k = min(500, n)
    t0 = time.perf_counter()
    for i in range(k):
        ctxs[pts[i]].run(a_l[i], b_l[i], c_l[i])
    plain = k / (time.perf_counter() - t0)
    res = {
        "requests": n, "rate_per_s": rate, "lanes": lanes, "max_batch": max_batch, "points": len(cat),
        "products_per_s": n / wall, "p50_us": float(np.percentile(lat, 50)), "p99_us": float(np.percentile(lat, 99)),
        "mean_us": float(lat.mean()), "max_us": float(lat.max()),
        "micro_batches": int(st.batches - b0), "max_lanes_busy": int(st.max_lanes_busy),
        "peak_device_bytes": int(st.peak_bytes), "budget_bytes": int(st.budget_bytes),
        "saturated_products_per_s": sat, "plain_sequential_products_per_s": plain,
        "saturated_vs_plain": sat / plain,
        "verified": f"{verified}/{len(last)} result buffers bit-exact against the product alone",
    }
    srv.close()
    for c in ctxs:
        c.close()
    return res


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
    launches_per_product = 3 if ctx.info.logN <= 10 or ctx.info.logR == 0 else 5

    def step(i):
        da, db, dc = sets_d[i % ROTATE]
        ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sp)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
    stream.synchronize()

    # Per-stage timing (dominant kernel for the roofline), outside the main region.
    AB = torch.empty((2 * K, N), dtype=torch.int32, device="cuda")   # A then B, as the paired launch writes
    A, B = AB[:K], AB[K:]
    # a then b of each operand set, contiguous (the paired decompose's input);
    # the four pairs rotate, so the limbs come from HBM as in a product.
    pairs = [torch.cat((x, y)).contiguous() for x, y, _ in sets_d]
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
    rot = [0]

    def dec_pair():
        ctx.stage_decompose(pairs[rot[0] % ROTATE].data_ptr(), AB.data_ptr(), 2, sp)
        rot[0] += 1

    stages["decompose"] = time_stage(dec_pair)
    ctx.stage_decompose(pairs[0].data_ptr(), AB.data_ptr(), 2, sp)
    stages["transform"] = time_stage(lambda: ctx.stage_transform(A.data_ptr(), B.data_ptr(), 0, sp))
    stages["crt"] = time_stage(lambda: ctx.stage_crt(A.data_ptr(), dc.data_ptr(), sp))
    # One kernel at a time (the transform's passes alone: modes 2, 3, 4).
    # Decompose and CRT: the persistent pipelines; the decompose stage is the
    # product's own paired launch (both operands, limbs rotating through HBM).
    kernels = {"k_decompose_pipe": stages["decompose"], "k_crt_pipe": stages["crt"]}
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
    clocks = clk.summary()

    def reduce_max(v):
        t = torch.tensor([v], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return t.item()

    ms, us_per_product = job_time(start.elapsed_time(end), args.steps, world, reduce_max)

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
        """Median and mean of n calls, each timed by wall clock around fpm_run
        (a host-side stall in one call moves the mean, not the median)."""
        ctx.run(a_, b_, c_)
        ts = []
        for _ in range(n):
            t0 = time.perf_counter()
            ctx.run(a_, b_, c_)
            ts.append((time.perf_counter() - t0) * 1e6)
        return statistics.median(ts), statistics.fmean(ts)

    io_chunks = ctx.tune_host_path()   # as fherma_init does, outside the timed calls
    e2e_us, e2e_mean_us = e2e(a_p, b_p, c_p, args.e2e_steps)
    c_h = np.empty((N, L), np.uint32)
    e2e_pageable_us, _ = e2e(a_h, b_h, c_h, args.e2e_steps)

    # The link itself: pinned copies of one product's operands in and result
    # out, timed alone with CUDA events (best of 5).  Their sum plus the device
    # time is what a synchronous call cannot beat.
    def copy_us(dst, src, reps=5):
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                dst.copy_(src, non_blocking=True)
                e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) * 1e3
            best = t if best is None else min(best, t)
        return best

    dev_in = torch.empty((2, N, L), dtype=torch.int32, device="cuda")
    host_in = torch.empty((2, N, L), dtype=torch.int32, pin_memory=True)
    dev_out = torch.empty((N, L), dtype=torch.int32, device="cuda")
    h2d_us = copy_us(dev_in, host_in)
    d2h_us = copy_us(c_pt, dev_out)
    del dev_in, host_in, dev_out
    link = {"h2d_gbs": 2 * N * L * 4 / (h2d_us * 1e3), "d2h_gbs": N * L * 4 / (d2h_us * 1e3),
            "h2d_us": h2d_us, "d2h_us": d2h_us,
            "floor_us": h2d_us + d2h_us + ms * 1e3 / args.steps,
            "note": "pinned copies of one product's operands and result timed alone (CUDA events, best of 5); "
                    "floor = both copies + the device time, the least a call that returns its result can take"}

    hbm, peak_kind = peaks()
    ab = algorithmic_bytes(N, L, K)
    kernel_bytes = {"k_decompose_pipe": 2 * ab["decompose"], "k_ntt_col_fwd": ab["ntt_col_fwd"],
                    "k_ntt_row": ab["ntt_row"], "k_ntt_col_inv": ab["ntt_col_inv"], "k_crt_pipe": ab["crt"]}
    # launches per product: the dominant kernel's time share in one product
    per_product = {"k_decompose_pipe": 1, "k_ntt_col_fwd": 1, "k_ntt_row": 1, "k_ntt_col_inv": 1, "k_crt_pipe": 1}
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

    sustained = (measure_sustained(torch, ctx, sets_d, stream, seconds=args.sustained_s)
                 if rank == 0 and args.sustained_s > 0 else None)

    # Context set-up (fpm_init): a new modulus of the width in use (the prime
    # basis's tables are shared, the CRT tables are built on the device), a
    # width not yet in use (the whole basis built and uploaded), and the
    # host-only plan of the same point for comparison.
    init = None
    if rank == 0:
        rng_i = np.random.Generator(np.random.PCG64(6000))

        def init_us(width):
            qq = workload.random_modulus(width, rng_i)
            t0 = time.perf_counter()
            c_ = polymul.Context(N, width, qq)
            t1 = time.perf_counter()
            c_.close()
            return (t1 - t0) * 1e6

        warm = sorted(init_us(W) for _ in range(5))
        cold = init_us(W - 1)
        t0 = time.perf_counter()
        polymul.plan_info(N, W, workload.random_modulus(W, rng_i))
        host_plan = (time.perf_counter() - t0) * 1e6
        init = {"new_modulus_us": statistics.median(warm), "new_width_us": cold, "host_plan_us": host_plan,
                "note": f"fpm_init at N={N}: a new W={W} modulus while a context of that width is open (median of "
                        f"5), a W={W - 1} modulus (a basis not yet built), and make_plan alone on the host"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            if oracle.ref_available():
                reps, reps1 = 5, 3
                cores = os.cpu_count() or 1
                _, secs = oracle.ref_polymul(N, W, q, a_h, b_h, reps=reps, threads=cores)
                _, secs1 = oracle.ref_polymul(N, W, q, a_h, b_h, reps=reps1, threads=1)
                cpu = {"value": 1e6 * statistics.median(secs), "unit": "us/product", "cores": cores,
                       "kind": "reference",
                       "one_thread_us": 1e6 * statistics.median(secs1),
                       "sample": f"median of {reps} products at N={N} W={W} with {cores} OpenMP threads, and of "
                                 f"{reps1} with 1 thread (one_thread_us): the reference's solve_cpu.cpp, "
                                 "steady_clock around fherma_run"}
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "unit": "us/product", "cores": None, "kind": "reference",
                   "sample": f"failed: {e}"}

    points = None
    if rank == 0 and world == 1 and not args.no_configs:
        points = [measure_point(torch, polymul, workload, name, dist, stream, hbm) for name, dist in CONFIG_POINTS]

    batched = batched_big = serving = None
    if rank == 0 and world == 1:
        if not args.no_batched:
            batched = measure_batched(torch, polymul, workload, stream)
            batched_big = measure_batched(torch, polymul, workload, stream, count=16, reps=10, mix="n65536")
        if not args.no_serving:
            serving = measure_serving(torch, polymul, workload, n=args.serve_requests, rate=args.serve_rate)

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
                    "d2h_bytes_per_step": N * L * 4, "host_buffers": "pinned (fpm_run, wall clock)",
                    "statistic": "median of the calls (mean_us beside it)", "mean_us": e2e_mean_us,
                    "io_chunks": io_chunks, "calls": args.e2e_steps},
            "e2e_pageable": {"value": e2e_pageable_us, "unit": "us/product",
                             "host_buffers": "pageable numpy (fpm_run stages through pinned memory)"},
            "pcie": link,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes": kernel_bytes[dom],
                         "note": "algorithmic bytes per launch (six-pass schedule, twiddles cache-resident) / "
                                 "CUDA-event launch time, against the measured copy bandwidth; traffic = ncu "
                                 "dram read+write per launch from profiles/ncu_traffic.json (includes the row "
                                 "pass's own twiddle-table reads)"},
            "stages_us": stages,
            "kernels_us": kernels,
            "product_algorithmic_bytes": ab["product"],
            "row_table_bytes": ab["row_tables"],
            "product_hbm_frac": ab["product"] / (us_per_product * world * 1e-6) / 1e9 / hbm,
            "gpu_launches": args.steps * launches_per_product,
            "clocks": clocks,
            "sustained": sustained,
            "init": init,
            "configs": points,
            "cpu_baseline": cpu,
            "batched": batched,
            "batched_n65536": batched_big,
            "serving": serving,
        }
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
