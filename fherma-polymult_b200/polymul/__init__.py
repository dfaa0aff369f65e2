"""Python mirror of the reference's plugin interface, over the C ABI of
lib/libfpm.so (include/fherma_polymult.h).

The reference's solution is three C++ functions bound by the FHERMA harness
(fherma.h:46-48):

    void*           fherma_init(const fherma::Point&)
    fherma::Outputs fherma_run(void* state, const fherma::Inputs&)
    void            fherma_free(void* state)

This module offers the same three names with the same argument meaning and the
same error behaviour (an out-of-range point or a mis-sized operand raises, as
the reference throws std::runtime_error), taking numpy arrays in place of
fherma::Tensor.  ``Context`` exposes the rest of the C ABI: products on device
buffers enqueued on a CUDA stream, the stage entry points, and the host-only
plan query.

There is no CPU fallback: loading fails if lib/libfpm.so is missing, and
fherma_init fails without a CUDA device.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libfpm.so")

FPM_OK, FPM_EINVAL, FPM_ECUDA, FPM_ENOMEM, FPM_EINTERNAL, FPM_ETIMEOUT = 0, 1, 2, 3, 4, 5
STALL_DECOMPOSE, STALL_CRT = 1, 2
MODE_PRODUCT, MODE_FORWARD = 0, 1

_u32p = ctypes.POINTER(ctypes.c_uint32)


class FpmInfo(ctypes.Structure):
    _fields_ = [("N", ctypes.c_uint32), ("W", ctypes.c_uint32), ("L", ctypes.c_uint32), ("K", ctypes.c_uint32),
                ("logN", ctypes.c_uint32), ("logR", ctypes.c_uint32), ("logS", ctypes.c_uint32),
                ("device", ctypes.c_int32), ("device_bytes", ctypes.c_uint64), ("prime_bits", ctypes.c_uint32)]


class FpmBatchInfo(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint32), ("layout", ctypes.c_int32), ("order", ctypes.c_int32),
                ("prime_group", ctypes.c_int32), ("grid", ctypes.c_int32), ("pipe_min_log_n", ctypes.c_int32),
                ("launches", ctypes.c_int32),
                ("device_bytes", ctypes.c_uint64), ("tuned_us", ctypes.c_double)]


class FpmServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("lanes", ctypes.c_uint32), ("max_lanes_busy", ctypes.c_uint32), ("budget_bytes", ctypes.c_uint64),
                ("peak_bytes", ctypes.c_uint64)]


class FpmError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads lib/libfpm.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `make -C fherma-polymult_b200` "
                           "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sig = {
        "fpm_init": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p, ctypes.POINTER(vp)], ctypes.c_int),
        "fpm_init_ex": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p, ctypes.c_int, ctypes.POINTER(vp)],
                        ctypes.c_int),
        "fpm_plan_info_ex": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p, ctypes.c_int,
                              ctypes.POINTER(FpmInfo), _u32p], ctypes.c_int),
        "fpm_run": ([vp, vp, vp, vp], ctypes.c_int),
        "fpm_run_device": ([vp, vp, vp, vp, vp], ctypes.c_int),
        "fpm_run_device_noalloc": ([vp, vp, vp, vp, vp], ctypes.c_int),
        "fpm_get_error": ([vp, vp], ctypes.c_int),
        "fpm_noalloc_get_error": ([vp], ctypes.c_int),
        "fpm_set_wait_limit": ([vp, ctypes.c_uint64], ctypes.c_int),
        "fpm_debug_inject_stall": ([vp, ctypes.c_uint32], ctypes.c_int),
        "fpm_free": ([vp], None),
        "fpm_last_error": ([], ctypes.c_char_p),
        "fpm_get_info": ([vp, ctypes.POINTER(FpmInfo)], ctypes.c_int),
        "fpm_plan_info": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p, ctypes.POINTER(FpmInfo), _u32p],
                          ctypes.c_int),
        "fpm_get_primes": ([vp, _u32p], ctypes.c_int),
        "fpm_get_crt_tables": ([vp, _u32p, _u32p], ctypes.c_int),
        "fpm_tune_host_path": ([vp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "fpm_server_add_point": ([vp, vp, ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
        "fpm_stage_decompose": ([vp, vp, vp, ctypes.c_int, vp], ctypes.c_int),
        "fpm_stage_transform": ([vp, vp, vp, ctypes.c_int, vp], ctypes.c_int),
        "fpm_stage_crt": ([vp, vp, vp, vp], ctypes.c_int),
        "fpm_batch_create": ([ctypes.POINTER(vp), ctypes.c_uint32, ctypes.POINTER(vp)], ctypes.c_int),
        "fpm_batch_buffers": ([vp, ctypes.c_uint32, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)],
                              ctypes.c_int),
        "fpm_batch_run_device": ([vp, vp], ctypes.c_int),
        "fpm_batch_run": ([vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)], ctypes.c_int),
        "fpm_batch_tune": ([vp, ctypes.c_int, ctypes.POINTER(FpmBatchInfo)], ctypes.c_int),
        "fpm_batch_set_schedule": ([vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int],
                                   ctypes.c_int),
        "fpm_batch_get_info": ([vp, ctypes.POINTER(FpmBatchInfo)], ctypes.c_int),
        "fpm_batch_free": ([vp], None),
        "fpm_server_create": ([ctypes.POINTER(vp), ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                               ctypes.POINTER(vp)], ctypes.c_int),
        "fpm_server_footprint": ([vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "fpm_server_submit": ([vp, ctypes.c_uint32, vp, vp, vp, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "fpm_server_wait": ([vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "fpm_server_replay": ([vp, ctypes.c_uint32, _u32p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(vp),
                               ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_double)],
                              ctypes.c_int),
        "fpm_server_get_stats": ([vp, ctypes.POINTER(FpmServerStats)], ctypes.c_int),
        "fpm_server_free": ([vp], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _check(rc: int):
    if rc != FPM_OK:
        raise FpmError(rc, load().fpm_last_error().decode())


def _limbs(x, rows: int, L: int, name: str) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.uint32)
    if x.size != rows * L:
        # reference solve.cu:877-879: "operand size does not match the point"
        raise FpmError(FPM_EINVAL, f"{name}: operand size does not match the point")
    return x.reshape(rows, L)


def plan_info(N: int, W: int, q, prime_bits: int = 0) -> tuple[FpmInfo, np.ndarray]:
    """Host-only: the plan fherma_init would build (raises on a bad point)."""
    lib = load()
    q = np.ascontiguousarray(q, dtype=np.uint32)
    info = FpmInfo()
    primes = np.zeros(160, np.uint32)
    _check(lib.fpm_plan_info_ex(N, W, q.shape[0], q.ctypes.data_as(_u32p), prime_bits, ctypes.byref(info),
                                primes.ctypes.data_as(_u32p)))
    return info, primes[:info.K].copy()


class Context:
    """One point's resident state on the current CUDA device (fpm_ctx)."""

    def __init__(self, N: int, W: int, q, prime_bits: int = 0):
        """prime_bits: 30 (primes below 2^30, the default) or 31 (the reference's
        prime set); 0 takes the default."""
        lib = load()
        q = np.ascontiguousarray(q, dtype=np.uint32)
        h = ctypes.c_void_p()
        _check(lib.fpm_init_ex(N, W, q.shape[0], q.ctypes.data_as(_u32p), prime_bits, ctypes.byref(h)))
        self._h = h
        self._lib = lib
        info = FpmInfo()
        _check(lib.fpm_get_info(h, ctypes.byref(info)))
        self.info = info
        self.N, self.W, self.L, self.K = info.N, W, info.L, info.K
        self.prime_bits = info.prime_bits

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fpm_free(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def primes(self) -> np.ndarray:
        out = np.zeros(self.K, np.uint32)
        _check(self._lib.fpm_get_primes(self._h, out.ctypes.data_as(_u32p)))
        return out

    def tune_host_path(self) -> int:
        """Measures the host path's copy chunking on this point (as
        fherma_init does); returns the chunk count kept."""
        n = ctypes.c_int()
        _check(self._lib.fpm_tune_host_path(self._h, ctypes.byref(n)))
        return n.value

    def crt_tables(self) -> tuple[np.ndarray, np.ndarray]:
        """The CRT constants built on the device: M (K x L), negvP ((K + 1) x L)."""
        M = np.zeros((self.K, self.L), np.uint32)
        negvP = np.zeros((self.K + 1, self.L), np.uint32)
        _check(self._lib.fpm_get_crt_tables(self._h, M.ctypes.data_as(_u32p), negvP.ctypes.data_as(_u32p)))
        return M, negvP

    def run(self, a, b, out=None) -> np.ndarray:
        """c = a b on host arrays (N x L u32)."""
        a = _limbs(a, self.N, self.L, "a")
        b = _limbs(b, self.N, self.L, "b")
        c = np.empty((self.N, self.L), np.uint32) if out is None else out
        _check(self._lib.fpm_run(self._h, a.ctypes.data, b.ctypes.data, c.ctypes.data))
        return c

    def run_device(self, d_a: int, d_b: int, d_c: int, stream: int = 0):
        """c = a b on device pointers (ints), enqueued on a cudaStream_t (int)."""
        _check(self._lib.fpm_run_device(self._h, d_a, d_b, d_c, stream or None))

    def get_error(self, stream: int = 0) -> int:
        """Waits for `stream`, then reads and clears the context's error word:
        FPM_ETIMEOUT if a kernel pipeline wait ran out since the last check."""
        return self._lib.fpm_get_error(self._h, stream or None)

    def set_wait_limit(self, ns: int):
        """Limit of every pipeline wait of later products, in nanoseconds."""
        _check(self._lib.fpm_set_wait_limit(self._h, int(ns)))

    def inject_stall(self, mask: int):
        """Test hook: STALL_DECOMPOSE / STALL_CRT make that pipeline's wait run
        out in later products (0 restores normal operation)."""
        _check(self._lib.fpm_debug_inject_stall(self._h, mask))

    def stage_decompose(self, d_limbs: int, d_res: int, operand: int, stream: int = 0):
        _check(self._lib.fpm_stage_decompose(self._h, d_limbs, d_res, operand, stream or None))

    def stage_transform(self, d_A: int, d_B: int, mode: int, stream: int = 0):
        _check(self._lib.fpm_stage_transform(self._h, d_A, d_B, mode, stream or None))

    def stage_crt(self, d_y: int, d_c: int, stream: int = 0):
        _check(self._lib.fpm_stage_crt(self._h, d_y, d_c, stream or None))


class Batch:
    """Many products of uneven (N, q) in one CUDA graph of grouped launches
    (fpm_batch).  ``contexts`` are Context objects (one per product, repeats
    allowed); they must stay open while the batch lives."""

    def __init__(self, contexts):
        lib = load()
        self._lib = lib
        self.contexts = list(contexts)
        arr = (ctypes.c_void_p * len(self.contexts))(*[c.handle.value for c in self.contexts])
        h = ctypes.c_void_p()
        _check(lib.fpm_batch_create(arr, len(self.contexts), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fpm_batch_free(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.contexts)

    @property
    def info(self) -> FpmBatchInfo:
        out = FpmBatchInfo()
        _check(self._lib.fpm_batch_get_info(self._h, ctypes.byref(out)))
        return out

    def buffers(self, i: int) -> tuple[int, int, int]:
        """Device pointers (a, b, c) of product i."""
        a, b, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _check(self._lib.fpm_batch_buffers(self._h, i, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def run_device(self, stream: int = 0):
        """Every product on the batch's device buffers: one graph launch."""
        _check(self._lib.fpm_batch_run_device(self._h, stream or None))

    def run(self, a_list, b_list, out=None) -> list:
        """c_i = a_i b_i for host arrays (N_i x L_i u32 each)."""
        n = len(self.contexts)
        if len(a_list) != n or len(b_list) != n:
            raise FpmError(FPM_EINVAL, f"expected {n} operand pairs")
        a = [_limbs(x, c.N, c.L, "a") for x, c in zip(a_list, self.contexts)]
        b = [_limbs(x, c.N, c.L, "b") for x, c in zip(b_list, self.contexts)]
        cs = out if out is not None else [np.empty((c.N, c.L), np.uint32) for c in self.contexts]
        pa = (ctypes.c_void_p * n)(*[x.ctypes.data for x in a])
        pb = (ctypes.c_void_p * n)(*[x.ctypes.data for x in b])
        pc = (ctypes.c_void_p * n)(*[x.ctypes.data for x in cs])
        _check(self._lib.fpm_batch_run(self._h, pa, pb, pc))
        return cs

    def tune(self, reps: int = 3) -> FpmBatchInfo:
        out = FpmBatchInfo()
        _check(self._lib.fpm_batch_tune(self._h, reps, ctypes.byref(out)))
        return out

    def set_schedule(self, layout: int = 1, order: int = 1, prime_group: int = 0, grid: int = 0,
                     pipe_min_log_n: int = 0):
        _check(self._lib.fpm_batch_set_schedule(self._h, layout, order, prime_group, grid, pipe_min_log_n))


class Server:
    """Serving loop over resident points (fpm_server): requests are admitted by
    their device footprint within ``budget_bytes`` and run as micro-batches on
    ``lanes`` concurrent streams.  Host buffers passed to submit / replay must
    stay alive until the request is done; pinned buffers overlap best."""

    def __init__(self, contexts, budget_bytes: int = 8 << 30, lanes: int = 4, max_batch: int = 16):
        lib = load()
        self._lib = lib
        self.contexts = list(contexts)
        arr = (ctypes.c_void_p * len(self.contexts))(*[c.handle.value for c in self.contexts])
        h = ctypes.c_void_p()
        _check(lib.fpm_server_create(arr, len(self.contexts), budget_bytes, lanes, max_batch, ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fpm_server_free(self._h)
            self._h = None
        self._keep = {}

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_point(self, ctx) -> int:
        """Adds a context while the server runs; returns its point index."""
        idx = ctypes.c_uint32()
        _check(self._lib.fpm_server_add_point(self._h, ctx.handle, ctypes.byref(idx)))
        self.contexts.append(ctx)
        return idx.value

    def footprint(self, point: int) -> int:
        out = ctypes.c_uint64()
        _check(self._lib.fpm_server_footprint(self._h, point, ctypes.byref(out)))
        return out.value

    @property
    def stats(self) -> FpmServerStats:
        out = FpmServerStats()
        _check(self._lib.fpm_server_get_stats(self._h, ctypes.byref(out)))
        return out

    def _check_buffers(self, point, a, b, c):
        ctx = self.contexts[point]
        for name, x in (("a", a), ("b", b), ("c", c)):
            if x.dtype != np.uint32 or x.size != ctx.N * ctx.L or not x.flags.c_contiguous:
                raise FpmError(FPM_EINVAL, f"{name}: operand size does not match the point")

    def submit(self, point: int, a: np.ndarray, b: np.ndarray, c: np.ndarray) -> int:
        """Queues c = a b on `point` (arrays N x L u32, kept alive until wait)."""
        self._check_buffers(point, a, b, c)
        t = ctypes.c_uint64()
        _check(self._lib.fpm_server_submit(self._h, point, a.ctypes.data, b.ctypes.data, c.ctypes.data,
                                           ctypes.byref(t)))
        self._keep[t.value] = (a, b, c)
        return t.value

    def wait(self, ticket: int) -> float:
        """Latency of the request in microseconds, once c is written."""
        us = ctypes.c_double()
        try:
            _check(self._lib.fpm_server_wait(self._h, ticket, ctypes.byref(us)))
        finally:
            self._keep.pop(ticket, None)
        return us.value

    def replay(self, points, arrival_us, a_list, b_list, c_list) -> np.ndarray:
        """Submits request i at arrival_us[i]; returns the latencies (us)."""
        n = len(points)
        for i in range(n):
            self._check_buffers(int(points[i]), a_list[i], b_list[i], c_list[i])
        pts = np.ascontiguousarray(points, dtype=np.uint32)
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        lat = np.zeros(n, np.float64)
        pa = (ctypes.c_void_p * n)(*[x.ctypes.data for x in a_list])
        pb = (ctypes.c_void_p * n)(*[x.ctypes.data for x in b_list])
        pc = (ctypes.c_void_p * n)(*[x.ctypes.data for x in c_list])
        _check(self._lib.fpm_server_replay(self._h, n, pts.ctypes.data_as(_u32p),
                                           arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), pa, pb, pc,
                                           lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return lat


# ---------------------------------------------------------------------------
# The reference's interface (fherma.h:16-48), numpy in place of fherma::Tensor.

@dataclass
class Point:
    N: int
    W: int
    L: int
    q: np.ndarray            # L u32


@dataclass
class Inputs:
    a: np.ndarray            # N x L u32
    b: np.ndarray


@dataclass
class Outputs:
    c: np.ndarray = field(default=None)   # N x L u32


def fherma_init(p: Point) -> Context:
    q = np.ascontiguousarray(p.q, dtype=np.uint32).reshape(-1)
    if q.shape[0] != p.L:
        raise FpmError(FPM_EINVAL, f"q has {q.shape[0]} limbs, expected L = {p.L}")
    return Context(p.N, p.W, q)


def fherma_run(state: Context, inputs: Inputs) -> Outputs:
    return Outputs(c=state.run(inputs.a, inputs.b))


def fherma_free(state: Context | None):
    if state is not None:
        state.close()
