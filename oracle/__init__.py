"""Test oracles for the exact negacyclic product c = a*b mod (X^N + 1, q).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs import this package, and only as the checker or
the timed CPU baseline.  The shipped library never imports it.

Four independent checkers:

* ``OraclePlan``  - ctypes binding of oracle/rns_oracle.c, our plain-C
  restatement of the reference's RNS + NTT + CRT algorithm, stage by stage.
* ``ref_polymul`` / ``ref_plan`` - the reference's own CPU implementation
  (solve_cpu.cpp) built from the reference tree into oracle/_ref/ by
  oracle/Makefile, behind oracle/ref_shim.cpp.
* ``kronecker``   - the product by Kronecker substitution with GMP (through
  ctypes on the system libgmp), the method of the reference's make_big.py:21-29;
  it shares no code with the RNS path.
* ``schoolbook``  - the O(N^2) Python big-integer product (reference
  oracle.py:81-91), full for small N or on sampled coefficients.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "lib", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_BIN = os.path.join(HERE, "_ref", "solution_cpu")

_u32p = ctypes.POINTER(ctypes.c_uint32)


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u32p)


# ---------------------------------------------------------------------------
# our C restatement

_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        lib = ctypes.CDLL(ORACLE_LIB)
        lib.ora_plan_make.argtypes = [ctypes.c_uint32, _u32p, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_size_t]
        lib.ora_plan_make.restype = ctypes.c_int
        lib.ora_plan_free.argtypes = [ctypes.c_void_p]
        for name in ("ora_plan_K", "ora_plan_L"):
            getattr(lib, name).argtypes = [ctypes.c_void_p]
            getattr(lib, name).restype = ctypes.c_int
        lib.ora_plan_N.argtypes = [ctypes.c_void_p]
        lib.ora_plan_N.restype = ctypes.c_uint32
        for name in ("ora_plan_primes", "ora_plan_roots"):
            getattr(lib, name).argtypes = [ctypes.c_void_p, _u32p]
        lib.ora_plan_crt_tables.argtypes = [ctypes.c_void_p, _u32p, _u32p]
        lib.ora_decompose.argtypes = [ctypes.c_void_p, _u32p, _u32p]
        lib.ora_ntt_forward.argtypes = [ctypes.c_void_p, _u32p]
        lib.ora_ntt_inverse.argtypes = [ctypes.c_void_p, _u32p]
        lib.ora_pointwise.argtypes = [ctypes.c_void_p, _u32p, _u32p]
        lib.ora_crt.argtypes = [ctypes.c_void_p, _u32p, _u32p]
        lib.ora_polymul.argtypes = [ctypes.c_void_p, _u32p, _u32p, _u32p, _u32p]
        lib.ora_polymul.restype = ctypes.c_int
        _olib = lib
    return _olib


class OraclePlan:
    """The oracle's plan for (N, q); stage functions mirror rns_oracle.h."""

    def __init__(self, N: int, q: np.ndarray, pmax_log2: int = 31):
        lib = _oracle_lib()
        q = np.ascontiguousarray(q, dtype=np.uint32)
        self.N, self.L = int(N), int(q.shape[0])
        err = ctypes.create_string_buffer(512)
        h = ctypes.c_void_p()
        if lib.ora_plan_make(self.N, _ptr(q), self.L, pmax_log2, ctypes.byref(h), err, 512):
            raise ValueError(err.value.decode())
        self._h = h
        self._lib = lib
        self.K = lib.ora_plan_K(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.ora_plan_free(h)
            self._h = None

    @property
    def primes(self) -> np.ndarray:
        out = np.zeros(self.K, np.uint32)
        self._lib.ora_plan_primes(self._h, _ptr(out))
        return out

    @property
    def roots(self) -> np.ndarray:
        out = np.zeros(self.K, np.uint32)
        self._lib.ora_plan_roots(self._h, _ptr(out))
        return out

    def crt_tables(self):
        M = np.zeros((self.K, self.L), np.uint32)
        negvP = np.zeros((self.K + 1, self.L), np.uint32)
        self._lib.ora_plan_crt_tables(self._h, _ptr(M), _ptr(negvP))
        return M, negvP

    def _limbs(self, x):
        x = np.ascontiguousarray(x, dtype=np.uint32)
        assert x.shape == (self.N, self.L), x.shape
        return x

    def decompose(self, limbs) -> np.ndarray:
        out = np.zeros((self.K, self.N), np.uint32)
        self._lib.ora_decompose(self._h, _ptr(self._limbs(limbs)), _ptr(out))
        return out

    def ntt_forward(self, res) -> np.ndarray:
        out = np.array(res, dtype=np.uint32, order="C", copy=True)
        self._lib.ora_ntt_forward(self._h, _ptr(out))
        return out

    def ntt_inverse(self, res) -> np.ndarray:
        out = np.array(res, dtype=np.uint32, order="C", copy=True)
        self._lib.ora_ntt_inverse(self._h, _ptr(out))
        return out

    def pointwise(self, A, B) -> np.ndarray:
        out = np.array(A, dtype=np.uint32, order="C", copy=True)
        B = np.ascontiguousarray(B, dtype=np.uint32)
        self._lib.ora_pointwise(self._h, _ptr(out), _ptr(B))
        return out

    def crt(self, y) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.uint32)
        out = np.zeros((self.N, self.L), np.uint32)
        self._lib.ora_crt(self._h, _ptr(y), _ptr(out))
        return out

    def polymul(self, a, b, want_y: bool = False):
        c = np.zeros((self.N, self.L), np.uint32)
        y = np.zeros((self.K, self.N), np.uint32) if want_y else None
        rc = self._lib.ora_polymul(self._h, _ptr(self._limbs(a)), _ptr(self._limbs(b)), _ptr(c),
                                   _ptr(y) if want_y else None)
        if rc:
            raise MemoryError("oracle polymul failed")
        return (c, y) if want_y else c


# ---------------------------------------------------------------------------
# the reference's own CPU build

_rlib = None


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _ref_lib():
    global _rlib
    if _rlib is None:
        if not os.path.exists(REF_LIB):
            raise RuntimeError(f"{REF_LIB} missing: run `make -C oracle` where the reference tree exists")
        lib = ctypes.CDLL(REF_LIB)
        lib.ref_polymul.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p, _u32p,
                                    _u32p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        lib.ref_polymul.restype = ctypes.c_int
        lib.ref_plan.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _u32p, ctypes.POINTER(ctypes.c_int), _u32p,
                                 _u32p, _u32p, _u32p]
        lib.ref_plan.restype = ctypes.c_int
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_set_threads.argtypes = [ctypes.c_int]
        lib.ref_set_threads.restype = ctypes.c_int
        _rlib = lib
    return _rlib


def ref_polymul(N: int, W: int, q, a, b, reps: int = 1, threads: int = 0):
    """The reference's fherma_run on (a, b): returns (c, seconds per call).
    threads: OpenMP threads of the reference's loops (0: all processors)."""
    lib = _ref_lib()
    lib.ref_set_threads(threads)
    q = np.ascontiguousarray(q, dtype=np.uint32)
    L = q.shape[0]
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    c = np.zeros((N, L), np.uint32)
    secs = (ctypes.c_double * reps)()
    if lib.ref_polymul(N, W, L, _ptr(q), _ptr(a), _ptr(b), _ptr(c), reps, secs):
        raise RuntimeError(lib.ref_last_error().decode())
    return c, list(secs)


def ref_plan(N: int, q):
    """The reference's make_plan tables: dict(K, primes, roots, M, negvP)."""
    lib = _ref_lib()
    q = np.ascontiguousarray(q, dtype=np.uint32)
    L = q.shape[0]
    K = ctypes.c_int()
    primes = np.zeros(160, np.uint32)
    roots = np.zeros(160, np.uint32)
    M = np.zeros(160 * L, np.uint32)
    negvP = np.zeros(161 * L, np.uint32)
    if lib.ref_plan(N, L, _ptr(q), ctypes.byref(K), _ptr(primes), _ptr(roots), _ptr(M), _ptr(negvP)):
        raise ValueError(lib.ref_last_error().decode())
    k = K.value
    return dict(K=k, primes=primes[:k].copy(), roots=roots[:k].copy(), M=M[:k * L].reshape(k, L).copy(),
                negvP=negvP[:(k + 1) * L].reshape(k + 1, L).copy())


# ---------------------------------------------------------------------------
# independent big-integer products

class _mpz(ctypes.Structure):
    _fields_ = [("_mp_alloc", ctypes.c_int), ("_mp_size", ctypes.c_int), ("_mp_d", ctypes.c_void_p)]


_gmp = None


def _gmp_lib():
    global _gmp
    if _gmp is None:
        path = ctypes.util.find_library("gmp") or "libgmp.so.10"
        lib = ctypes.CDLL(path)
        mp = ctypes.POINTER(_mpz)
        lib.__gmpz_init.argtypes = [mp]
        lib.__gmpz_clear.argtypes = [mp]
        lib.__gmpz_mul.argtypes = [mp, mp, mp]
        lib.__gmpz_import.argtypes = [mp, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t, ctypes.c_int,
                                      ctypes.c_size_t, ctypes.c_void_p]
        lib.__gmpz_export.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
                                      ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t, mp]
        lib.__gmpz_export.restype = ctypes.c_void_p
        lib.__gmpz_sizeinbase.argtypes = [mp, ctypes.c_int]
        lib.__gmpz_sizeinbase.restype = ctypes.c_size_t
        _gmp = lib
    return _gmp


def kronecker(q, a, b) -> np.ndarray:
    """c = a*b mod (X^N + 1, q) by Kronecker substitution with GMP.

    Each polynomial is packed into one integer with a slot wide enough for any
    coefficient of the plain product, multiplied once, unpacked, and the top
    half folded back negated (reference make_big.py:21-29).
    """
    lib = _gmp_lib()
    q = np.ascontiguousarray(q, dtype=np.uint32)
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    N, L = a.shape
    qi = int.from_bytes(q.astype("<u4").tobytes(), "little")
    slot = (2 * qi.bit_length() + N.bit_length() + 1 + 7) // 8
    slot = max(slot, 4 * L)

    def pack(x):
        buf = np.zeros((N, slot), np.uint8)
        buf[:, :4 * L] = x.astype("<u4").view(np.uint8).reshape(N, 4 * L)
        return buf

    A, B, C = _mpz(), _mpz(), _mpz()
    for z in (A, B, C):
        lib.__gmpz_init(ctypes.byref(z))
    try:
        pa, pb = pack(a), pack(b)
        lib.__gmpz_import(ctypes.byref(A), pa.size, -1, 1, 0, 0, pa.ctypes.data)
        lib.__gmpz_import(ctypes.byref(B), pb.size, -1, 1, 0, 0, pb.ctypes.data)
        lib.__gmpz_mul(ctypes.byref(C), ctypes.byref(A), ctypes.byref(B))
        out = np.zeros(2 * N * slot + 16, np.uint8)
        count = ctypes.c_size_t(0)
        lib.__gmpz_export(out.ctypes.data, ctypes.byref(count), -1, 1, 0, 0, ctypes.byref(C))
        raw = out[:2 * N * slot].tobytes()
    finally:
        for z in (A, B, C):
            lib.__gmpz_clear(ctypes.byref(z))
    res = bytearray()
    for k in range(N):
        lo = int.from_bytes(raw[k * slot:(k + 1) * slot], "little")
        hi = int.from_bytes(raw[(k + N) * slot:(k + N + 1) * slot], "little")
        res += ((lo - hi) % qi).to_bytes(4 * L, "little")
    return np.frombuffer(bytes(res), dtype="<u4").reshape(N, L).astype(np.uint32)


def schoolbook(q, a, b, coeffs=None) -> dict | np.ndarray:
    """Exact O(N^2) negacyclic product in Python big integers (reference
    oracle.py:81-91).  With ``coeffs`` (indices), only those coefficients are
    computed and a dict {k: limbs} is returned; otherwise the full N x L array."""
    q = np.asarray(q, dtype=np.uint32)
    N, L = a.shape
    qi = int.from_bytes(q.astype("<u4").tobytes(), "little")

    def ints(x):
        raw = np.ascontiguousarray(x, dtype="<u4").tobytes()
        return [int.from_bytes(raw[i * 4 * L:(i + 1) * 4 * L], "little") for i in range(N)]

    ai, bi = ints(a), ints(b)
    ks = range(N) if coeffs is None else coeffs
    out = {}
    for k in ks:
        s = 0
        for i in range(N):
            if ai[i] == 0:
                continue
            j = k - i
            if j >= 0:
                s += ai[i] * bi[j]
            else:
                s -= ai[i] * bi[j + N]
        out[k] = np.frombuffer((s % qi).to_bytes(4 * L, "little"), dtype="<u4").astype(np.uint32)
    if coeffs is not None:
        return out
    return np.stack([out[k] for k in range(N)])
