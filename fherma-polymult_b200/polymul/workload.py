"""Seeded synthetic operands for the negacyclic product.

No public benchmark set is involved: every modulus and operand is drawn from a
seeded numpy PCG64 generator.  Conventions:

* q is a random odd integer with exactly W bits (bit W-1 and bit 0 set), stored
  as L = ceil(W/32) little-endian u32 limbs, so the top limb is nonzero (the
  reference's plan requires that, rns_plan.h:134).
* Operands are N x L u32 arrays, coefficient-major (row n = coefficient n's
  limbs, least significant first), the layout of fherma::Inputs (fherma.h:34-37).
* Distributions: "uniform" in [0, q) (rejection sampling, so exactly uniform),
  "max" (every coefficient q - 1), "sparse" (90% zeros, the rest uniform), plus
  the known-answer patterns the reference's fuzzer uses (fuzz.py:53-63):
  "zero", "wrap", "identity", "alternating".
"""
from __future__ import annotations

import numpy as np

PATTERNS = ("uniform", "max", "sparse", "zero", "wrap", "identity", "alternating")


def limbs_of(W: int) -> int:
    return (W + 31) // 32


def to_int(limbs) -> int:
    """Little-endian u32 limbs -> Python int."""
    return int.from_bytes(np.asarray(limbs, dtype="<u4").tobytes(), "little")


def from_int(x: int, L: int) -> np.ndarray:
    """Python int -> L little-endian u32 limbs."""
    return np.frombuffer(int(x).to_bytes(4 * L, "little"), dtype="<u4").astype(np.uint32)


def rows_to_ints(rows: np.ndarray) -> list:
    """N x L limbs -> list of N Python ints."""
    raw = np.ascontiguousarray(rows, dtype="<u4").tobytes()
    w = 4 * rows.shape[1]
    return [int.from_bytes(raw[i * w:(i + 1) * w], "little") for i in range(rows.shape[0])]


def ints_to_rows(values, L: int) -> np.ndarray:
    out = bytearray()
    for v in values:
        out += int(v).to_bytes(4 * L, "little")
    return np.frombuffer(bytes(out), dtype="<u4").reshape(len(values), L).astype(np.uint32)


def random_modulus(W: int, rng: np.random.Generator) -> np.ndarray:
    """A random odd modulus with exactly W bits (W >= 2), as L limbs."""
    if W < 2:
        raise ValueError("W must be at least 2")
    L = limbs_of(W)
    q = rng.integers(0, 1 << 32, size=L, dtype=np.uint64).astype(np.uint32)
    top_bits = W - 32 * (L - 1)
    top_mask = np.uint32((1 << top_bits) - 1) if top_bits < 32 else np.uint32(0xFFFFFFFF)
    q[L - 1] &= top_mask
    q[L - 1] |= np.uint32(1 << (top_bits - 1))
    q[0] |= np.uint32(1)
    return q


def _less_than(rows: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Row-wise rows < q as multi-limb integers."""
    diff = rows != q[None, :]
    any_diff = diff.any(axis=1)
    # index of the most significant differing limb
    top = rows.shape[1] - 1 - np.argmax(diff[:, ::-1], axis=1)
    n = np.arange(rows.shape[0])
    return any_diff & (rows[n, top] < q[top])


def uniform_below(q: np.ndarray, count: int, rng: np.random.Generator) -> np.ndarray:
    """count values uniform in [0, q), count x L limbs (rejection sampling)."""
    L = q.shape[0]
    bits = int(q[L - 1]).bit_length()
    top_mask = np.uint32((1 << bits) - 1) if bits < 32 else np.uint32(0xFFFFFFFF)
    out = np.empty((count, L), dtype=np.uint32)
    todo = np.arange(count)
    while todo.size:
        cand = rng.integers(0, 1 << 32, size=(todo.size, L), dtype=np.uint64).astype(np.uint32)
        cand[:, L - 1] &= top_mask
        ok = _less_than(cand, q)
        out[todo[ok]] = cand[ok]
        todo = todo[~ok]
    return out


def minus_one(q: np.ndarray) -> np.ndarray:
    L = q.shape[0]
    return from_int(to_int(q) - 1, L)


def operands(q: np.ndarray, N: int, pattern: str, rng: np.random.Generator):
    """(a, b), each N x L u32, for one of PATTERNS."""
    L = q.shape[0]
    if pattern == "uniform":
        return uniform_below(q, N, rng), uniform_below(q, N, rng)
    if pattern == "max":
        m = minus_one(q)
        a = np.tile(m, (N, 1))
        return a, a.copy()
    if pattern == "sparse":
        a, b = uniform_below(q, N, rng), uniform_below(q, N, rng)
        a[rng.random(N) < 0.9] = 0
        b[rng.random(N) < 0.9] = 0
        return a, b
    if pattern == "zero":
        return np.zeros((N, L), np.uint32), uniform_below(q, N, rng)
    if pattern == "wrap":
        # x^(N-1) * (q-1) x^(N-1) = -(q-1) x^(N-2): known answer c[N-2] = 1, all
        # other coefficients 0 (for N = 2 the product is -(q-1) x^0, also 1).
        a = np.zeros((N, L), np.uint32)
        b = np.zeros((N, L), np.uint32)
        a[N - 1, 0] = 1
        b[N - 1] = minus_one(q)
        return a, b
    if pattern == "identity":
        b = np.zeros((N, L), np.uint32)
        b[0, 0] = 1
        return uniform_below(q, N, rng), b
    if pattern == "alternating":
        m = minus_one(q)
        a = np.zeros((N, L), np.uint32)
        b = np.zeros((N, L), np.uint32)
        a[1::2] = m
        b[0::2] = m
        return a, b
    raise ValueError(f"unknown pattern {pattern!r}")


def case(N: int, W: int, pattern: str = "uniform", seed: int = 0):
    """(q, a, b) for one seeded case: PCG64(seed) draws q, then the operands."""
    rng = np.random.Generator(np.random.PCG64(seed))
    q = random_modulus(W, rng)
    a, b = operands(q, N, pattern, rng)
    return q, a, b


MIX_N = (4096, 8192, 16384, 32768, 65536)
MIX_W = (128, 512, 868, 1747, 2048)


def mix_points(count: int, seed: int):
    """(N, W, q) for `count` products drawn from the batched / serving mix:
    N from MIX_N and W from MIX_W, uniformly, each with its own seeded q."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        N = int(rng.choice(MIX_N))
        W = int(rng.choice(MIX_W))
        out.append((N, W, random_modulus(W, rng)))
    return out


def mix_operands(points, seed: int):
    """Uniform operands below each point's q."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [operands(q, N, "uniform", rng) for N, W, q in points]


def poisson_arrivals(count: int, rate_per_s: float, seed: int) -> np.ndarray:
    """Arrival times (us) of a seeded Poisson stream: exponential gaps of mean
    1e6 / rate_per_s, starting at the first gap."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1e6 / rate_per_s, size=count))
