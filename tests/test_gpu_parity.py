"""Parity of the CUDA path with the oracle, through the C ABI.  Bit-exact
everywhere (integer arithmetic).

* every golden vector the reference wrote, through fpm_run (host buffers);
* stage by stage (decompose, forward transform, y_j, CRT) against the oracle
  across every transform geometry;
* full-size products at the benchmark points, bit-exact against the oracle
  (which was pinned against the reference and GMP in test_oracle.py);
* device-buffer and host-buffer paths agree; repeated calls are identical.
"""
import numpy as np
import pytest

import oracle
import polymul
from conftest import golden_cases, load_golden
from polymul import workload as wl

pytestmark = pytest.mark.gpu

CASES = golden_cases()


def dev(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint32).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


def scaled(pl, res, N):
    """The decompose of operand b: residues times N^-1 (P/p_j)^-1 2^32 mod p_j."""
    primes = [int(p) for p in pl.primes]
    out = np.empty_like(res)
    for j, p in enumerate(primes):
        Pj = 1
        for i, pi in enumerate(primes):
            if i != j:
                Pj = Pj * pi % p
        s = pow(N, p - 2, p) * pow(Pj, p - 2, p) % p * (2**32 % p) % p
        out[j] = (res[j].astype(np.uint64) * s % p).astype(np.uint32)
    return out


@pytest.mark.parametrize("entry", CASES, ids=[c["file"][:-4] for c in CASES])
def test_golden_vectors(cuda, entry):
    """Default prime window (p < 2^30): same products as the reference."""
    g = load_golden(entry)
    with polymul.Context(entry["N"], entry["W"], g["q"]) as ctx:
        assert ctx.prime_bits == 30
        assert np.array_equal(ctx.run(g["a"], g["b"]), g["c"])


@pytest.mark.parametrize("entry", CASES[::2], ids=[c["file"][:-4] for c in CASES[::2]])
def test_golden_vectors_reference_primes(cuda, entry):
    """prime_bits = 31: the reference's own prime set, bit for bit."""
    g = load_golden(entry)
    with polymul.Context(entry["N"], entry["W"], g["q"], prime_bits=31) as ctx:
        assert ctx.K == int(g["K"])
        assert np.array_equal(ctx.primes, g["primes"])
        assert np.array_equal(ctx.run(g["a"], g["b"]), g["c"])


# Every transform split: one block per prime (N <= 1024), the single row tile
# (N = 2048), R = 64 columns with rows of 2^6 .. 2^11 (N = 2^12 .. 2^17), and
# rows of 2048 with columns of 2^7 .. 2^11 (N = 2^18 .. 2^22, the 16-element
# column rounds).
GEOMETRIES = [(2, 33), (8, 97), (64, 100), (512, 250), (1024, 512), (2048, 129), (4096, 256), (8192, 868),
              (16384, 300), (32768, 868), (65536, 2048), (1 << 17, 512), (1 << 18, 128), (1 << 19, 96),
              (1 << 20, 64), (1 << 21, 48), (1 << 22, 32)]


@pytest.mark.parametrize("prime_bits", [30, 31])
@pytest.mark.parametrize("N,W", GEOMETRIES)
def test_stages_match_oracle(cuda, N, W, prime_bits):
    torch = cuda
    q, a, b = wl.case(N, W, "uniform", seed=N + W)
    pl = oracle.OraclePlan(N, q, pmax_log2=prime_bits)
    with polymul.Context(N, W, q, prime_bits=prime_bits) as ctx:
        assert np.array_equal(ctx.primes, pl.primes)
        K = ctx.K
        da, db = dev(torch, a), dev(torch, b)
        A = torch.zeros((K, N), dtype=torch.int32, device="cuda")
        B = torch.zeros((K, N), dtype=torch.int32, device="cuda")
        ctx.stage_decompose(da.data_ptr(), A.data_ptr(), 0)
        ctx.stage_decompose(db.data_ptr(), B.data_ptr(), 1)
        torch.cuda.synchronize()
        ra, rb = pl.decompose(a), pl.decompose(b)
        # Canonical, or below 4p and congruent (30-bit primes, N > 1024).
        pj = ctx.primes.astype(np.uint64)[:, None]
        bound = 4 if prime_bits == 30 and N > 1024 else 1
        for got, want, what in ((host(A), ra, "decompose a"), (host(B), scaled(pl, rb, N), "decompose b (scaled)")):
            assert (got.astype(np.uint64) < bound * pj).all(), what + ": range"
            assert np.array_equal(got.astype(np.uint64) % pj, want.astype(np.uint64)), what
        # The paired launch a product uses (operand 2: a then b in, A then B out).
        AB = torch.zeros((2 * K, N), dtype=torch.int32, device="cuda")
        lab = torch.cat((da, db))
        ctx.stage_decompose(lab.data_ptr(), AB.data_ptr(), 2)
        torch.cuda.synchronize()
        assert np.array_equal(host(AB[:K]), host(A)) and np.array_equal(host(AB[K:]), host(B)), "paired decompose"
        rb_s = scaled(pl, rb, N)

        ctx.stage_transform(A.data_ptr(), B.data_ptr(), polymul.MODE_FORWARD)
        torch.cuda.synchronize()
        assert np.array_equal(host(A), pl.ntt_forward(ra)), "forward transform of a"
        assert np.array_equal(host(B), pl.ntt_forward(rb_s)), "forward transform of b"

        ctx.stage_decompose(da.data_ptr(), A.data_ptr(), 0)
        ctx.stage_decompose(db.data_ptr(), B.data_ptr(), 1)
        ctx.stage_transform(A.data_ptr(), B.data_ptr(), polymul.MODE_PRODUCT)
        torch.cuda.synchronize()
        c_ref, y_ref = pl.polymul(a, b, want_y=True)
        assert np.array_equal(host(A), y_ref), "y_j"

        C = torch.zeros((N, ctx.L), dtype=torch.int32, device="cuda")
        ctx.stage_crt(dev(torch, y_ref).data_ptr(), C.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(host(C), c_ref), "crt"


FULL = [(65536, 2048, "uniform"), (65536, 2048, "max"), (65536, 1747, "uniform"), (65536, 1747, "max"),
        (32768, 868, "uniform"), (32768, 868, "max"), (32768, 868, "sparse")]


@pytest.mark.parametrize("N,W,pattern", FULL)
def test_full_size_products(cuda, N, W, pattern):
    q, a, b = wl.case(N, W, pattern, seed=7 * N + W)
    expect = oracle.OraclePlan(N, q).polymul(a, b)
    with polymul.Context(N, W, q) as ctx:
        assert np.array_equal(ctx.run(a, b), expect)
    if pattern == "max":
        with polymul.Context(N, W, q, prime_bits=31) as ctx:
            assert np.array_equal(ctx.run(a, b), expect)


def test_device_path_matches_host_path_and_repeats(cuda):
    torch = cuda
    N, W = 65536, 2048
    q, a, b = wl.case(N, W, "uniform", seed=123)
    with polymul.Context(N, W, q) as ctx:
        c_host = ctx.run(a, b)
        da, db = dev(torch, a), dev(torch, b)
        dc = torch.zeros((N, ctx.L), dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        for _ in range(3):
            dc.zero_()
            torch.cuda.synchronize()
            ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), s.cuda_stream)
            s.synchronize()
            assert np.array_equal(host(dc), c_host)
        assert np.array_equal(ctx.run(a, b), c_host)


@pytest.mark.parametrize("N,W", [(65536, 2048), (4096, 868), (1024, 1747)])
def test_unaligned_device_buffers(cuda, N, W):
    """Operands, result and y at a one-word offset: the pipelined decompose
    and CRT take their word-wise load and store paths (and a y that is not
    16-byte aligned goes to the per-tile CRT), with the same results."""
    torch = cuda
    q, a, b = wl.case(N, W, "uniform", seed=N + 3)
    L = q.shape[0]
    with polymul.Context(N, W, q) as ctx:
        da, db = dev(torch, a), dev(torch, b)
        dc = torch.empty_like(da)
        ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr())
        expect = host(dc)

        def shifted(x):
            t = torch.zeros(x.numel() + 1, dtype=torch.int32, device="cuda")
            t[1:] = x.reshape(-1)
            return t

        sa, sb, sc = shifted(da), shifted(db), torch.zeros(N * L + 1, dtype=torch.int32, device="cuda")
        ctx.run_device(sa.data_ptr() + 4, sb.data_ptr() + 4, sc.data_ptr() + 4)
        assert np.array_equal(sc[1:].cpu().numpy().view(np.uint32).reshape(N, L), expect)
        # y through the stage entry points, at an offset too.
        K = ctx.K
        A = torch.zeros(K * N + 1, dtype=torch.int32, device="cuda")
        B = torch.zeros(K * N + 1, dtype=torch.int32, device="cuda")
        ctx.stage_decompose(sa.data_ptr() + 4, A.data_ptr() + 4, 0)
        ctx.stage_decompose(sb.data_ptr() + 4, B.data_ptr() + 4, 1)
        ctx.stage_transform(A.data_ptr() + 4, B.data_ptr() + 4, polymul.MODE_PRODUCT)
        sc.zero_()
        ctx.stage_crt(A.data_ptr() + 4, sc.data_ptr() + 4)
        torch.cuda.synchronize()
        assert np.array_equal(sc[1:].cpu().numpy().view(np.uint32).reshape(N, L), expect)


@pytest.mark.parametrize("N,W", [(4096, 256), (2, 2048), (1 << 18, 128)])
def test_known_answer_patterns(cuda, N, W):
    for pattern in ("zero", "identity", "wrap"):
        q, a, b = wl.case(N, W, pattern, seed=N + len(pattern))
        with polymul.Context(N, W, q) as ctx:
            c = ctx.run(a, b)
        if pattern == "zero":
            assert not c.any()
        elif pattern == "identity":
            assert np.array_equal(c, a)
        else:
            expect = np.zeros_like(c)
            expect[N - 2, 0] = 1
            assert np.array_equal(c, expect)


def test_error_behaviour(cuda):
    q, a, b = wl.case(1024, 512, "uniform", seed=3)
    with pytest.raises(polymul.FpmError) as e:
        polymul.Context(1000, 512, q)
    assert e.value.code == polymul.FPM_EINVAL
    with pytest.raises(polymul.FpmError):
        polymul.Context(1 << 23, 512, q)
    with polymul.Context(1024, 512, q) as ctx:
        with pytest.raises(polymul.FpmError):
            ctx.run(a[:-1], b)
        # the context stays usable after a refused call
        assert np.array_equal(ctx.run(a, b), oracle.OraclePlan(1024, q).polymul(a, b))
