"""Batches (fpm_batch): many products of uneven N and q in one CUDA graph of
grouped launches must give, product by product, exactly what the plain entry
point gives, for every schedule the autotuner can pick.

The plain path is itself checked against the oracle (test_gpu_parity.py); here
a few products are also checked against the oracle directly.
"""
import numpy as np
import pytest

import oracle
import polymul
from polymul import workload as wl

pytestmark = pytest.mark.gpu

# (N, W, prime_bits): every geometry class, the single-tile row pass (N = 2048),
# the one-block-per-prime transform (N <= 1024), one-limb moduli (CUDA-core
# CRT), and both prime windows (lazy and full-reduction butterflies).
MIXED = [(65536, 2048, 0), (32768, 868, 0), (16384, 512, 0), (8192, 1747, 0), (4096, 128, 0), (2048, 256, 0),
         (1024, 64, 0), (64, 32, 0), (4096, 32, 0), (16384, 868, 31), (4096, 256, 31)]

# (layout, order, prime_group, grid, pipe_min_log_n)
SCHEDULES = [(0, 1, 0, 0, 0), (1, 1, 0, 0, 0), (2, 1, 0, 0, 0), (1, 0, 16, 1, 0), (2, 1, 16, 2, 0), (0, 0, 8, 1, 0),
             (1, 1, 3, 0, 0), (1, 1, 0, 0, 11), (2, 0, 16, 1, 12), (0, 1, 0, 0, 16), (3, 1, 0, 0, 0), (3, 0, 16, 1, 0),
             (3, 1, 5, 2, 16)]


@pytest.fixture(scope="module")
def mixed(cuda):
    ctxs, ops, expect = [], [], []
    for i, (N, W, bits) in enumerate(MIXED):
        q, a, b = wl.case(N, W, "uniform", seed=900 + i)
        ctx = polymul.Context(N, W, q, prime_bits=bits)
        ctxs.append(ctx)
        ops.append((a, b))
        expect.append(ctx.run(a, b))
    # The first context a second time, with other operands.
    q0 = wl.case(MIXED[0][0], MIXED[0][1], "uniform", seed=900)[0]
    a2, b2 = wl.operands(q0, MIXED[0][0], "max", np.random.default_rng(5))
    ctxs.append(ctxs[0])
    ops.append((a2, b2))
    expect.append(ctxs[0].run(a2, b2))
    yield ctxs, ops, expect
    for c in ctxs:
        c.close()


def test_batch_members_match_oracle(mixed):
    """Every member of the mix, the N = 65536 / 2048-bit ones included, against
    the oracle (the batch schedules below are then checked against these)."""
    ctxs, ops, expect = mixed
    for ctx, (a, b), e in zip(ctxs, ops, expect):
        q = oracle_q(ctx)
        bits = 31 if ctx.prime_bits == 31 else 30
        assert np.array_equal(e, oracle.OraclePlan(ctx.N, q, pmax_log2=bits).polymul(a, b)), (ctx.N, ctx.W)


def oracle_q(ctx):
    for i, (N, W, bits) in enumerate(MIXED):
        if (N, W) == (ctx.N, ctx.W):
            return wl.case(N, W, "uniform", seed=900 + i)[0]
    raise KeyError


def test_batch_n65536_members_match_oracle(cuda):
    """Two N = 65536 products (W = 2048 and 1747) in one batch with the tuned
    schedule, each against the oracle."""
    pts = [(65536, 2048), (65536, 1747)]
    ctxs, qs, ops = [], [], []
    try:
        for i, (N, W) in enumerate(pts):
            q, a, b = wl.case(N, W, "uniform", seed=3100 + i)
            ctxs.append(polymul.Context(N, W, q))
            qs.append(q)
            ops.append((a, b))
        with polymul.Batch(ctxs) as bt:
            bt.tune(reps=1)
            got = bt.run([a for a, _ in ops], [b for _, b in ops])
        for (N, W), q, (a, b), g in zip(pts, qs, ops, got):
            assert np.array_equal(g, oracle.OraclePlan(N, q).polymul(a, b)), (N, W)
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("sched", SCHEDULES, ids=lambda s: "L%d-o%d-g%d-p%d-pipe%d" % s)
def test_batch_matches_plain(mixed, sched):
    ctxs, ops, expect = mixed
    with polymul.Batch(ctxs) as bt:
        bt.set_schedule(*sched)
        info = bt.info
        assert (info.layout, info.order, info.prime_group, info.grid, info.pipe_min_log_n) == sched
        assert info.count == len(ctxs) and info.launches > 0
        for rep in range(2):   # a replay of the same graph gives the same results
            got = bt.run([a for a, _ in ops], [b for _, b in ops])
            for g, e in zip(got, expect):
                assert np.array_equal(g, e)


def test_batch_tune_keeps_results(mixed):
    ctxs, ops, expect = mixed
    with polymul.Batch(ctxs) as bt:
        bt.run([a for a, _ in ops], [b for _, b in ops])
        info = bt.tune(reps=2)
        assert info.tuned_us > 0 and 0 <= info.layout <= 3
        got = bt.run([a for a, _ in ops], [b for _, b in ops])
        for g, e in zip(got, expect):
            assert np.array_equal(g, e)


def test_batch_beyond_one_table(cuda):
    """70 products: more than one grouped table per launch."""
    pts = [(4096, (128, 512)[i % 2]) for i in range(70)]
    ctxs = []
    try:
        ops, expect = [], []
        for i, (N, W) in enumerate(pts):
            q, a, b = wl.case(N, W, "uniform", seed=2000 + i)
            ctx = polymul.Context(N, W, q)
            ctxs.append(ctx)
            ops.append((a, b))
            expect.append(ctx.run(a, b))
        with polymul.Batch(ctxs) as bt:
            for sched in [(0, 1, 0, 0, 0), (1, 1, 4, 1, 12)]:
                bt.set_schedule(*sched)
                got = bt.run([a for a, _ in ops], [b for _, b in ops])
                for g, e in zip(got, expect):
                    assert np.array_equal(g, e)
    finally:
        for c in ctxs:
            c.close()


def test_batch_mix_matches_plain(cuda):
    """A seeded draw of the batched mix (N 4096 .. 65536, W 128 .. 2048)."""
    pts = wl.mix_points(24, seed=4001)
    ops = wl.mix_operands(pts, seed=4002)
    ctxs = [polymul.Context(N, W, q) for N, W, q in pts]
    try:
        expect = [c.run(a, b) for c, (a, b) in zip(ctxs, ops)]
        with polymul.Batch(ctxs) as bt:
            bt.tune(reps=1)
            got = bt.run([a for a, _ in ops], [b for _, b in ops])
            for g, e in zip(got, expect):
                assert np.array_equal(g, e)
    finally:
        for c in ctxs:
            c.close()


def test_batch_errors(cuda):
    q, a, b = wl.case(4096, 128, "uniform", seed=1)
    with polymul.Context(4096, 128, q) as ctx:
        with polymul.Batch([ctx]) as bt:
            with pytest.raises(polymul.FpmError) as e:
                bt.set_schedule(4, 1, 0, 0)
            with pytest.raises(polymul.FpmError):
                bt.set_schedule(1, 1, 0, 0, 40)
            assert e.value.code == polymul.FPM_EINVAL
            with pytest.raises(polymul.FpmError):
                bt.buffers(1)
            with pytest.raises(polymul.FpmError):
                bt.run([a], [b[:100]])
            assert np.array_equal(bt.run([a], [b])[0], ctx.run(a, b))
