"""The modulus tables built on the device, and the prime-basis tables shared
between contexts.

fpm_init builds M_j = P / p_j mod q and negvP_v = -v P mod q on the device
(the reference's make_plan builds them on the host, rns_plan.h:224-247); the
q-independent tables are shared by every context on the device with the same
N, limb count, bit length of q and prime window.  These tests check the device
tables entry by entry against the oracle's plan, products of contexts sharing
a basis (also after the first of them is freed), and a server that takes a new
modulus while requests are in flight.
"""
import numpy as np
import pytest

import oracle
import polymul
from polymul import workload as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,W,bits", [(4096, 256, 30), (4096, 256, 31), (32768, 868, 30), (65536, 2048, 30),
                                      (65536, 1747, 31), (1024, 64, 30), (2048, 33, 30), (4096, 32, 30)])
def test_device_crt_tables_match_oracle(cuda, N, W, bits):
    q, _, _ = wl.case(2, W, "zero", seed=W + bits)
    with polymul.Context(N, W, q, prime_bits=bits) as ctx:
        M, negvP = ctx.crt_tables()
        eM, enegvP = oracle.OraclePlan(N, q, pmax_log2=bits).crt_tables()
        assert np.array_equal(M, eM)
        assert np.array_equal(negvP, enegvP)


def test_contexts_sharing_a_basis(cuda):
    N, W = 4096, 512
    rng = np.random.default_rng(11)
    qs = [wl.random_modulus(W, rng) for _ in range(3)]
    ctxs = [polymul.Context(N, W, q) for q in qs]
    assert len({c.K for c in ctxs}) == 1
    ops = [wl.operands(q, N, "uniform", rng) for q in qs]
    for c, q, (a, b) in zip(ctxs, qs, ops):
        assert np.array_equal(c.run(a, b), oracle.OraclePlan(N, q).polymul(a, b))
    ctxs[0].close()                    # the basis stays with the others
    for c, q, (a, b) in zip(ctxs[1:], qs[1:], ops[1:]):
        assert np.array_equal(c.run(a, b), oracle.OraclePlan(N, q).polymul(a, b))
    for c in ctxs[1:]:
        c.close()


def test_tuned_host_path_keeps_results(cuda):
    q, a, b = wl.case(65536, 2048, "uniform", seed=71)
    with polymul.Context(65536, 2048, q) as ctx:
        chunks = ctx.tune_host_path()
        assert 1 <= chunks <= 4
        assert np.array_equal(ctx.run(a, b), oracle.OraclePlan(65536, q).polymul(a, b))


def test_server_admits_new_modulus_mid_stream(cuda):
    N, W = 4096, 868
    rng = np.random.default_rng(12)
    q1, q2 = wl.random_modulus(W, rng), wl.random_modulus(W, rng)
    c1 = polymul.Context(N, W, q1)
    c2 = None
    srv = polymul.Server([c1], budget_bytes=1 << 30, lanes=2, max_batch=4)
    try:
        jobs = []
        for _ in range(8):
            a, b = wl.operands(q1, N, "uniform", rng)
            c = np.zeros((N, c1.L), np.uint32)
            jobs.append((0, q1, a, b, c, srv.submit(0, a, b, c)))
        c2 = polymul.Context(N, W, q2)       # a modulus the server has not seen
        p2 = srv.add_point(c2)
        for _ in range(8):
            a, b = wl.operands(q2, N, "uniform", rng)
            c = np.zeros((N, c2.L), np.uint32)
            jobs.append((p2, q2, a, b, c, srv.submit(p2, a, b, c)))
        for p, q, a, b, c, t in jobs:
            srv.wait(t)
            assert np.array_equal(c, oracle.OraclePlan(N, q).polymul(a, b)), f"point {p}"
    finally:
        srv.close()
        c1.close()
        if c2 is not None:
            c2.close()
