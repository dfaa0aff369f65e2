"""The seeded synthetic operand generators."""
import numpy as np
import pytest

from polymul import workload as wl


@pytest.mark.parametrize("W", [2, 3, 31, 32, 33, 64, 255, 868, 1747, 2048])
def test_modulus_has_exactly_W_bits_and_is_odd(W):
    q = wl.random_modulus(W, np.random.Generator(np.random.PCG64(W)))
    qi = wl.to_int(q)
    assert qi.bit_length() == W and qi & 1
    assert q.shape[0] == (W + 31) // 32 and q[-1] != 0


@pytest.mark.parametrize("pattern", wl.PATTERNS)
def test_operands_are_canonical(pattern):
    q, a, b = wl.case(512, 300, pattern, seed=4)
    qi = wl.to_int(q)
    for x in (a, b):
        assert x.shape == (512, q.shape[0]) and x.dtype == np.uint32
        assert all(v < qi for v in wl.rows_to_ints(x))


def test_seeded_cases_are_deterministic():
    q1, a1, b1 = wl.case(1024, 868, "uniform", seed=11)
    q2, a2, b2 = wl.case(1024, 868, "uniform", seed=11)
    assert np.array_equal(q1, q2) and np.array_equal(a1, a2) and np.array_equal(b1, b2)


def test_sparse_is_mostly_zero():
    _, a, _ = wl.case(8192, 256, "sparse", seed=3)
    zero = (a == 0).all(axis=1).mean()
    assert 0.85 < zero < 0.95


def test_uniform_hits_the_top_of_the_range():
    q, a, _ = wl.case(4096, 40, "uniform", seed=8)
    vals = np.array(wl.rows_to_ints(a), dtype=object)
    qi = wl.to_int(q)
    assert max(vals) > qi * 0.99 and min(vals) < qi * 0.01


def test_poisson_arrivals_seeded_and_rate():
    t1 = wl.poisson_arrivals(10000, 2000.0, seed=7)
    t2 = wl.poisson_arrivals(10000, 2000.0, seed=7)
    assert np.array_equal(t1, t2)
    gaps = np.diff(np.concatenate([[0.0], t1]))
    assert (gaps > 0).all()
    assert abs(gaps.mean() - 500.0) < 15.0          # mean gap 1e6 / rate us


def test_mix_points_draw_from_the_mix():
    pts = wl.mix_points(64, seed=4000)
    assert len(pts) == 64
    for N, W, q in pts:
        assert N in wl.MIX_N and W in wl.MIX_W
        assert q.shape[0] == (W + 31) // 32 and q[0] & 1
        assert wl.to_int(q).bit_length() == W
