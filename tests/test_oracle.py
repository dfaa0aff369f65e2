"""The oracle is pinned before it is trusted: our C restatement, the GMP
Kronecker product and the Python schoolbook are checked against the golden
vectors the REFERENCE's own CPU build wrote (tests/golden/make_golden.py), and
the restated plan against the reference's make_plan tables."""
import numpy as np
import pytest

import oracle
from conftest import golden_cases, load_golden
from polymul import workload as wl

CASES = golden_cases()


@pytest.mark.parametrize("entry", CASES, ids=[c["file"][:-4] for c in CASES])
def test_oracle_matches_reference_golden(entry):
    g = load_golden(entry)
    pl = oracle.OraclePlan(entry["N"], g["q"])
    assert pl.K == int(g["K"])
    assert np.array_equal(pl.primes, g["primes"])
    c = pl.polymul(g["a"], g["b"])
    assert np.array_equal(c, g["c"])


@pytest.mark.parametrize("entry", CASES[::3], ids=[c["file"][:-4] for c in CASES[::3]])
def test_gmp_matches_reference_golden(entry):
    g = load_golden(entry)
    assert np.array_equal(oracle.kronecker(g["q"], g["a"], g["b"]), g["c"])


@pytest.mark.parametrize("entry", [c for c in CASES if c["N"] <= 64],
                         ids=[c["file"][:-4] for c in CASES if c["N"] <= 64])
def test_schoolbook_matches_reference_golden(entry):
    g = load_golden(entry)
    assert np.array_equal(oracle.schoolbook(g["q"], g["a"], g["b"]), g["c"])


def test_schoolbook_sampled_coefficients():
    g = load_golden(next(c for c in CASES if c["N"] == 4096 and c["pattern"] == "uniform"))
    ks = [0, 1, 2047, 4094, 4095]
    got = oracle.schoolbook(g["q"], g["a"], g["b"], coeffs=ks)
    for k in ks:
        assert np.array_equal(got[k], g["c"][k])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU build not present")
@pytest.mark.parametrize("N,W", [(2, 3), (64, 100), (1024, 868), (4096, 256), (32768, 868), (65536, 1747),
                                 (65536, 2048), (1 << 17, 512)])
def test_plan_tables_match_reference(N, W):
    q, _, _ = wl.case(2, W, "zero", seed=N + W)
    ref = oracle.ref_plan(N, q)
    pl = oracle.OraclePlan(N, q)
    M, negvP = pl.crt_tables()
    assert pl.K == ref["K"]
    assert np.array_equal(pl.primes, ref["primes"])
    assert np.array_equal(pl.roots, ref["roots"])
    assert np.array_equal(M, ref["M"])
    assert np.array_equal(negvP, ref["negvP"])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU build not present")
def test_oracle_matches_reference_at_config_size():
    q, a, b = wl.case(32768, 868, "max", seed=2)
    c_ref, _ = oracle.ref_polymul(32768, 868, q, a, b)
    assert np.array_equal(oracle.OraclePlan(32768, q).polymul(a, b), c_ref)


def test_known_answers():
    N, W = 256, 300
    q, a, b = wl.case(N, W, "wrap", seed=5)
    c = oracle.OraclePlan(N, q).polymul(a, b)
    expect = np.zeros_like(c)
    expect[N - 2, 0] = 1                       # x^(N-1) (q-1) x^(N-1) = -(q-1) x^(N-2) = 1 x^(N-2)
    assert np.array_equal(c, expect)
    q, a, b = wl.case(N, W, "identity", seed=6)
    assert np.array_equal(oracle.OraclePlan(N, q).polymul(a, b), a)
    q, a, b = wl.case(N, W, "zero", seed=7)
    assert not oracle.OraclePlan(N, q).polymul(a, b).any()


def test_out_of_range_points_refused():
    q, _, _ = wl.case(2, 64, "zero", seed=1)
    for N in (3, 1 << 23, 1):
        with pytest.raises(ValueError):
            oracle.OraclePlan(N, q)
    with pytest.raises(ValueError):
        oracle.OraclePlan(64, np.zeros(65, np.uint32) + 1)
