"""Host-side checks of the shipped library that need no GPU: it loads, it
exports every symbol include/*.h declares, its host plan agrees with the oracle
and the reference, and it refuses bad points and runs nothing without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
import polymul
from conftest import ROOT
from polymul import workload as wl

HEADER_C = os.path.join(ROOT, "include", "fherma_polymult.h")
CPP_SYMBOLS = ["_Z11fherma_initRKN6fherma5PointE", "_Z10fherma_runPvRKN6fherma6InputsE", "_Z11fherma_freePv"]


def declared_c_symbols():
    text = open(HEADER_C).read()
    return sorted(set(re.findall(r"FPM_API\s+[\w\s\*]+?\b(fpm_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = polymul.load()
    names = declared_c_symbols()
    assert {"fpm_init", "fpm_run", "fpm_run_device", "fpm_free", "fpm_last_error"} <= set(names), names
    for name in names:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", polymul.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for name in names + CPP_SYMBOLS:
        assert name in exported, name


@pytest.mark.parametrize("N,W", [(2, 3), (4, 65), (256, 128), (1024, 868), (2048, 129), (4096, 256),
                                 (8192, 512), (32768, 868), (65536, 1747), (65536, 2048), (1 << 17, 512)])
def test_plan_primes_match_oracle(N, W):
    q, _, _ = wl.case(2, W, "zero", seed=N ^ W)
    for bits in (30, 31):
        info, primes = polymul.plan_info(N, W, q, prime_bits=bits)
        pl = oracle.OraclePlan(N, q, pmax_log2=bits)
        assert info.K == pl.K and info.prime_bits == bits
        assert np.array_equal(primes, pl.primes)
        assert int(primes.max()) < 2**bits
    info, primes = polymul.plan_info(N, W, q)
    assert info.prime_bits == 30
    assert info.N == N and info.L == q.shape[0]
    assert info.logR + info.logS == info.logN == N.bit_length() - 1
    assert info.device == -1


def test_footprint_covers_workspaces():
    q, _, _ = wl.case(2, 2048, "zero", seed=9)
    info, _ = polymul.plan_info(65536, 2048, q)
    assert info.device_bytes >= 2 * info.K * 65536 * 4 + 3 * 65536 * 64 * 4


@pytest.mark.parametrize("N,L", [(3, 2), (1 << 23, 1), (0, 1), (64, 65), (64, 0)])
def test_bad_points_are_refused(N, L):
    q = np.ones(max(L, 1), np.uint32)
    with pytest.raises(polymul.FpmError) as e:
        polymul.plan_info(N, 32 * L, q[:L] if L else q[:0])
    assert e.value.code == polymul.FPM_EINVAL


def test_top_limb_zero_refused():
    with pytest.raises(polymul.FpmError):
        polymul.plan_info(64, 64, np.array([5, 0], np.uint32))


def test_no_cpu_fallback_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    q, _, _ = wl.case(2, 256, "zero", seed=1)
    with pytest.raises(polymul.FpmError) as e:
        polymul.Context(4096, 256, q)
    assert e.value.code == polymul.FPM_ECUDA


def test_missing_library_fails_loudly(tmp_path):
    saved = polymul._lib
    polymul._lib = None
    try:
        with pytest.raises(RuntimeError):
            polymul.load(str(tmp_path / "libfpm.so"))
    finally:
        polymul._lib = saved
