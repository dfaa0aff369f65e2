"""The host-facing paths on the GPU:

* the reference's own generated harness (main.cpp, built against its fherma.h and
  linked to this library by oracle/Makefile as oracle/_ref/solution_b200) runs a
  point directory in the reference's wire format through the exported C++
  fherma_init / fherma_run / fherma_free, bit-exact against the golden vectors,
  and refuses out-of-range points the way the reference does (non-zero exit, no
  output; fuzz.py:150-160);
* fpm_run with pinned and with pageable host buffers, for several I/O chunk
  counts, bit-exact against the oracle.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
import polymul
from conftest import ROOT, golden_cases, load_golden
from polymul import workload as wl

pytestmark = pytest.mark.gpu

HARNESS = os.path.join(ROOT, "oracle", "_ref", "solution_b200")


def write_point(root, N, W, q, cases):
    L = q.shape[0]
    os.makedirs(os.path.join(root, "point"), exist_ok=True)
    q.astype("<u4").tofile(os.path.join(root, "point", "q.bin"))
    with open(os.path.join(root, "manifest.json"), "w") as f:
        json.dump({"N": N, "W": W, "L": L, "cases": len(cases)}, f)
    for i, (a, b) in enumerate(cases):
        d = os.path.join(root, "cases", "%06d" % i)
        os.makedirs(d, exist_ok=True)
        a.astype("<u4").tofile(os.path.join(d, "a.bin"))
        b.astype("<u4").tofile(os.path.join(d, "b.bin"))


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="harness not built (make -C oracle)")
@pytest.mark.parametrize("entry", [c for c in golden_cases() if c["N"] in (64, 1024, 4096)],
                         ids=lambda c: c["file"][:-4])
def test_reference_harness_golden(cuda, tmp_path, entry):
    g = load_golden(entry)
    N, W = entry["N"], entry["W"]
    write_point(str(tmp_path), N, W, g["q"], [(g["a"], g["b"]), (g["b"], g["a"])])
    r = subprocess.run([HARNESS, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = json.load(open(tmp_path / "out" / "results.json"))
    assert [c["status"] for c in res["cases"]] == ["ok", "ok"]
    for i in range(2):
        c = np.fromfile(tmp_path / "out" / ("%06d" % i) / "c.bin", dtype="<u4").reshape(N, -1)
        assert np.array_equal(c, g["c"])


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="harness not built (make -C oracle)")
def test_reference_harness_full_size(cuda, tmp_path):
    N, W = 32768, 868
    q, a, b = wl.case(N, W, "max", seed=77)
    write_point(str(tmp_path), N, W, q, [(a, b)])
    r = subprocess.run([HARNESS, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    c = np.fromfile(tmp_path / "out" / "000000" / "c.bin", dtype="<u4").reshape(N, -1)
    assert np.array_equal(c, oracle.OraclePlan(N, q).polymul(a, b))


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="harness not built (make -C oracle)")
@pytest.mark.parametrize("N,W", [(1 << 23, 32), (1000, 64)])
def test_reference_harness_refuses_out_of_range(cuda, tmp_path, N, W):
    L = (W + 31) // 32
    q = np.zeros(L, np.uint32)
    q[0] = 0xFFFFFFFB
    os.makedirs(tmp_path / "point")
    q.astype("<u4").tofile(tmp_path / "point" / "q.bin")
    with open(tmp_path / "manifest.json", "w") as f:
        json.dump({"N": N, "W": W, "L": L, "cases": 0}, f)
    r = subprocess.run([HARNESS, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert not os.path.exists(tmp_path / "out" / "000000")


@pytest.mark.parametrize("chunks", ["1", "3", "4", "8"])
def test_host_paths_pinned_and_pageable(cuda, chunks, monkeypatch):
    torch = cuda
    monkeypatch.setenv("FPM_IO_CHUNKS", chunks)
    N, W = 65536, 1747
    q, a, b = wl.case(N, W, "uniform", seed=int(chunks))
    expect = oracle.OraclePlan(N, q).polymul(a, b)
    with polymul.Context(N, W, q) as ctx:
        assert np.array_equal(ctx.run(a, b), expect)                 # pageable in and out

        def pin(x):
            t = torch.empty(x.shape, dtype=torch.int32, pin_memory=True)
            v = t.numpy().view(np.uint32)
            v[...] = x
            return t, v

        (ta, pa), (tb, pb), (tc, pc) = pin(a), pin(b), pin(np.zeros_like(a))
        ctx.run(pa, pb, pc)
        assert np.array_equal(pc, expect)                             # pinned in and out
        c2 = np.zeros_like(a)
        ctx.run(pa, b, c2)
        assert np.array_equal(c2, expect)                             # mixed
        for _ in range(2):
            assert np.array_equal(ctx.run(a, pb), expect)
