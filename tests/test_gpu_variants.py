"""The column-pass variants (FPM_COL_PASS: plain, tma1, tma2) give the same
products, bit for bit, as the oracle.  The variable is read once per process,
so each variant runs in a child process that writes its products to a file.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from polymul import workload as wl

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
POINTS = [(65536, 2048), (8192, 256)]

CHILD = r"""
import sys, numpy as np
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/fherma-polymult_b200"]
import polymul
from polymul import workload as wl
out = {}
for spec in sys.argv[3:]:
    N, W = map(int, spec.split("x"))
    q, a, b = wl.case(N, W, "uniform", seed=N + W)
    with polymul.Context(N, W, q) as ctx:
        out[spec] = ctx.run(a, b)
np.savez(sys.argv[2], **out)
"""


@pytest.fixture(scope="module")
def expected():
    want = {}
    for N, W in POINTS:
        q, a, b = wl.case(N, W, "uniform", seed=N + W)
        want[f"{N}x{W}"] = oracle.OraclePlan(N, q).polymul(a, b)
    return want


@pytest.mark.parametrize("variant", ["plain", "tma1", "tma2"])
def test_column_pass_variants(cuda, expected, variant, tmp_path):
    path = tmp_path / f"{variant}.npz"
    env = dict(os.environ, FPM_COL_PASS=variant)
    specs = [f"{N}x{W}" for N, W in POINTS]
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(path), *specs], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.load(path)
    for spec in specs:
        assert np.array_equal(got[spec], expected[spec]), f"{variant} {spec}"
