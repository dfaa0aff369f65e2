"""Writes the golden vectors in tests/golden/ by running the REFERENCE's own CPU
implementation (solve_cpu.cpp, built from the reference tree into oracle/_ref/
by `make -C oracle`) on seeded inputs.

    python tests/golden/make_golden.py

Each case file NNN_N<N>_W<W>_<pattern>.npz holds q, a, b, the reference's c, and
the reference's plan (K and the primes).  manifest.json lists the cases.  The
points follow the reference's own test matrix (run_tests.sh:18-21, fuzz.py:119-
123): every NTT geometry up to N = 4096, the limb edges (L = 1, a q that fills its
limbs, one bit into a new limb, L = 64) and the fuzzer's six operand patterns
(fuzz.py:53-63), plus the sparse distribution.  Sizes are kept small so the
fixtures stay around a megabyte.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "fherma-polymult_b200"))

import oracle  # noqa: E402
from polymul import workload  # noqa: E402

CASES = [
    # (N, W, pattern)
    (2, 3, "uniform"), (2, 32, "max"), (2, 33, "uniform"), (4, 30, "uniform"), (4, 64, "max"),
    (4, 65, "wrap"), (8, 60, "uniform"), (8, 97, "alternating"), (16, 64, "uniform"),
    (16, 127, "identity"), (32, 31, "uniform"), (64, 32, "uniform"), (64, 100, "wrap"),
    (64, 2047, "max"), (64, 2048, "uniform"), (128, 1023, "uniform"), (128, 1025, "sparse"),
    (128, 2048, "max"), (256, 63, "uniform"), (256, 64, "zero"), (256, 65, "uniform"),
    (256, 128, "uniform"), (256, 1747, "uniform"), (256, 1747, "max"), (512, 250, "uniform"),
    (512, 257, "identity"), (1024, 512, "uniform"), (1024, 868, "alternating"),
    (2048, 129, "uniform"), (2048, 129, "max"), (4096, 256, "uniform"), (4096, 256, "max"),
    (4096, 256, "sparse"),
]


def main():
    manifest = []
    for i, (N, W, pattern) in enumerate(CASES):
        seed = 1000 + i
        q, a, b = workload.case(N, W, pattern, seed)
        c, _ = oracle.ref_polymul(N, W, q, a, b)
        plan = oracle.ref_plan(N, q)
        name = f"{i:03d}_N{N}_W{W}_{pattern}.npz"
        np.savez_compressed(os.path.join(HERE, name), q=q, a=a, b=b, c=c,
                            primes=plan["primes"], K=np.array(plan["K"]))
        manifest.append(dict(file=name, N=N, W=W, L=int(q.shape[0]), pattern=pattern, seed=seed,
                             K=int(plan["K"])))
        print(name, "K =", plan["K"])
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(dict(generator="reference solve_cpu.cpp via oracle/ref_shim.cpp",
                       seeds="numpy PCG64(seed); q then operands (polymul.workload.case)",
                       cases=manifest), f, indent=1)


if __name__ == "__main__":
    main()
