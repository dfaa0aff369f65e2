"""fpm_run_device_noalloc: the product with its scratch in a static device array.

Callers that cannot allocate device memory once they are running (a process
held to a fixed device-memory budget, or one issuing work where cudaMalloc is
not allowed) use this entry point: its residue workspaces and error word live
in one static 80 MiB device array, so the call allocates nothing.  These tests
call it through the C ABI and check it bit-exact (the tolerance of every
integer test here) against fpm_run_device on the same operands, on two calls
in a row, so the second call also shows that what the first left in the shared
array does not leak into its result, and that the array's error word stays
clear.  The cases cover the tensor-core pipelines (two or more limbs) and the
one-limb CRT on the CUDA cores.  The file is named to be collected last:
it passes alone in a fresh process, where its first call is the one that looks
up the array's address, and after every other test.
"""
import ctypes

import numpy as np
import pytest

import polymul
from polymul import workload as wl

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 80 << 20


def noalloc_fn():
    lib = polymul.load()
    fn = lib.fpm_run_device_noalloc
    vp = ctypes.c_void_p
    fn.argtypes = [vp, vp, vp, vp, vp]
    fn.restype = ctypes.c_int
    return lib, fn


@pytest.mark.parametrize("N,W,pattern", [(4096, 256, "uniform"), (65536, 2048, "max"), (2048, 1747, "uniform"),
                                         (4096, 32, "uniform")])
def test_noalloc_matches_run_device_twice(cuda, N, W, pattern):
    torch = cuda
    lib, run_noalloc = noalloc_fn()
    q, a1, b1 = wl.case(N, W, pattern, seed=N + 1)
    a2, b2 = wl.operands(q, N, "uniform", np.random.default_rng(N + 2))

    def dev(x):
        return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to("cuda")

    with polymul.Context(N, W, q) as ctx:
        assert 2 * ctx.K * N * 4 + 256 <= SCRATCH_BYTES
        pairs = [(dev(a1), dev(b1)), (dev(a2), dev(b2))]
        stream = torch.cuda.current_stream().cuda_stream
        expect = []
        for da, db in pairs:
            dc = torch.empty_like(da)
            ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream)
            expect.append(dc)
        got = []
        for da, db in pairs:                      # two calls in a row
            dc = torch.full_like(da, -1)
            rc = run_noalloc(ctx.handle, da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream)
            assert rc == polymul.FPM_OK, lib.fpm_last_error().decode()
            got.append(dc)
        assert lib.fpm_noalloc_get_error(stream) == polymul.FPM_OK
        torch.cuda.synchronize()
        for e, g in zip(expect, got):
            assert torch.equal(e, g)


def test_noalloc_refuses_point_beyond_scratch(cuda):
    torch = cuda
    lib, run_noalloc = noalloc_fn()
    N, W = 131072, 2048
    q, a, b = wl.case(N, W, "uniform", seed=5)
    with polymul.Context(N, W, q) as ctx:
        assert 2 * ctx.K * N * 4 > SCRATCH_BYTES
        da = torch.from_numpy(a.view(np.int32)).to("cuda")
        db = torch.from_numpy(b.view(np.int32)).to("cuda")
        dc = torch.zeros_like(da)
        rc = run_noalloc(ctx.handle, da.data_ptr(), db.data_ptr(), dc.data_ptr(), None)
        assert rc == polymul.FPM_EINVAL
        msg = lib.fpm_last_error().decode()
        assert "static scratch" in msg and str(SCRATCH_BYTES) in msg
        torch.cuda.synchronize()
        assert not dc.any()
