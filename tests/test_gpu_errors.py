"""Device-path errors: a kernel pipeline wait that runs out is reported, and
the context stays usable afterwards.

Every wait inside the tensor-core pipelines is bounded (DevPoint::wait_ns).
The test shortens the limit to 2 ms and uses the library's stall hook
(fpm_debug_inject_stall): the decompose or CRT pipeline then never requests
one of its shared-memory copies, so the wait for it runs out, the kernel sets
the error word and returns.  No GPU fault is involved.  The error must reach
the caller through fpm_get_error (device path), as FPM_ETIMEOUT from fpm_run
(host path), and through fpm_noalloc_get_error (static-scratch path); the next
product without the hook must be bit-exact against the oracle.
"""
import numpy as np
import pytest

import oracle
import polymul
from polymul import workload as wl

pytestmark = pytest.mark.gpu

LIMIT_NS = 2_000_000   # 2 ms


def _dev(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to("cuda")


@pytest.fixture(scope="module")
def point():
    N, W = 4096, 256
    q, a, b = wl.case(N, W, "uniform", seed=77)
    return N, W, q, a, b, oracle.OraclePlan(N, q).polymul(a, b)


@pytest.mark.parametrize("mask", [polymul.STALL_DECOMPOSE, polymul.STALL_CRT])
def test_device_path_reports_timeout(cuda, point, mask):
    torch = cuda
    N, W, q, a, b, expect = point
    with polymul.Context(N, W, q) as ctx:
        da, db = _dev(torch, a), _dev(torch, b)
        dc = torch.zeros_like(da)
        stream = torch.cuda.current_stream().cuda_stream
        assert ctx.get_error(stream) == polymul.FPM_OK
        ctx.set_wait_limit(LIMIT_NS)
        ctx.inject_stall(mask)
        ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream)   # enqueues fine
        assert ctx.get_error(stream) == polymul.FPM_ETIMEOUT
        assert "ran out of time" in polymul.load().fpm_last_error().decode()
        assert ctx.get_error(stream) == polymul.FPM_OK                         # read and cleared
        ctx.inject_stall(0)
        ctx.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream)
        assert ctx.get_error(stream) == polymul.FPM_OK
        got = dc.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, expect)


@pytest.mark.parametrize("mask", [polymul.STALL_DECOMPOSE, polymul.STALL_CRT])
def test_host_path_raises_timeout(cuda, point, mask):
    N, W, q, a, b, expect = point
    with polymul.Context(N, W, q) as ctx:
        ctx.set_wait_limit(LIMIT_NS)
        ctx.inject_stall(mask)
        with pytest.raises(polymul.FpmError) as err:
            ctx.run(a, b)
        assert err.value.code == polymul.FPM_ETIMEOUT
        ctx.inject_stall(0)
        assert np.array_equal(ctx.run(a, b), expect)


def test_noalloc_path_reports_timeout(cuda, point):
    torch = cuda
    N, W, q, a, b, expect = point
    lib = polymul.load()
    with polymul.Context(N, W, q) as ctx:
        da, db = _dev(torch, a), _dev(torch, b)
        dc = torch.zeros_like(da)
        stream = torch.cuda.current_stream().cuda_stream
        assert lib.fpm_noalloc_get_error(stream) == polymul.FPM_OK
        ctx.set_wait_limit(LIMIT_NS)
        ctx.inject_stall(polymul.STALL_CRT)
        assert lib.fpm_run_device_noalloc(ctx.handle, da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream) == 0
        assert lib.fpm_noalloc_get_error(stream) == polymul.FPM_ETIMEOUT
        assert ctx.get_error(stream) == polymul.FPM_OK      # the context's own word is untouched
        ctx.inject_stall(0)
        assert lib.fpm_run_device_noalloc(ctx.handle, da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream) == 0
        assert lib.fpm_noalloc_get_error(stream) == polymul.FPM_OK
        assert np.array_equal(dc.cpu().numpy().view(np.uint32), expect)
