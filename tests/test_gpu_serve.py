"""Serving loop (fpm_server): requests admitted by device footprint, batched as
they arrive, run on concurrent lanes.  Each result must be exactly the product
the plain entry point gives for the same request alone, whatever else was in
flight with it.
"""
import numpy as np
import pytest

import polymul
from polymul import workload as wl

pytestmark = pytest.mark.gpu

# A catalog of resident points: the mix's N and W corners plus a few between.
CATALOG = [(4096, 128), (4096, 2048), (8192, 512), (16384, 868), (32768, 1747), (65536, 2048), (2048, 256)]


@pytest.fixture(scope="module")
def catalog(cuda):
    ctxs, qs = [], []
    for i, (N, W) in enumerate(CATALOG):
        q = wl.case(N, W, "uniform", seed=5100 + i)[0]
        ctxs.append(polymul.Context(N, W, q))
        qs.append(q)
    yield ctxs, qs
    for c in ctxs:
        c.close()


def requests(ctxs, qs, n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = rng.integers(0, len(ctxs), size=n)
    a_list, b_list, c_list = [], [], []
    for p in pts:
        a, b = wl.operands(qs[p], ctxs[p].N, "uniform", rng)
        a_list.append(a)
        b_list.append(b)
        c_list.append(np.full_like(a, 0xFFFFFFFF))
    return pts, a_list, b_list, c_list


def check_alone(ctxs, pts, a_list, b_list, c_list):
    for p, a, b, c in zip(pts, a_list, b_list, c_list):
        assert np.array_equal(c, ctxs[p].run(a, b))


def test_serve_burst_batches_and_overlaps(catalog):
    """Every request arrives at once: the queue forms, lanes take micro-batches
    and run concurrently; each result equals the same product alone."""
    ctxs, qs = catalog
    pts, a_list, b_list, c_list = requests(ctxs, qs, 120, seed=1)
    with polymul.Server(ctxs, budget_bytes=4 << 30, lanes=4, max_batch=16) as srv:
        lat = srv.replay(pts, np.zeros(len(pts)), a_list, b_list, c_list)
        st = srv.stats
        assert st.completed == len(pts) and st.failed == 0
        assert st.batches < len(pts)          # requests were batched
        assert st.max_lanes_busy >= 2         # micro-batches overlapped on the device
        assert st.peak_bytes <= st.budget_bytes
        assert (lat > 0).all()
    check_alone(ctxs, pts, a_list, b_list, c_list)


def test_serve_poisson_stream(catalog):
    ctxs, qs = catalog
    pts, a_list, b_list, c_list = requests(ctxs, qs, 300, seed=2)
    arrivals = wl.poisson_arrivals(len(pts), 4000.0, seed=3)
    with polymul.Server(ctxs, budget_bytes=2 << 30, lanes=3, max_batch=8) as srv:
        lat = srv.replay(pts, arrivals, a_list, b_list, c_list)
        assert srv.stats.completed == len(pts)
        assert np.percentile(lat, 99) >= np.percentile(lat, 50) > 0
    check_alone(ctxs, pts, a_list, b_list, c_list)


def test_serve_admission_by_footprint(catalog):
    """A budget that holds one request on the largest point (and little else):
    requests queue for memory, the arena never overflows, results are exact."""
    ctxs, qs = catalog
    big = CATALOG.index((65536, 2048))
    with polymul.Server(ctxs, budget_bytes=1 << 30, lanes=2, max_batch=4) as probe:
        need = probe.footprint(big)
    pts, a_list, b_list, c_list = requests(ctxs, qs, 40, seed=4)
    pts[:8] = big
    for i in range(8):
        a_list[i], b_list[i] = wl.operands(qs[big], ctxs[big].N, "max", np.random.default_rng(i))
        c_list[i] = np.zeros_like(a_list[i])
    with polymul.Server(ctxs, budget_bytes=need + (1 << 20), lanes=4, max_batch=4) as srv:
        srv.replay(pts, np.zeros(len(pts)), a_list, b_list, c_list)
        st = srv.stats
        assert st.completed == len(pts)
        assert st.peak_bytes <= need + (1 << 20)
    check_alone(ctxs, pts, a_list, b_list, c_list)


def test_serve_submit_wait_and_refusal(catalog):
    ctxs, qs = catalog
    small = CATALOG.index((4096, 128))
    big = CATALOG.index((65536, 2048))
    with polymul.Server(ctxs, budget_bytes=64 << 20, lanes=1, max_batch=1) as srv:
        assert srv.footprint(big) > 64 << 20
        a, b = wl.operands(qs[big], ctxs[big].N, "uniform", np.random.default_rng(9))
        with pytest.raises(polymul.FpmError) as e:
            srv.submit(big, a, b, np.zeros_like(a))
        assert e.value.code == polymul.FPM_EINVAL and "budget" in str(e.value)
        out = []
        for i in range(5):
            a, b = wl.operands(qs[small], ctxs[small].N, "uniform", np.random.default_rng(i))
            c = np.zeros_like(a)
            out.append((srv.submit(small, a, b, c), a, b, c))
        for t, a, b, c in out:
            assert srv.wait(t) > 0
            assert np.array_equal(c, ctxs[small].run(a, b))
