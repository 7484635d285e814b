"""GPU tests of the continuous-batching server: every result converges to
true residual 1e-10 (checked by the oracle in FP64), requests that arrive while
others run are served, a result is bitwise the same alone and in the mix,
cancellation and budget rejection work."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def make(hw, ctx, oracle, dims, seed):
    U = oracle.gen_links(dims, 0.3, seed)
    lat = hw.Lattice(ctx, dims, True)
    return U, lat, hw.GaugeField(lat, U)


@pytest.mark.parametrize("precision", ["f16", "f32"])
def test_server_mix_and_determinism(hw, ctx, oracle, precision):
    specs = [((8, 8, 8, 8), 61), ((4, 4, 4, 8), 62), ((6, 4, 4, 4), 63)]
    gauges = [make(hw, ctx, oracle, d, s) for d, s in specs]
    srv = hw.Server(ctx, precision=precision, chunk_iters=4)
    try:
        _mix_and_determinism(hw, oracle, srv, specs, gauges)
    finally:
        srv.close()


def _mix_and_determinism(hw, oracle, srv, specs, gauges):
    gids = [srv.add_gauge(G) for (_, _, G) in gauges]
    rng = np.random.default_rng(5)
    reqs = []
    for n in range(12):
        g = n % 3
        dims = specs[g][0]
        nrhs = int(rng.integers(1, 5))
        kappa = float(rng.uniform(0.115, 0.124))
        srcs = [oracle.gen_spinor(dims, 7000 + 10 * n + k, oracle.EVEN) for k in range(nrhs)]
        reqs.append((g, kappa, srcs))
    # request 0 alone first
    g0, k0, s0 = reqs[0]
    rid = srv.submit(gids[g0], k0, s0, TOL)
    alone, r_alone = srv.wait(rid, len(s0), gauges[g0][1].volume)
    assert r_alone.converged
    # then everything, submitted from a thread while earlier ones run
    ids = [None] * len(reqs)

    def submitter():
        for n, (g, kappa, srcs) in enumerate(reqs):
            ids[n] = srv.submit(gids[g], kappa, srcs, TOL)
            time.sleep(0.002)

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    for n, (g, kappa, srcs) in enumerate(reqs):
        sols, res = srv.wait(ids[n], len(srcs), gauges[g][1].volume)
        assert res.converged, res
        U = gauges[g][0]
        for b, x in zip(srcs, sols):
            assert oracle.true_residual(specs[g][0], U, kappa, b, x) <= TOL
        if n == 0:
            for a, b in zip(alone, sols):
                assert np.array_equal(a, b)  # same alone and in the mix
    st = srv.stats()
    assert st["completed"] == 13 and st["bytes_in_use"] == 0


def test_server_cancel_and_reject(hw, ctx, oracle):
    dims = (8, 8, 8, 8)
    U, lat, G = make(hw, ctx, oracle, dims, 71)
    # one source of an 8^4 lattice needs about 2.2 MB of solve memory: 16 exceed 16 MiB
    srv = hw.Server(ctx, precision="f16", hbm_budget_bytes=16 << 20, chunk_iters=2)
    try:
        _cancel_and_reject(hw, oracle, srv, dims, U, lat, G)
    finally:
        srv.close()


def _cancel_and_reject(hw, oracle, srv, dims, U, lat, G):
    gid = srv.add_gauge(G)
    b = oracle.gen_spinor(dims, 72, oracle.EVEN)
    rid = srv.submit(gid, 0.12, [b] * 16, TOL)
    _, res = srv.wait(rid, 16, lat.volume)
    assert res.status == hw.HW_ERR_REJECTED
    # a request cancelled while queued or running ends as cancelled (or done, if it won the race)
    rid = srv.submit(gid, 0.12, [b], TOL, maxiters=100000)
    srv.cancel(rid)
    _, res = srv.wait(rid, 1, lat.volume)
    assert res.status in (hw.HW_ERR_CANCELLED, hw.HW_OK)
    # the server keeps serving afterwards
    rid = srv.submit(gid, 0.12, [b], TOL)
    sols, res = srv.wait(rid, 1, lat.volume)
    assert res.converged and oracle.true_residual(dims, U, 0.12, b, sols[0]) <= TOL
    st = srv.stats()
    assert st["rejected"] == 1
