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


def test_server_continuous_batching_fields(hw, ctx, oracle):
    """Continuous batching, not a queue: request A (a 12^4 lattice, 4 sources, 2 iterations per
    chunk) is admitted first; request B (another lattice) is submitted once A is running and is
    admitted while A is still iterating (B's admission chunk lies inside A's [admit, retire)
    interval).  Both are served from device fields (hw_server_submit_fields, no copies), both
    converge to true residual 1e-10 by the oracle, and B's solution is bitwise the one B gets
    when it is served alone."""
    specs = [((12, 12, 12, 12), 81, 0.124, 4), ((8, 8, 8, 8), 82, 0.12, 2)]
    built = []
    for dims, seed, kappa, nsrc in specs:
        U, lat, G = make(hw, ctx, oracle, dims, seed)
        srcs = [oracle.gen_spinor(dims, 800 + 10 * seed + k, oracle.EVEN) for k in range(nsrc)]
        built.append((dims, U, lat, G, kappa, srcs))
    srv = hw.Server(ctx, precision="f16", chunk_iters=2)
    try:
        gids = [srv.add_gauge(b[3]) for b in built]
        fields = []
        for dims, U, lat, G, kappa, srcs in built:
            fields.append(([hw.Field(lat, s_) for s_ in srcs], [hw.Field(lat) for _ in srcs]))
        ida = srv.submit_fields(gids[0], built[0][4], fields[0][0], fields[0][1], TOL)
        t0 = time.time()
        while srv.stats()["chunks"] < 3 and time.time() - t0 < 60:
            time.sleep(0.001)
        idb = srv.submit_fields(gids[1], built[1][4], fields[1][0], fields[1][1], TOL)
        _, ra = srv.wait(ida, 4, built[0][2].volume, copy=False)
        _, rb = srv.wait(idb, 2, built[1][2].volume, copy=False)
        assert ra.converged and rb.converged, (ra, rb)
        assert ra.admit_chunk < rb.admit_chunk < ra.retire_chunk, (ra, rb)
        for (dims, U, lat, G, kappa, srcs), (fb, fx) in zip(built, fields):
            for b, f in zip(srcs, fx):
                assert oracle.true_residual(dims, U, kappa, b, f.download()) <= TOL
        # B alone
        dims, U, lat, G, kappa, srcs = built[1]
        fb, fx = [hw.Field(lat, s_) for s_ in srcs], [hw.Field(lat) for _ in srcs]
        idb2 = srv.submit_fields(gids[1], kappa, fb, fx, TOL)
        _, rb2 = srv.wait(idb2, 2, lat.volume, copy=False)
        assert rb2.iterations == rb.iterations
        for a, b in zip(fx, fields[1][1]):
            assert np.array_equal(a.download(), b.download())
    finally:
        srv.close()


def test_server_even_first_host_arrays(hw, ctx, oracle):
    """hw_server_submit_eo: host arrays in HILA's even-first site order, page-locked (copied by
    DMA directly) and pageable (staged), give bitwise the solutions of the lexicographic
    hw_server_submit path; the ODD half of a solution array is left untouched."""
    dims, kappa = (8, 8, 8, 8), 0.12
    U, lat, G = make(hw, ctx, oracle, dims, 91)
    V = lat.volume
    order = hw.eo_order(dims)
    srcs = [oracle.gen_spinor(dims, 910 + k, oracle.EVEN) for k in range(3)]
    srv = hw.Server(ctx, precision="f16", chunk_iters=4)
    pins = []
    try:
        gid = srv.add_gauge(G)
        rid = srv.submit(gid, kappa, srcs, TOL)
        lex, rl = srv.wait(rid, 3, V)
        assert rl.converged
        # sources 0, 1 page-locked, source 2 pageable; solution 1 pageable
        src_eo, sol_eo = [], []
        for k, s_ in enumerate(srcs):
            if k < 2:
                pa = hw.PinnedArray((V, 4, 3, 2))
                pins.append(pa)
                pa.array[:] = s_[order]
                src_eo.append(pa.array)
            else:
                src_eo.append(np.ascontiguousarray(s_[order]))
            if k != 1:
                pa = hw.PinnedArray((V, 4, 3, 2))
                pins.append(pa)
                pa.array[:] = 7.0
                sol_eo.append(pa.array)
            else:
                sol_eo.append(np.full((V, 4, 3, 2), 7.0))
        rid = srv.submit_eo(gid, kappa, src_eo, sol_eo, TOL)
        _, re_ = srv.wait(rid, 3, V, copy=False)
        assert re_.converged and re_.iterations == rl.iterations
        for x_lex, x_eo in zip(lex, sol_eo):
            assert np.array_equal(x_eo[:V // 2], x_lex[order[:V // 2]])
            assert np.all(x_eo[V // 2:] == 7.0)
    finally:
        srv.close()
        for pa in pins:
            pa.free()


def test_field_even_first_transfers(hw, ctx, oracle):
    """hw_field_upload_eo / download_eo move one parity of an even-first host array and agree
    with the lexicographic transfers."""
    dims = (4, 6, 4, 8)
    lat = hw.Lattice(ctx, dims, True)
    psi = oracle.gen_spinor(dims, 5, oracle.ALL)
    order = hw.eo_order(dims)
    eo = np.ascontiguousarray(psi[order])
    for par, mask in ((hw.EVEN, 0), (hw.ODD, 1), (hw.ALL, None)):
        f = hw.Field(lat)
        f.upload_eo(eo, par)
        got = f.download()
        want = psi.copy()
        if mask is not None:
            want[oracle.parity_mask(dims) != mask] = 0
        assert np.array_equal(got, want), par
        out = np.full_like(eo, 3.0)
        f.download_eo(par, out)
        half = lat.volume // 2
        if par == hw.EVEN:
            assert np.array_equal(out[:half], eo[:half]) and np.all(out[half:] == 3.0)
        elif par == hw.ODD:
            assert np.array_equal(out[half:], eo[half:]) and np.all(out[:half] == 3.0)
        else:
            assert np.array_equal(out, eo)
        f.close()
    lat.close()
