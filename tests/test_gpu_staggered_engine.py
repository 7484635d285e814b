"""Staggered solves on the shared batched engine and through the server (GPU).

dirac_staggered_evenodd (staggered.h:193-279) runs on the same engine as the Wilson
solves: the same slot tables, phase sequence, reliable-update state machine,
per-(slot, tile) reductions and chunk graphs, with FP64 staggered phase kernels.
Every solve is judged by its true residual recomputed by the CPU oracle in FP64
(<= 1e-10); a solve is bitwise the same alone and in any batch, also beside Wilson
solves in the same server."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _c(a):
    return a[..., 0] + 1j * a[..., 1]


def residual(oracle, dims, U, mass, b, x, normal=False):
    ev = oracle.parity_mask(dims) == 0
    mx = oracle.staggered_eo_apply(dims, U, mass, x, 1)
    if normal:
        mx = oracle.staggered_eo_apply(dims, U, mass, mx, -1)
    return np.linalg.norm(_c(b)[ev] - _c(mx)[ev]) / np.linalg.norm(_c(b)[ev])


def build(hw, ctx, oracle, specs):
    out = []
    for n, (dims, seed, mass, nsrc, link_format) in enumerate(specs):
        U = oracle.gen_links(dims, 0.3, seed)
        lat = hw.Lattice(ctx, dims, True)
        G = hw.GaugeField(lat, U, link_format)
        D = hw.dirac_staggered_evenodd(mass, G)
        srcs = [oracle.gen_colour_vector(dims, 3000 + 10 * n + k, oracle.EVEN) for k in range(nsrc)]
        out.append((dims, U, lat, G, D, mass, srcs))
    return out


SPECS = [((8, 8, 8, 8), 301, 5.0, 2, 18), ((4, 4, 4, 8), 302, 4.5, 1, 18), ((2, 4, 6, 8), 303, 6.0, 2, 12)]


def test_staggered_batch(hw, ctx, oracle):
    """Uneven lattices and masses, both link formats, one nonzero initial guess: every solve
    converges by the oracle's true residual and is bitwise the same alone."""
    built = build(hw, ctx, oracle, SPECS)
    work = []
    for n, (dims, U, lat, G, D, mass, srcs) in enumerate(built):
        for k, b in enumerate(srcs):
            guess = oracle.gen_colour_vector(dims, 4000 + n, oracle.EVEN) if (n, k) == (0, 1) else None
            fx = hw.StaggeredField(lat, guess) if guess is not None else hw.StaggeredField(lat)
            work.append((dims, U, lat, D, mass, b, guess, hw.StaggeredField(lat, b), fx))
    res = hw.staggered_batch_solve(ctx, [(D, fb, fx, TOL) for (_, _, _, D, _, _, _, fb, fx) in work])
    for (dims, U, lat, D, mass, b, guess, fb, fx), r in zip(work, res):
        assert r.converged, r
        x = fx.download()
        assert residual(oracle, dims, U, mass, b, x) <= TOL
        assert abs(r.true_residual - residual(oracle, dims, U, mass, b, x)) <= 1e-3 * TOL
        alone = hw.StaggeredField(lat, guess) if guess is not None else hw.StaggeredField(lat)
        [ra] = hw.staggered_batch_solve(ctx, [(D, fb, alone, TOL)])
        assert ra.iterations == r.iterations
        assert np.array_equal(alone.download(), x)


def test_staggered_batch_normal_equations(hw, ctx, oracle):
    """CG<dirac_staggered_evenodd>::apply semantics (M^dag M out = in) on the engine, against the
    oracle's recomputed normal-equation residual and the standalone FP64 CG."""
    [(dims, U, lat, G, D, mass, srcs)] = build(hw, ctx, oracle, [((8, 8, 8, 8), 311, 5.0, 1, 18)])
    fb, fx = hw.StaggeredField(lat, srcs[0]), hw.StaggeredField(lat)
    [r] = hw.staggered_batch_solve(ctx, [(D, fb, fx, TOL, 10000, True)])
    assert r.converged, r
    x = fx.download()
    assert residual(oracle, dims, U, mass, srcs[0], x, normal=True) <= TOL
    fy = hw.StaggeredField(lat)
    r2 = D.cg(fb, fy, accuracy=1e-12, true_residual=True)
    assert r2.converged
    y = fy.download()
    ev = oracle.parity_mask(dims) == 0
    assert np.linalg.norm(_c(x)[ev] - _c(y)[ev]) / np.linalg.norm(_c(y)[ev]) <= 1e-9


def test_staggered_and_wilson_in_one_server(hw, ctx, oracle):
    """Staggered and Wilson requests served together by one server: both converge, and the
    staggered solutions are bitwise those of a staggered-only batch."""
    [(dims, U, lat, G, D, mass, srcs)] = build(hw, ctx, oracle, [((8, 8, 8, 8), 321, 5.0, 2, 18)])
    Uw = oracle.gen_links((8, 8, 8, 8), 0.3, 322)
    latw = hw.Lattice(ctx, (8, 8, 8, 8), True)
    Gw = hw.GaugeField(latw, Uw)
    bw = [oracle.gen_spinor((8, 8, 8, 8), 323 + k, oracle.EVEN) for k in range(3)]
    srv = hw.Server(ctx, precision="f16", chunk_iters=2)
    try:
        gw, gs = srv.add_gauge(Gw), srv.add_gauge(G)
        fwb, fwx = [hw.Field(latw, b) for b in bw], [hw.Field(latw) for _ in bw]
        fsb, fsx = [hw.StaggeredField(lat, b) for b in srcs], [hw.StaggeredField(lat) for _ in srcs]
        idw = srv.submit_fields(gw, 0.124, fwb, fwx, TOL)
        ids = srv.submit_staggered(gs, mass, fsb, fsx, TOL)
        _, rw = srv.wait(idw, 3, latw.volume, copy=False)
        _, rs = srv.wait(ids, 2, lat.volume, copy=False)
        assert rw.converged and rs.converged, (rw, rs)
        for b, f in zip(bw, fwx):
            assert oracle.true_residual((8, 8, 8, 8), Uw, 0.124, b, f.download()) <= TOL
        for b, f in zip(srcs, fsx):
            assert residual(oracle, dims, U, mass, b, f.download()) <= TOL
        # the staggered request alone, through the batch entry point
        alone = [hw.StaggeredField(lat) for _ in srcs]
        res = hw.staggered_batch_solve(ctx, [(D, fb, fa, TOL) for fb, fa in zip(fsb, alone)])
        assert all(r.converged for r in res)
        for a, f in zip(alone, fsx):
            assert np.array_equal(a.download(), f.download())
    finally:
        srv.close()


def test_staggered_batch_mixed_precision(hw, ctx, oracle):
    """FP16 inner iterations with FP64 reliable updates (precision "f16"): masses from just
    above the spectral radius of the hop (|D| is about 2.25 for these links, so at m = 2.4
    M = m - D^dag D / m stays positive with a condition number near 8) to heavy, both link
    formats, both systems; every solve reaches the oracle's FP64 true residual, the lightest
    takes several reliable updates, and a solve is bitwise the same alone as in the batch."""
    built = build(hw, ctx, oracle, [((8, 8, 8, 8), 331, 2.4, 3, 18), ((4, 4, 4, 8), 332, 4.5, 1, 12),
                                     ((2, 4, 6, 8), 333, 6.0, 1, 18)])
    work = []
    for n, (dims, U, lat, G, D, mass, srcs) in enumerate(built):
        for k, b in enumerate(srcs):
            normal = (n, k) == (0, 2)
            work.append((dims, U, lat, D, mass, b, normal, hw.StaggeredField(lat, b), hw.StaggeredField(lat)))
    reqs = [(D, fb, fx, TOL, 10000, normal) for (_, _, _, D, _, _, normal, fb, fx) in work]
    res = hw.staggered_batch_solve(ctx, reqs, precision="f16")
    for (dims, U, lat, D, mass, b, normal, fb, fx), r in zip(work, res):
        assert r.converged, r
        x = fx.download()
        assert residual(oracle, dims, U, mass, b, x, normal=normal) <= TOL
        if mass < 3:
            assert r.reliable_updates >= 2, r
        alone = hw.StaggeredField(lat)
        [ra] = hw.staggered_batch_solve(ctx, [(D, fb, alone, TOL, 10000, normal)], precision="f16")
        assert ra.iterations == r.iterations
        assert np.array_equal(alone.download(), x)
    # the same light-mass system in FP64 on the engine: the same solution to the tolerance
    (dims, U, lat, D, mass, b, normal, fb, fx) = work[0]
    f64 = hw.StaggeredField(lat)
    [r64] = hw.staggered_batch_solve(ctx, [(D, fb, f64, TOL)])
    assert r64.converged
    ev = oracle.parity_mask(dims) == 0
    x, y = fx.download(), f64.download()
    assert np.linalg.norm(_c(x)[ev] - _c(y)[ev]) / np.linalg.norm(_c(y)[ev]) <= 1e-6


def test_staggered_mixed_precision_served(hw, ctx, oracle):
    """A server with staggered_precision "f16" serves staggered requests with FP16 inner
    iterations beside Wilson requests; the results reach the oracle's true residual and are
    bitwise those of the FP16 staggered batch entry point (factor 0.05 in both)."""
    [(dims, U, lat, G, D, mass, srcs)] = build(hw, ctx, oracle, [((8, 8, 8, 8), 341, 2.4, 2, 18)])
    Uw = oracle.gen_links((8, 8, 8, 8), 0.3, 342)
    latw = hw.Lattice(ctx, (8, 8, 8, 8), True)
    Gw = hw.GaugeField(latw, Uw)
    bw = [oracle.gen_spinor((8, 8, 8, 8), 343, oracle.EVEN)]
    srv = hw.Server(ctx, precision="f16", chunk_iters=4, staggered_precision="f16")
    try:
        gw, gs = srv.add_gauge(Gw), srv.add_gauge(G)
        fwb, fwx = [hw.Field(latw, b) for b in bw], [hw.Field(latw) for _ in bw]
        fsb, fsx = [hw.StaggeredField(lat, b) for b in srcs], [hw.StaggeredField(lat) for _ in srcs]
        ids = srv.submit_staggered(gs, mass, fsb, fsx, TOL)
        idw = srv.submit_fields(gw, 0.124, fwb, fwx, TOL)
        _, rs = srv.wait(ids, 2, lat.volume, copy=False)
        _, rw = srv.wait(idw, 1, latw.volume, copy=False)
        assert rw.converged and rs.converged, (rw, rs)
        assert rs.reliable_updates >= 2, rs
        for b, f in zip(srcs, fsx):
            assert residual(oracle, dims, U, mass, b, f.download()) <= TOL
        alone = [hw.StaggeredField(lat) for _ in srcs]
        res = hw.staggered_batch_solve(ctx, [(D, fb, fa, TOL) for fb, fa in zip(fsb, alone)], precision="f16")
        assert all(r.converged for r in res)
        for a, f in zip(alone, fsx):
            assert np.array_equal(a.download(), f.download())
    finally:
        srv.close()
