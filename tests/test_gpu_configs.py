"""The full-size benchmark configurations of the mixed-precision and batched solves,
checked by size-independent properties: every solve's true residual |b - M x| / |b|
recomputed by the CPU oracle in FP64 (<= 1e-10), agreement with the plain FP64 CG,
and bitwise batch invariance (a solve alone and in the mix)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def test_mixed_48x96(hw, ctx, oracle):
    """48^3 x 96, links exp(i 0.25 H), kappa 0.124, one Gaussian source: the FP32 and
    the FP16-with-norm inner solvers (FP64 reliable updates and solution accumulation)
    against the plain FP64 CG on the same GPU."""
    dims, kappa = (48, 48, 48, 96), 0.124
    U = hw.generate_links(dims, 0.25, 300)
    b = hw.generate_spinor(dims, 301, hw.EVEN)
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, U, 12)
    D = hw.Dirac_Wilson_evenodd(kappa, G)
    fb, fx64 = hw.Field(lat, b), hw.Field(lat)
    t0 = time.perf_counter()
    r64 = D.solve(fb, fx64, accuracy=TOL)
    t64 = time.perf_counter() - t0
    assert r64.converged, r64
    x64 = fx64.download()
    fx64.close()
    assert oracle.true_residual(dims, U, kappa, b, x64) <= TOL
    for precision, delta in (("f32", 1e-5), ("f16", 0.005)):
        fx = hw.Field(lat)
        t0 = time.perf_counter()
        r = D.solve(fb, fx, accuracy=TOL, precision=precision, delta=delta)
        t = time.perf_counter() - t0
        assert r.converged, (precision, r)
        x = fx.download()
        fx.close()
        tr = oracle.true_residual(dims, U, kappa, b, x)
        assert tr <= TOL, (precision, tr)
        # mixed precision with reliable updates needs about as many iterations as FP64
        assert r.iterations <= r64.iterations + 10, (precision, r.iterations, r64.iterations)
        assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-8
        print(f"48^3x96 {precision}: {r.iterations} iterations ({r.reliable_updates} reliable updates) "
              f"{t:.3f} s; FP64 {r64.iterations} iterations {t64:.3f} s")


def test_batch_16_uneven_lattices(hw, ctx, oracle):
    """16 gauge fields (eps 0.3) cycling through 8^4, 12^4, 16^4 and 16^3 x 32, each with
    1-12 Gaussian sources and kappa uniform in [0.115, 0.124], solved in one batch to 1e-10
    (more right-hand sides than engine slots: later ones join as slots free up)."""
    rng = np.random.default_rng(7)
    shapes = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (16, 16, 16, 32)]
    reqs, checks, keep = [], [], []
    for n in range(16):
        dims = shapes[n % 4]
        U = hw.generate_links(dims, 0.3, 400 + n)
        lat = hw.Lattice(ctx, dims, True)
        G = hw.GaugeField(lat, U, 18)
        keep += [lat, G]
        nrhs = int(rng.integers(1, 13))
        for k in range(nrhs):
            kappa = float(rng.uniform(0.115, 0.124))
            b = hw.generate_spinor(dims, 10000 * n + k, hw.EVEN)
            D = hw.Dirac_Wilson_evenodd(kappa, G)
            fb, fx = hw.Field(lat, b), hw.Field(lat)
            reqs.append((D, fb, fx, TOL))
            checks.append((dims, U, kappa, b, fx))
    assert len(reqs) > 64
    results = hw.batch_solve(ctx, reqs, precision="f16", delta=0.005)
    for (dims, U, kappa, b, fx), r in zip(checks, results):
        assert r.converged, r
        assert oracle.true_residual(dims, U, kappa, b, fx.download()) <= TOL
    # one solve of the mix, alone: bitwise the same solution
    j = len(reqs) // 2
    D, fb, fx, _ = reqs[j]
    fx2 = hw.Field(D.gauge.lattice)
    r2 = hw.batch_solve(ctx, [(D, fb, fx2, TOL)], precision="f16", delta=0.005)[0]
    assert r2.iterations == results[j].iterations
    assert np.array_equal(fx2.download(), fx.download())
