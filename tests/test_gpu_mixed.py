"""GPU tests of the mixed-precision solves and of the batched engine.

Every solve is checked by its true residual |b - M x| / |b| recomputed by the
CPU oracle in FP64: <= 1e-10.  Batched solves must give bitwise the same
solution alone and inside a batch.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def make(hw, ctx, oracle, dims, seed, link_format=18):
    U = oracle.gen_links(dims, 0.3, seed)
    lat = hw.Lattice(ctx, dims, True)
    return U, lat, hw.GaugeField(lat, U, link_format)


@pytest.mark.parametrize("precision", ["f32", "f16"])
@pytest.mark.parametrize("dims,kappa,link_format", [((8, 8, 8, 8), 0.12, 18), ((16, 8, 8, 16), 0.124, 12),
                                                    ((2, 4, 6, 8), 0.115, 18)])
def test_mixed_solve(hw, ctx, oracle, precision, dims, kappa, link_format):
    U, lat, G = make(hw, ctx, oracle, dims, 11, link_format)
    b = oracle.gen_spinor(dims, 12, oracle.EVEN)
    D = hw.Dirac_Wilson_evenodd(kappa, G)
    fb, fx = hw.Field(lat, b), hw.Field(lat)
    res = D.solve(fb, fx, accuracy=TOL, precision=precision)
    assert res.converged, res
    assert res.reliable_updates >= 2
    x = fx.download()
    tr = oracle.true_residual(dims, U, kappa, b, x)
    assert tr <= TOL
    assert abs(tr - res.true_residual) <= 1e-3 * tr + 1e-15
    # the FP64 solve agrees to the accuracy the condition number allows
    fx64 = hw.Field(lat)
    r64 = D.solve(fb, fx64, accuracy=TOL)
    x64 = fx64.download()
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-8


@pytest.mark.parametrize("precision", ["f32", "f16"])
def test_mixed_normal_equations(hw, ctx, oracle, precision):
    """CG<Op>::apply semantics in mixed precision: M^dag M x = in to 1e-10 (true)."""
    dims = (8, 8, 8, 8)
    U, lat, G = make(hw, ctx, oracle, dims, 21)
    src = oracle.gen_spinor(dims, 22, oracle.EVEN)
    D = hw.Dirac_Wilson_evenodd(0.12, G)
    fin, fout = hw.Field(lat, src), hw.Field(lat)
    res = hw.CG(D, accuracy=TOL, precision=precision).apply(fin, fout)
    assert res.converged, res
    assert oracle.true_residual_normal(dims, U, 0.12, src, fout.download()) <= TOL


@pytest.mark.parametrize("precision", ["f32", "f16"])
def test_mixed_initial_guess(hw, ctx, oracle, precision):
    """The solve starts from the x it is given (CG<Op>::apply starts from `out`).  A guess
    near the solution saves iterations; a guess that is nonzero on a single component must
    still be used (the first reliable update skips its FP64 hops only when x is zero
    everywhere); and a batch mixing zero and nonzero guesses gives bitwise the same
    solutions as each request alone."""
    dims, kappa = (8, 8, 8, 8), 0.12
    U, lat, G = make(hw, ctx, oracle, dims, 61)
    b = oracle.gen_spinor(dims, 62, oracle.EVEN)
    D = hw.Dirac_Wilson_evenodd(kappa, G)
    fb = hw.Field(lat, b)
    fx0 = hw.Field(lat)
    r0 = D.solve(fb, fx0, accuracy=TOL, precision=precision)
    assert r0.converged
    near = fx0.download() + 1e-4 * oracle.gen_spinor(dims, 63, oracle.EVEN)
    fx = hw.Field(lat, near)
    r = D.solve(fb, fx, accuracy=TOL, precision=precision)
    assert r.converged and r.iterations < r0.iterations, (r.iterations, r0.iterations)
    assert oracle.true_residual(dims, U, kappa, b, fx.download()) <= TOL
    even = np.flatnonzero(oracle.parity_mask(dims) == 0)
    spike = np.zeros_like(b)
    spike[even[len(even) // 2], 2, 1, 0] = 3.0
    fs = hw.Field(lat, spike)
    rs = D.solve(fb, fs, accuracy=TOL, precision=precision)
    assert rs.converged
    assert oracle.true_residual(dims, U, kappa, b, fs.download()) <= TOL
    # batched: a zero guess and the single-component guess together, then each alone
    fz, fsp = hw.Field(lat), hw.Field(lat, spike)
    both = hw.batch_solve(ctx, [(D, fb, fz, TOL), (D, fb, fsp, TOL)], precision=precision)
    assert all(q.converged for q in both)
    for guess, fout, res in ((None, fz, both[0]), (spike, fsp, both[1])):
        alone = hw.Field(lat) if guess is None else hw.Field(lat, guess)
        [ra] = hw.batch_solve(ctx, [(D, fb, alone, TOL)], precision=precision)
        assert ra.iterations == res.iterations
        assert np.array_equal(alone.download(), fout.download())
        assert oracle.true_residual(dims, U, kappa, b, fout.download()) <= TOL


def test_mixed_edge_cases(hw, ctx, oracle):
    dims = (4, 4, 4, 4)
    U, lat, G = make(hw, ctx, oracle, dims, 31)
    D = hw.Dirac_Wilson_evenodd(0.12, G)
    fb, fx = hw.Field(lat), hw.Field(lat)
    res = D.solve(fb, fx, precision="f16")
    assert res.converged and res.iterations == 0 and not fx.download().any()
    b = oracle.gen_spinor(dims, 32, oracle.EVEN)
    fb.upload(b)
    res = D.solve(fb, fx, accuracy=TOL, maxiters=3, precision="f16")
    assert res.status == hw.HW_ERR_NOT_CONVERGED and res.iterations == 3
    bad = b.copy()
    bad[5, 1, 1, 1] = np.inf
    fb.upload(bad)
    fx.zero()
    res = D.solve(fb, fx, precision="f32")
    assert res.status == hw.HW_ERR_BREAKDOWN
    fb.upload(b)
    fx.zero()
    assert D.solve(fb, fx, accuracy=TOL, precision="f32").converged


@pytest.mark.parametrize("precision", ["f16", "f32"])
def test_batch_uneven_lattices(hw, ctx, oracle, precision):
    """Several lattices of uneven volume, several right-hand sides each, in one batch."""
    specs = [((8, 8, 8, 8), 41, [0.115, 0.12, 0.124]), ((4, 4, 4, 8), 42, [0.12, 0.118]),
             ((6, 4, 4, 4), 43, [0.121]), ((8, 8, 4, 8), 44, [0.116, 0.124, 0.119, 0.12])]
    reqs, checks = [], []
    keep = []
    for dims, seed, kappas in specs:
        U, lat, G = make(hw, ctx, oracle, dims, seed)
        keep += [lat, G]
        for n, kappa in enumerate(kappas):
            b = oracle.gen_spinor(dims, 1000 * seed + n, oracle.EVEN)
            fb, fx = hw.Field(lat, b), hw.Field(lat)
            D = hw.Dirac_Wilson_evenodd(kappa, G)
            reqs.append((D, fb, fx, TOL))
            checks.append((dims, U, kappa, b, fx, D, fb))
    results = hw.batch_solve(ctx, reqs, precision=precision)
    for (dims, U, kappa, b, fx, D, fb), r in zip(checks, results):
        assert r.converged, r
        assert oracle.true_residual(dims, U, kappa, b, fx.download()) <= TOL
    # the same request alone gives bitwise the same solution
    dims, U, kappa, b, fx, D, fb = checks[1]
    fx2 = hw.Field(D.gauge.lattice)
    r2 = hw.batch_solve(ctx, [(D, fb, fx2, TOL)], precision=precision)[0]
    assert r2.iterations == results[1].iterations
    assert np.array_equal(fx2.download(), fx.download())


def test_batch_refills_slots(hw, ctx, oracle):
    """More right-hand sides than one lattice's 16 slots: later ones are admitted as slots free up."""
    dims = (4, 4, 4, 4)
    U, lat, G = make(hw, ctx, oracle, dims, 51)
    reqs, bs = [], []
    for n in range(20):
        b = oracle.gen_spinor(dims, 5100 + n, oracle.EVEN)
        D = hw.Dirac_Wilson_evenodd(0.115 + 0.0005 * (n % 10), G)
        reqs.append((D, hw.Field(lat, b), hw.Field(lat), TOL))
        bs.append(b)
    results = hw.batch_solve(ctx, reqs, precision="f16")
    for (D, fb, fx, _), b, r in zip(reqs, bs, results):
        assert r.converged
        assert oracle.true_residual(dims, U, D.kappa, b, fx.download()) <= TOL


@pytest.mark.parametrize("variant", [2, 4, 7])
def test_engine_launch_shapes(hw, ctx, oracle, variant, monkeypatch):
    """Every launch shape the FP16 engine keeps (HW_ENGINE_VARIANT: 2 one source per thread,
    4 the tensor-core hop, 7 the packed default): a batch of three sources on two lattices
    converges to true residual 1e-10 by the oracle, and each solve is bitwise the same alone
    as in the batch.  The tensor-core shape sums its products in another order, so its
    solutions are compared with the others only through the true residual."""
    monkeypatch.setenv("HW_ENGINE_VARIANT", str(variant))
    specs = [((8, 8, 8, 8), 81, 0.124), ((4, 4, 4, 8), 82, 0.12)]
    built = []
    for dims, seed, kappa in specs:
        U, lat, G = make(hw, ctx, oracle, dims, seed)
        built.append((dims, U, lat, hw.Dirac_Wilson_evenodd(kappa, G), kappa))
    work = []
    for n, (dims, U, lat, D, kappa) in enumerate(built):
        for k in range(2 if n == 0 else 1):
            b = oracle.gen_spinor(dims, 90 + 10 * n + k, oracle.EVEN)
            work.append((dims, U, lat, D, kappa, b, hw.Field(lat, b), hw.Field(lat)))
    res = hw.batch_solve(ctx, [(D, fb, fx, TOL) for (_, _, _, D, _, _, fb, fx) in work], precision="f16")
    for (dims, U, lat, D, kappa, b, fb, fx), r in zip(work, res):
        assert r.converged, (variant, r)
        x = fx.download()
        assert oracle.true_residual(dims, U, kappa, b, x) <= TOL
        alone = hw.Field(lat)
        [ra] = hw.batch_solve(ctx, [(D, fb, alone, TOL)], precision="f16")
        assert ra.iterations == r.iterations
        assert np.array_equal(alone.download(), x), variant


def test_engine_shapes_round_alike(hw, ctx, oracle, monkeypatch):
    """The one-source-per-thread shape (2) and the packed two-source default (7) round every
    product and sum in the same order: a batch gives bitwise the same solutions and
    iteration counts in both, so the shape can be chosen by speed alone."""
    specs = [((8, 8, 8, 8), 83, 0.124), ((4, 4, 4, 8), 84, 0.12)]
    work = []
    for n, (dims, seed, kappa) in enumerate(specs):
        U, lat, G = make(hw, ctx, oracle, dims, seed)
        D = hw.Dirac_Wilson_evenodd(kappa, G)
        for k in range(3 if n == 0 else 2):
            b = oracle.gen_spinor(dims, 300 + 10 * n + k, oracle.EVEN)
            work.append((lat, D, hw.Field(lat, b)))
    out = {}
    for variant in (7, 2):
        monkeypatch.setenv("HW_ENGINE_VARIANT", str(variant))
        xs = [hw.Field(lat) for (lat, _, _) in work]
        res = hw.batch_solve(ctx, [(D, fb, x, TOL) for (_, D, fb), x in zip(work, xs)], precision="f16")
        assert all(r.converged for r in res)
        out[variant] = ([r.iterations for r in res], [x.download() for x in xs])
    assert out[7][0] == out[2][0]
    for a, b in zip(out[7][1], out[2][1]):
        assert np.array_equal(a, b)


def test_engine_tuner(hw, ctx, oracle, monkeypatch):
    """The launch-shape tuner times its candidate shapes on the running solves, keeps the
    fastest for the work class, and the solves it switches shapes under give bitwise the
    same results as with one shape forced."""
    for k in ("HW_ENGINE_VARIANT", "HW_ENGINE_SCHED", "HW_ENGINE_TUNE"):
        monkeypatch.delenv(k, raising=False)
    dims, kappa = (12, 12, 12, 12), 0.122
    U, lat, G = make(hw, ctx, oracle, dims, 85)
    D = hw.Dirac_Wilson_evenodd(kappa, G)
    bs = [hw.Field(lat, oracle.gen_spinor(dims, 400 + k, oracle.EVEN)) for k in range(7)]

    def solve():
        xs = [hw.Field(lat) for _ in bs]
        res = hw.batch_solve(ctx, [(D, fb, x, TOL) for fb, x in zip(bs, xs)], precision="f16")
        assert all(r.converged for r in res)
        return [r.iterations for r in res], [x.download() for x in xs]

    # 7 solves x 81 tiles of 12^4 = 567: work class 10, the smallest the tuner times
    first = solve()
    entry = None
    for _ in range(16):
        entry = next((t for t in ctx.engine_tuning("f16") if t["work_class"] == 10), None)
        if entry is not None and entry["chosen"] is not None:
            break
        again = solve()
        assert again[0] == first[0]
        assert all(np.array_equal(a, b) for a, b in zip(again[1], first[1]))
    assert entry is not None and entry["chosen"] is not None, entry
    assert {(v, d) for v, d, _, _ in entry["shapes"]} == {(7, 1), (2, 1), (7, 0), (2, 0)}
    assert all(ms > 0 for _, _, ms, _ in entry["shapes"])
    monkeypatch.setenv("HW_ENGINE_VARIANT", "2")
    monkeypatch.setenv("HW_ENGINE_SCHED", "0")
    forced = solve()
    assert forced[0] == first[0]
    assert all(np.array_equal(a, b) for a, b in zip(forced[1], first[1]))
