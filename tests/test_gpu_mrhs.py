"""GPU: multi-right-hand-side mixed-precision CG (c2q_cg_multi).

Every right-hand side of a batch must reach the true FP64 residual bar
||b - A x|| / ||b|| <= 1e-10 and agree with the same right-hand side solved
alone: the batched sweeps and vector updates keep per-right-hand-side
reductions in the same block order as a single solve, so the iterates are the
same whether a source is solved alone or in a batch (asserted to 1e-12
relative).  Graph-captured iterations must give the same result as eager ones.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(port, c2q, system, ns=8, nt=8, eps=0.3, seed=3):
    port.set_lattice(ns, nt, 1.0, 0.0)
    L = c2q.Lattice(ns, nt, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, eps, seed)
    return L, g, c2q.Gaugefield(system, L, g)


def _params(c2q, precision, graph=False, cgmax=5000):
    return c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=cgmax, precision=precision,
                                use_rec12=True, use_graph=graph)


@pytest.mark.parametrize("precision", [32, 16])
def test_batch_matches_single_solves(port, system, O, precision):
    import cl2qcd_b200 as c2q
    L, g, gf = _problem(port, c2q, system)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    add = c2q.AdditionalParameters(kappa, mubar)
    A = c2q.host.QplusQminus_eo()
    srcs = [c2q.host.generate_source(L.seo, "z2" if k % 2 else "gaussian", 100 + k) for k in range(5)]
    bs = [c2q.Spinorfield_eo(system, L, s) for s in srcs]
    xs = [c2q.Spinorfield_eo(system, L) for _ in srcs]
    reps = []
    its = c2q.host.cg_multi(xs, A, gf, bs, _params(c2q, precision), add, reps)
    assert len(its) == 5
    for k, s in enumerate(srcs):
        assert reps[k]["true_resid_rel"] <= 1e-10, (k, reps[k])
        r = port.apply(O.OP_QPQM_EO, xs[k].dump(), g, kappa, mubar)
        assert np.linalg.norm(r - s) / np.linalg.norm(s) <= 1.5e-10
        x1 = c2q.Spinorfield_eo(system, L)
        rep1 = {}
        c2q.host.cg(x1, A, gf, bs[k], _params(c2q, precision), add, rep1)
        assert rep1["iterations"] == reps[k]["iterations"]
        d = np.linalg.norm(x1.dump() - xs[k].dump()) / np.linalg.norm(x1.dump())
        assert d <= 1e-12, (k, d)


@pytest.mark.parametrize("precision", [32, 16])
def test_twelve_point_sources_with_graphs(port, system, O, precision):
    """12 spin-colour point sources at the origin, one batch, graph-captured iterations."""
    import cl2qcd_b200 as c2q
    L, g, gf = _problem(port, c2q, system, 8, 8, 0.25, 7)
    kappa, mubar = 0.16, 2 * 0.16 * 0.005
    add = c2q.AdditionalParameters(kappa, mubar)
    A = c2q.host.QplusQminus_eo()
    srcs = [c2q.host.point_source(L.seo, k) for k in range(12)]
    bs = [c2q.Spinorfield_eo(system, L, s) for s in srcs]
    xg = [c2q.Spinorfield_eo(system, L) for _ in srcs]
    xe = [c2q.Spinorfield_eo(system, L) for _ in srcs]
    rg, re_ = [], []
    c2q.host.cg_multi(xg, A, gf, bs, _params(c2q, precision, graph=True), add, rg)
    c2q.host.cg_multi(xe, A, gf, bs, _params(c2q, precision, graph=False), add, re_)
    for k in range(12):
        assert rg[k]["true_resid_rel"] <= 1e-10, (k, rg[k])
        assert rg[k]["iterations"] == re_[k]["iterations"]
        assert np.array_equal(xg[k].dump(), xe[k].dump())
        r = port.apply(O.OP_QPQM_EO, xg[k].dump(), g, kappa, mubar)
        assert np.linalg.norm(r - srcs[k]) <= 1.5e-10


def test_more_sources_than_one_batch(port, system, O):
    """17 sources: one batch of 16 and one of 1, FP16, graph-captured."""
    import cl2qcd_b200 as c2q
    L, g, gf = _problem(port, c2q, system, 4, 8, 0.3, 11)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    add = c2q.AdditionalParameters(kappa, mubar)
    A = c2q.host.QplusQminus_eo()
    srcs = [c2q.host.generate_source(L.seo, "gaussian", 300 + k) for k in range(17)]
    bs = [c2q.Spinorfield_eo(system, L, s) for s in srcs]
    xs = [c2q.Spinorfield_eo(system, L) for _ in srcs]
    reps = []
    c2q.host.cg_multi(xs, A, gf, bs, _params(c2q, 16, graph=True), add, reps)
    for k in range(17):
        assert reps[k]["true_resid_rel"] <= 1e-10, (k, reps[k])


def test_multi_fp64_is_the_reference_cg(port, system, O):
    import cl2qcd_b200 as c2q
    L, g, gf = _problem(port, c2q, system, 4, 4, 0.3, 5)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    add = c2q.AdditionalParameters(kappa, mubar)
    A = c2q.host.QplusQminus_eo()
    srcs = [c2q.host.generate_source(L.seo, "z2", 40 + k) for k in range(3)]
    bs = [c2q.Spinorfield_eo(system, L, s) for s in srcs]
    xs = [c2q.Spinorfield_eo(system, L) for _ in srcs]
    reps = []
    c2q.host.cg_multi(xs, A, gf, bs, c2q.SolverParameters(solver="cg", prec=1e-22, cgmax=2000), add, reps)
    P = O.SolverParams(prec=1e-22, cgmax=2000, solver=1)
    for k in range(3):
        xo = port.eo_field()
        it = port.cg(xo, O.OP_QPQM_EO, srcs[k], g, kappa, mubar, O.TWISTEDMASS, P)
        assert reps[k]["iterations"] == it
        assert np.linalg.norm(xs[k].dump() - xo) / np.linalg.norm(xo) <= 1e-10


def test_multi_rejects_aliasing(system):
    import cl2qcd_b200 as c2q
    L = c2q.Lattice(4, 4)
    gf = c2q.Gaugefield(system, L, c2q.host.generate_gaugefield(L, 0.3, 1))
    b = c2q.Spinorfield_eo(system, L, c2q.host.generate_source(L.seo, "z2", 1))
    x = c2q.Spinorfield_eo(system, L)
    with pytest.raises(c2q.InvalidParameters):
        c2q.host.cg_multi([x, x], c2q.host.QplusQminus_eo(), gf, [b, b], c2q.SolverParameters(precision=16),
                          c2q.AdditionalParameters(0.15, 0.003))


@pytest.mark.parametrize("precision", [32, 16])
def test_zero_source_in_batch(port, system, O, precision):
    """A zero source in a batch is solved exactly by x = 0 without iterating (alpha would be 0/0);
    the other right-hand sides iterate as if solved alone.  The FP64 CG keeps the reference's
    behaviour on a zero source (a stuck solver, physics/algorithms/solvers/cg.cpp:93-119)."""
    import cl2qcd_b200 as c2q
    L, g, gf = _problem(port, c2q, system)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    add = c2q.AdditionalParameters(kappa, mubar)
    A = c2q.host.QplusQminus_eo()
    srcs = [c2q.host.generate_source(L.seo, "gaussian", 200), np.zeros((L.seo, 24)),
            c2q.host.generate_source(L.seo, "z2", 201)]
    bs = [c2q.Spinorfield_eo(system, L, s) for s in srcs]
    xs = [c2q.Spinorfield_eo(system, L) for _ in srcs]
    reps = []
    its = c2q.host.cg_multi(xs, A, gf, bs, _params(c2q, precision, graph=True), add, reps)
    assert its[1] == 0 and reps[1]["status"] == 0 and reps[1]["true_resid_rel"] == 0.0
    assert not np.any(xs[1].dump())
    for k in (0, 2):
        assert reps[k]["true_resid_rel"] <= 1e-10, (k, reps[k])
        x1 = c2q.Spinorfield_eo(system, L)
        rep1 = {}
        c2q.host.cg(x1, A, gf, bs[k], _params(c2q, precision), add, rep1)
        assert rep1["iterations"] == reps[k]["iterations"]
    x0 = c2q.Spinorfield_eo(system, L)
    c2q.host.cg(x0, A, gf, bs[1], _params(c2q, precision), add)
    assert not np.any(x0.dump())
    with pytest.raises(c2q.SolverStuck):
        c2q.host.cg(x0, A, gf, bs[1], c2q.SolverParameters(solver="cg", prec=1e-22, cgmax=50), add)


@pytest.mark.parametrize("rec12", [True, False])
@pytest.mark.parametrize("nsrc", [2, 5, 12])
def test_two_sources_per_thread_is_bitwise_the_same(port, system, O, nsrc, rec12):
    """The FP16 batched sweeps that run two right-hand sides per thread (each link
    staged and decoded once for both; sweep choice 4) give bitwise the solutions
    of the one-source-per-thread sweeps (choice 0), an odd last source included,
    and every solution meets the true-residual bar of the oracle's operator."""
    import cl2qcd_b200 as c2q
    L, g, gf = _problem(port, c2q, system, 8, 8, 0.3, 5)
    kappa, mubar = 0.155, 2 * 0.155 * 0.008
    add = c2q.AdditionalParameters(kappa, mubar)
    A = c2q.host.QplusQminus_eo()
    srcs = [c2q.host.generate_source(L.seo, "gaussian", 300 + k) for k in range(nsrc)]
    bs = [c2q.Spinorfield_eo(system, L, s) for s in srcs]
    P = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=5000, precision=16, use_rec12=rec12)
    out = {}
    try:
        for choice in (0, 4):
            system.set_sweep_choice(choice)
            xs = [c2q.Spinorfield_eo(system, L) for _ in srcs]
            reps = []
            c2q.host.cg_multi(xs, A, gf, bs, P, add, reps)
            out[choice] = ([x.dump() for x in xs], [r["iterations"] for r in reps])
    finally:
        system.set_sweep_choice(-1)
    assert out[0][1] == out[4][1]
    for k in range(nsrc):
        assert np.array_equal(out[0][0][k], out[4][0][k]), k
        r = port.apply(O.OP_QPQM_EO, out[4][0][k], g, kappa, mubar)
        assert np.linalg.norm(r - srcs[k]) / np.linalg.norm(srcs[k]) <= 1.5e-10


@pytest.mark.parametrize("shape", [(8, 8), (6, 8), (4, 12)])
def test_every_sweep_choice_is_bitwise_the_same(port, system, O, shape):
    """The FP16 mixed-precision CG (temporal gauge, 12-real links, fused x / r
    updates) gives bitwise the same solution and iterations with every launch
    choice (both configurations, one block per tile or grid-stride).  6^3x8 and
    4^3x12 end in a ragged last tile."""
    import cl2qcd_b200 as c2q
    ns, nt = shape
    L, g, gf = _problem(port, c2q, system, ns, nt, 0.3, 5)
    add = c2q.AdditionalParameters(0.15, 2 * 0.15 * 0.01)
    src = c2q.host.generate_source(L.seo, "gaussian", 77)
    B = c2q.Spinorfield_eo(system, L, src)
    P = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=5000, precision=16, use_rec12=True)
    out = {}
    try:
        for choice in (0, 1, 2, 3):
            system.set_sweep_choice(choice)
            X = c2q.Spinorfield_eo(system, L)
            rep = {}
            c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, B, P, add, rep)
            out[choice] = (X.dump(), rep["iterations"])
    finally:
        system.set_sweep_choice(-1)
    for choice in (1, 2, 3):
        assert out[choice][1] == out[0][1], (choice, out[choice][1], out[0][1])
        assert np.array_equal(out[choice][0], out[0][0]), choice
    r = port.apply(O.OP_QPQM_EO, out[0][0], g, 0.15, 2 * 0.15 * 0.01)
    assert np.linalg.norm(r - src) / np.linalg.norm(src) <= 1.5e-10


def test_sweep_choice_falls_back_where_it_does_not_apply(port, system, O):
    """Choice 4 on an FP32 batch (no two-per-thread kernel) runs choice 0."""
    import cl2qcd_b200 as c2q
    L, g, gf = _problem(port, c2q, system, 8, 8, 0.3, 5)
    add = c2q.AdditionalParameters(0.15, 0.003)
    srcs = [c2q.host.generate_source(L.seo, "z2", 400 + k) for k in range(3)]
    bs = [c2q.Spinorfield_eo(system, L, s) for s in srcs]
    P = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=5000, precision=32, use_rec12=True)
    res = {}
    try:
        for choice in (0, 4):
            system.set_sweep_choice(choice)
            xs = [c2q.Spinorfield_eo(system, L) for _ in srcs]
            c2q.host.cg_multi(xs, c2q.host.QplusQminus_eo(), gf, bs, P, add)
            res[choice] = [x.dump() for x in xs]
    finally:
        system.set_sweep_choice(-1)
    assert all(np.array_equal(a, b) for a, b in zip(res[0], res[4]))
