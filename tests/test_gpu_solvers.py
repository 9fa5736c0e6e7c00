"""GPU parity of the eo fermion matrices and the CG / BiCGStab solvers, and the
true-residual bar ||b - A x|| / ||b|| <= 1e-10 for every precision mode."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

OPS = ["Aee", "Aee_minus", "Qplus_eo", "Qminus_eo", "QplusQminus_eo", "Aee_AND_gamma5_eo",
       "Aee_minus_AND_gamma5_eo"]


def _prob(port, c2q, system, ns=8, nt=8, eps=0.3, seed=3, kind="z2"):
    port.set_lattice(ns, nt, 1.0, 0.0)
    L = c2q.Lattice(ns, nt, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, eps, seed)
    gf = c2q.Gaugefield(system, L, g)
    b = c2q.host.generate_source(port.seo, kind, seed + 100)
    return L, g, gf, b


@pytest.mark.parametrize("name", OPS)
@pytest.mark.parametrize("action", ["twistedmass", "wilson"])
def test_fermionmatrix_matches_oracle(port, system, O, name, action):
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    op = {"Aee": O.OP_AEE, "Aee_minus": O.OP_AEE_MINUS, "Qplus_eo": O.OP_QPLUS_EO, "Qminus_eo": O.OP_QMINUS_EO,
          "QplusQminus_eo": O.OP_QPQM_EO, "Aee_AND_gamma5_eo": O.OP_AEE_G5,
          "Aee_minus_AND_gamma5_eo": O.OP_AEE_MINUS_G5}[name]
    ref = port.apply(op, b, g, kappa, mubar, action=O.WILSON if action == "wilson" else O.TWISTEDMASS)
    A = getattr(c2q.host, name)(action)
    X, Y = c2q.Spinorfield_eo(system, L, b), c2q.Spinorfield_eo(system, L)
    A(Y, gf, X, c2q.AdditionalParameters(kappa, mubar))
    assert rel_l2(Y.dump(), ref) <= 1e-12


def test_cg_matches_oracle_iteration_by_iteration(port, system, O):
    """Reference semantics (|r|^2 < prec absolute, checks every 10, refresh every 100):
    same iteration count and solution as the oracle's restated cg.cpp."""
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system, 8, 8)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    P = O.SolverParams(prec=1e-18, cgmax=3000, solver=1)
    x_ref = np.zeros_like(b)
    it_ref = port.cg(x_ref, O.OP_QPQM_EO, b, g, kappa, mubar, params=P)
    assert it_ref > 0
    X, B = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L, b)
    rep = {}
    it = c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, B,
                     c2q.SolverParameters(solver="cg", prec=1e-18, cgmax=3000), c2q.AdditionalParameters(kappa, mubar),
                     rep)
    assert it == it_ref
    assert rel_l2(X.dump(), x_ref) < 1e-8


@pytest.mark.parametrize("variant", ["bicgstab", "bicgstab_save"])
def test_bicgstab_matches_oracle(port, system, O, variant):
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system, 8, 4)
    kappa, mubar = 0.13, 2 * 0.13 * 0.05
    P = O.SolverParams(prec=1e-20, cgmax=1000, solver=2 if variant == "bicgstab" else 3)
    x_ref = np.zeros_like(b)
    it_ref = port.bicgstab(x_ref, O.OP_AEE, b, g, kappa, mubar, params=P)
    assert it_ref > 0
    X, B = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L, b)
    it = c2q.host.bicgstab(X, c2q.host.Aee(), gf, B, c2q.SolverParameters(solver=variant, prec=1e-20, cgmax=1000),
                           c2q.AdditionalParameters(kappa, mubar))
    assert abs(it - it_ref) <= 2
    assert rel_l2(X.dump(), x_ref) < 1e-8


@pytest.mark.parametrize("variant", ["bicgstab", "bicgstab_save"])
@pytest.mark.parametrize("precision", [32, 16])
@pytest.mark.parametrize("opname", ["Aee", "Qminus_eo"])
def test_mixed_bicgstab_true_residual(port, system, O, variant, precision, opname):
    """Mixed-precision BiCGStab (the iteration on FP32 / FP16 fields, FP64 reliable updates)
    reaches ||b - A x|| / ||b|| <= 1e-10, checked with the oracle operator, and agrees with the
    solution of the oracle's FP64 BiCGStab."""
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system, 8, 4)
    kappa, mubar = 0.13, 2 * 0.13 * 0.05
    opc = {"Aee": O.OP_AEE, "Qminus_eo": O.OP_QMINUS_EO}[opname]
    X, B = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L, b)
    rep = {}
    it = c2q.host.bicgstab(X, getattr(c2q.host, opname)(), gf, B,
                           c2q.SolverParameters(solver=variant, prec=0.0, rel_tol=1e-10, cgmax=5000,
                                                precision=precision), c2q.AdditionalParameters(kappa, mubar), rep)
    assert it > 0 and rep["reliable_updates"] >= 2, rep
    assert rep["true_resid_rel"] <= 1e-10, rep
    r = port.apply(opc, X.dump(), g, kappa, mubar)
    assert np.linalg.norm(r - b) / np.linalg.norm(b) <= 1.5e-10
    x_ref = np.zeros_like(b)
    assert port.bicgstab(x_ref, opc, b, g, kappa, mubar, params=O.SolverParams(prec=1e-20, cgmax=5000)) > 0
    assert rel_l2(X.dump(), x_ref) < 1e-8


@pytest.mark.parametrize("precision", [64, 32, 16])
@pytest.mark.parametrize("rec12", [False, True])
def test_cg_true_residual_1e10(port, system, O, precision, rec12):
    """8^4, eps 0.3, kappa 0.15, mu 0.01, Z2 source (the small plain-method configuration)."""
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system, 8, 8, 0.3, 1)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    X, B = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L, b)
    rep = {}
    c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, B,
                c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=20000, precision=precision,
                                     use_rec12=rec12), c2q.AdditionalParameters(kappa, mubar), rep)
    assert rep["true_resid_rel"] <= 1e-10, rep
    # independent check with the oracle operator
    r = port.apply(O.OP_QPQM_EO, X.dump(), g, kappa, mubar)
    assert np.linalg.norm(r - b) / np.linalg.norm(b) <= 1.5e-10


@pytest.mark.parametrize("iter_refresh", [100, 7])
def test_fp64_cg_graph_replay_matches_eager(port, system, O, iter_refresh):
    """FP64 CG with use_graph: the iterations between refreshes replay as a
    captured graph of the same kernels, so the iterates are bitwise those of the
    eager loop (also across refreshes, iter_refresh 7)."""
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system, 8, 8, 0.3, 1)
    add = c2q.AdditionalParameters(0.15, 2 * 0.15 * 0.01)
    B = c2q.Spinorfield_eo(system, L, b)
    out = {}
    for graph in (False, True):
        X = c2q.Spinorfield_eo(system, L)
        rep = {}
        c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, B,
                    c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=20000, precision=64,
                                         iter_refresh=iter_refresh, use_graph=graph), add, rep)
        assert rep["true_resid_rel"] <= 1e-10, rep
        out[graph] = (X.dump(), rep["iterations"], rep["dslash_applications"])
    assert out[True][1] == out[False][1] and out[True][2] == out[False][2]
    assert np.array_equal(out[True][0], out[False][0])


def test_solver_errors(port, system, O):
    """Host-side failure injection: NaN in the source -> SolverStuck; cgmax too small -> SolverDidNotSolve."""
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system, 4, 4)
    add = c2q.AdditionalParameters(0.15, 0.003)
    X = c2q.Spinorfield_eo(system, L)
    with pytest.raises(c2q.SolverDidNotSolve):
        c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, c2q.Spinorfield_eo(system, L, b),
                    c2q.SolverParameters(solver="cg", cgmax=3), add)
    bad = b.copy()
    bad[3, 5] = np.nan
    X.zero()
    with pytest.raises(c2q.SolverStuck):
        c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, c2q.Spinorfield_eo(system, L, bad),
                    c2q.SolverParameters(solver="cg", cgmax=50), add)
    X.zero()
    with pytest.raises(c2q.SolverStuck):
        c2q.host.bicgstab(X, c2q.host.Aee(), gf, c2q.Spinorfield_eo(system, L, bad),
                          c2q.SolverParameters(solver="bicgstab", cgmax=50), add)
    with pytest.raises(c2q.host.InvalidParameters):
        c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, c2q.Spinorfield_eo(system, L, b),
                    c2q.SolverParameters(solver="cg", iter_refresh=0), add)


@pytest.mark.parametrize("solver", ["bicgstab", "cg"])
def test_perform_inversion_matches_oracle(port, system, O, solver):
    import cl2qcd_b200 as c2q
    port.set_lattice(4, 8, 1.0, 0.0)
    L = c2q.Lattice(4, 8, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, 0.25, 4)
    gf = c2q.Gaugefield(system, L, g)
    src = c2q.host.generate_source(port.vol, "gaussian", 5)
    kappa, mubar = 0.14, 2 * 0.14 * 0.05
    P = O.SolverParams(prec=1e-22, cgmax=2000, solver=1 if solver == "cg" else 2)
    ref, it_ref, used = port.perform_inversion_eo(src, g, kappa, mubar, params=P)
    out, it = c2q.host.perform_inversion(system, gf, src, c2q.SolverParameters(solver=solver, prec=1e-22,
                                                                               cgmax=2000),
                                         c2q.AdditionalParameters(kappa, mubar))
    assert rel_l2(out, ref) < 1e-9
    # the reference's eo inversion returns -M^{-1} b
    assert rel_l2(port.m_tm_plus(-out, g, kappa, mubar), src) < 1e-9


@pytest.mark.parametrize("precision", [32, 16])
def test_perform_inversion_mixed_bicgstab(port, system, O, precision):
    """perform_inversion with the reference's default solver (bicgstab) in mixed precision."""
    import cl2qcd_b200 as c2q
    port.set_lattice(4, 8, 1.0, 0.0)
    L = c2q.Lattice(4, 8, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, 0.25, 4)
    gf = c2q.Gaugefield(system, L, g)
    src = c2q.host.generate_source(port.vol, "gaussian", 5)
    kappa, mubar = 0.14, 2 * 0.14 * 0.05
    ref, _, _ = port.perform_inversion_eo(src, g, kappa, mubar, params=O.SolverParams(prec=1e-22, cgmax=2000))
    out, it = c2q.host.perform_inversion(system, gf, src, c2q.SolverParameters(
        solver="bicgstab", prec=0.0, rel_tol=1e-11, cgmax=2000, precision=precision),
        c2q.AdditionalParameters(kappa, mubar))
    assert rel_l2(out, ref) < 1e-9
    assert rel_l2(port.m_tm_plus(-out, g, kappa, mubar), src) < 1e-9


@pytest.mark.parametrize("bc", [(0.0, 0.0, None, None), (1.0, 0.0, None, None), (1.0, 0.5, None, 0.1)])
@pytest.mark.parametrize("precision", [32, 16])
def test_mixed_cg_all_phase_patterns(port, system, O, bc, precision):
    """The reduced-precision sweeps are specialised for all-real phases, complex T
    phases only, and general phases; each must drive the mixed CG to 1e-10 in about
    as many iterations as FP64 (a wrong inner operator would not converge).  The
    general case uses a spatial phase and an imaginary chemical potential: a real
    chemical potential breaks the gamma5-hermiticity that CG on QplusQminus_eo needs."""
    import cl2qcd_b200 as c2q
    tt, ts, cpr, cpi = bc
    port.set_lattice(8, 8, tt, ts, cpr, cpi)
    L = c2q.Lattice(8, 8, tt, ts, cpr, cpi)
    g = c2q.host.generate_gaugefield(L, 0.3, 9)
    gf = c2q.Gaugefield(system, L, g)
    b = c2q.host.generate_source(port.seo, "gaussian", 10)
    add = c2q.AdditionalParameters(0.14, 2 * 0.14 * 0.02)
    B = c2q.Spinorfield_eo(system, L, b)
    reps = {}
    for prec in (64, precision):
        X = c2q.Spinorfield_eo(system, L)
        reps[prec] = {}
        c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, B,
                    c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=5000, precision=prec,
                                         use_rec12=True), add, reps[prec])
        assert reps[prec]["true_resid_rel"] <= 1e-10
        r = port.apply(O.OP_QPQM_EO, X.dump(), g, add.kappa, add.mubar)
        assert np.linalg.norm(r - b) / np.linalg.norm(b) <= 1.5e-10
    assert reps[precision]["iterations"] <= 1.3 * reps[64]["iterations"] + 10
