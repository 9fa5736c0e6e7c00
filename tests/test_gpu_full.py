"""GPU: the full-lattice (non-eo) fermion matrices through c2q_apply_full.

* physics/fermionmatrix/explicit_test.cpp: M_wilson, M_tm_plus, M_tm_minus on the
  cold 4^3x16 field (first blocks) and on the ILDG configuration conf.00200
  (second blocks), at the reference's 0.01 %;
* M_tm_plus / minus, Qplus / Qminus (= g5 M) and QplusQminus against the oracle's
  full-lattice operator (relative L2 <= 1e-12) with boundary phases;
* the eo inversion solves the full system: M_tm_plus phi = -b for the result phi of
  perform_inversion (its sign convention), checked in FP64 on the GPU.
"""
import json
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KATS = json.load(open(os.path.join(GOLD, "reference_kats.json")))


@pytest.mark.parametrize("block", ["explicit_full_cold", "explicit_conf00200"])
@pytest.mark.parametrize("name", ["M_wilson", "M_tm_plus", "M_tm_minus"])
def test_explicit_full_kats(system, port, block, name):
    import cl2qcd_b200 as c2q
    kat = KATS[block][name]
    ns, nt = kat["lattice"]
    port.set_lattice(ns, nt)
    L = c2q.Lattice(ns, nt)
    if block == "explicit_full_cold":
        g = np.zeros((4 * L.vol, 18))
        g[:, 0] = g[:, 8] = g[:, 16] = 1.0
    else:
        g = np.load(os.path.join(GOLD, "conf00200.npz"))["gauge"]
    gf = c2q.Gaugefield(system, L, g)
    sf1 = c2q.host.Spinorfield(system, L, port.pseudo_randomize(L.vol, kat["seeds"]["sf1"]))
    sf2 = c2q.host.Spinorfield(system, L)
    kappa, mubar = kat["kappa"], 2 * kat["kappa"] * kat["mu"]
    add = c2q.AdditionalParameters(kappa, mubar)
    if name == "M_wilson":
        op = lambda o, i: c2q.host.M_wilson(o, gf, i, kappa)
    else:
        A = {"M_tm_plus": c2q.host.M_tm_plus(), "M_tm_minus": c2q.host.M_tm_minus()}[name]
        op = lambda o, i: A(o, gf, i, add)
    op(sf2, sf1)
    assert c2q.host.squarenorm_full(sf2) == pytest.approx(kat["refs"][0], rel=1e-4)
    op(sf1, sf2)
    assert c2q.host.squarenorm_full(sf1) == pytest.approx(kat["refs"][1], rel=1e-4)


@pytest.mark.parametrize("name", ["M_tm_plus", "M_tm_minus", "Qplus", "Qminus", "QplusQminus"])
def test_full_operators_match_oracle(system, port, name):
    import cl2qcd_b200 as c2q
    ns, nt, tt, ts = 6, 8, 1.0, 0.3
    port.set_lattice(ns, nt, tt, ts)
    L = c2q.Lattice(ns, nt, tt, ts)
    g = c2q.host.generate_gaugefield(L, 0.3, 21)
    gf = c2q.Gaugefield(system, L, g)
    s = port.pseudo_randomize(L.vol, 17)
    kappa, mubar = 0.15, 0.03
    X, Y = c2q.host.Spinorfield(system, L, s), c2q.host.Spinorfield(system, L)
    getattr(c2q.host, name)()(Y, gf, X, c2q.AdditionalParameters(kappa, mubar))

    def g5(a):
        a = a.copy()
        port.lib.c2qo_gamma5_full(a)
        return a

    mp = lambda a: port.m_tm_plus(a, g, kappa, mubar)
    mm = lambda a: port.m_tm_minus(a, g, kappa, mubar)
    ref = {"M_tm_plus": lambda: mp(s), "M_tm_minus": lambda: mm(s), "Qplus": lambda: g5(mp(s)),
           "Qminus": lambda: g5(mm(s)), "QplusQminus": lambda: g5(mp(g5(mm(s))))}[name]()
    assert rel_l2(Y.dump(), ref) <= 1e-12


def test_inversion_solves_the_full_system(system, port):
    """perform_inversion returns -M^{-1} b (inversion.cpp:165-169, :204-221): M phi = -b."""
    import cl2qcd_b200 as c2q
    ns, nt = 8, 8
    port.set_lattice(ns, nt, 1.0, 0.0)
    L = c2q.Lattice(ns, nt, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, 0.3, 5)
    gf = c2q.Gaugefield(system, L, g)
    b = port.pseudo_randomize(L.vol, 9)
    add = c2q.AdditionalParameters(0.15, 2 * 0.15 * 0.01)
    phi, _ = c2q.host.perform_inversion(system, gf, b, c2q.SolverParameters(solver="bicgstab", prec=1e-24), add)
    P, R = c2q.host.Spinorfield(system, L, phi), c2q.host.Spinorfield(system, L)
    c2q.host.M_tm_plus()(R, gf, P, add)
    assert np.linalg.norm(R.dump() + b) / np.linalg.norm(b) <= 1e-10


@pytest.mark.parametrize("solver", ["bicgstab", "cg", "bicgstab_save"])
def test_full_lattice_inversion(system, port, solver):
    """useEO=false (inversion.cpp:98-122): the full-lattice solve returns M^{-1} b,
    and agrees with the eo solve (whose convention is -M^{-1} b)."""
    import cl2qcd_b200 as c2q
    ns, nt = 8, 8
    port.set_lattice(ns, nt, 1.0, 0.0)
    L = c2q.Lattice(ns, nt, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, 0.3, 5)
    gf = c2q.Gaugefield(system, L, g)
    b = port.pseudo_randomize(L.vol, 9)
    add = c2q.AdditionalParameters(0.15, 2 * 0.15 * 0.01)
    params = c2q.SolverParameters(solver=solver, prec=1e-24, cgmax=4000)
    rep = {}
    phi, _ = c2q.host.perform_inversion(system, gf, b, params, add, report=rep, use_eo=False)
    r = port.m_tm_plus(np.ascontiguousarray(phi.reshape(-1, 24)), g, 0.15, 2 * 0.15 * 0.01)
    assert np.linalg.norm(r - b) / np.linalg.norm(b) <= 1e-10, rep
    phi_eo, _ = c2q.host.perform_inversion(system, gf, b, params, add)
    assert np.linalg.norm(phi + phi_eo) / np.linalg.norm(phi) <= 1e-9


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
def test_full_lattice_solvers(system, port, solver):
    """solvers::cg on QplusQminus and bicgstab on M_tm_plus with full fields."""
    import cl2qcd_b200 as c2q
    ns, nt = 4, 8
    port.set_lattice(ns, nt, 1.0, 0.3)
    L = c2q.Lattice(ns, nt, 1.0, 0.3)
    g = c2q.host.generate_gaugefield(L, 0.3, 7)
    gf = c2q.Gaugefield(system, L, g)
    kappa, mubar = 0.15, 2 * 0.15 * 0.02
    add = c2q.AdditionalParameters(kappa, mubar)
    bh = port.pseudo_randomize(L.vol, 3)
    b = c2q.host.Spinorfield(system, L, bh)
    x = c2q.host.Spinorfield(system, L)
    params = c2q.SolverParameters(solver=solver, prec=0.0, rel_tol=1e-11, cgmax=4000)
    rep = {}
    if solver == "cg":
        it = c2q.host.cg(x, c2q.host.QplusQminus(), gf, b, params, add, rep)
        g5 = np.where(np.arange(24) < 12, 1.0, -1.0)  # spins 2, 3 flip sign
        xm = port.m_tm_minus(x.dump(), g, kappa, mubar) * g5
        ax = port.m_tm_plus(np.ascontiguousarray(xm), g, kappa, mubar) * g5  # Q+ Q- x = g5 M+ g5 M- x
    else:
        it = c2q.host.bicgstab(x, c2q.host.M_tm_plus(), gf, b, params, add, rep)
        ax = port.m_tm_plus(x.dump(), g, kappa, mubar)
    assert it > 0 and rep["true_resid_rel"] <= 1e-11
    assert np.linalg.norm(ax - bh) / np.linalg.norm(bh) <= 1e-10
