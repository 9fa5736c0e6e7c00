"""GPU: the HMC callers of the eo solvers.

* gauge momenta: upload / download round trip, zero, squarenorm;
* the eo fermion force kernel (c2q_fermion_force_eo) against the oracle on
  non-trivial links with twisted boundary phases and chemical potentials
  (every link and generator component to 1e-12 of the largest), and against the
  known answers of physics/algorithms/fermion_force_test.cpp (cold 4^3x16 and
  conf.00200) to 1e-10;
* calc_fermion_force and calc_s_fermion (the eo CG branches of
  fermion_force.cpp and metropolis.cpp) against the oracle's restatement, with
  the FP64 CG of the reference's semantics and with the mixed-precision CG.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KATS = json.load(open(os.path.join(GOLD, "reference_kats.json")))
CONF = np.load(os.path.join(GOLD, "conf00200.npz"))


def test_gaugemomenta_round_trip(system):
    import cl2qcd_b200 as c2q
    L = c2q.Lattice(4, 8)
    a = np.random.default_rng(1).standard_normal((4 * L.vol, 8))
    gm = c2q.host.Gaugemomenta(system, L, a)
    assert np.array_equal(gm.download(), a)
    assert c2q.host.squarenorm(gm) == pytest.approx(float((a * a).sum()), rel=1e-13)
    gm.zero()
    assert not gm.download().any()
    assert c2q.host.squarenorm(gm) == 0.0


@pytest.mark.parametrize("bc", [(1.0, 0.0, None, None), (0.5, 0.3, None, 0.2), (1.0, 0.0, 0.1, None)])
def test_fermion_force_matches_oracle(port, system, O, bc):
    import cl2qcd_b200 as c2q
    tt, ts, cpr, cpi = bc
    ns, nt = 4, 8
    port.set_lattice(ns, nt, tt, ts, cpr, cpi)
    L = c2q.Lattice(ns, nt, tt, ts, cpr, cpi)
    g = port.gauge_fill(True)
    gf = c2q.Gaugefield(system, L, g)
    Yh = port.pseudo_randomize(port.seo, 21)
    Xh = port.pseudo_randomize(port.seo, 22)
    Y, X = c2q.Spinorfield_eo(system, L, Yh), c2q.Spinorfield_eo(system, L, Xh)
    gm0 = np.random.default_rng(23).standard_normal((4 * port.vol, 8))
    gm = c2q.host.Gaugemomenta(system, L, gm0)
    add = c2q.AdditionalParameters(0.15, 0.0)
    c2q.host.fermion_force(gm, Y, X, c2q.host.EVEN, gf, add)
    c2q.host.fermion_force(gm, X, Y, c2q.host.ODD, gf, add)
    ref = gm0.copy()
    port.fermion_force_eo(ref, Yh, Xh, g, O.EVEN, 0.15)
    port.fermion_force_eo(ref, Xh, Yh, g, O.ODD, 0.15)
    got = gm.download()
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("case", range(len(KATS["fermion_force_eo"])))
def test_fermion_force_kats(port, system, case):
    import cl2qcd_b200 as c2q
    kat = KATS["fermion_force_eo"][case]
    port.set_lattice(4, kat["nt"])
    L = c2q.Lattice(4, kat["nt"])
    g = CONF["gauge"] if kat["gauge"] == "conf.00200" else port.gauge_fill(False)
    gf = c2q.Gaugefield(system, L, g)
    e, o = port.convert_to_eo(port.pseudo_randomize(port.vol, kat["seed"]))
    sf1, sf2 = c2q.Spinorfield_eo(system, L, e), c2q.Spinorfield_eo(system, L, o)
    gm = c2q.host.Gaugemomenta(system, L)
    add = c2q.AdditionalParameters(kat["kappa"], 0.0)
    c2q.host.fermion_force(gm, sf1, sf2, c2q.host.EVEN, gf, add)
    assert c2q.host.squarenorm(gm) == pytest.approx(kat["refs"][0], rel=1e-10)
    c2q.host.fermion_force(gm, sf1, sf2, c2q.host.ODD, gf, add)
    assert c2q.host.squarenorm(gm) == pytest.approx(kat["refs"][1], rel=1e-10)


@pytest.mark.parametrize("case", range(len(KATS["fermion_force_full"])))
def test_fermion_force_full_kats(port, system, case):
    """the non-eo overload fermion_force(gm, Y, X, gf, params) on full fields"""
    import cl2qcd_b200 as c2q
    kat = KATS["fermion_force_full"][case]
    port.set_lattice(4, kat["nt"])
    L = c2q.Lattice(4, kat["nt"])
    g = CONF["gauge"] if kat["gauge"] == "conf.00200" else port.gauge_fill(False)
    gf = c2q.Gaugefield(system, L, g)
    sf1 = c2q.host.Spinorfield(system, L, port.pseudo_randomize(port.vol, kat["seeds"]["sf1"]))
    sf2 = c2q.host.Spinorfield(system, L, port.pseudo_randomize(port.vol, kat["seeds"]["sf2"]))
    gm = c2q.host.Gaugemomenta(system, L)
    c2q.host.fermion_force(gm, sf1, sf2, gf, c2q.AdditionalParameters(kat["kappa"], 0.0))
    assert c2q.host.squarenorm(gm) == pytest.approx(kat["refs"][0], rel=1e-10)


@pytest.mark.parametrize("precision", [64, 16])
@pytest.mark.parametrize("action", ["twistedmass", "wilson"])
def test_calc_fermion_force_and_energy(port, system, O, precision, action):
    import cl2qcd_b200 as c2q
    ns, nt = 8, 8
    port.set_lattice(ns, nt, 1.0, 0.0)
    L = c2q.Lattice(ns, nt, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, 0.3, 17)
    gf = c2q.Gaugefield(system, L, g)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    phih = c2q.host.generate_source(L.seo, "gaussian", 33)
    phi = c2q.Spinorfield_eo(system, L, phih)
    add = c2q.AdditionalParameters(kappa, mubar)
    act = O.TWISTEDMASS if action == "twistedmass" else O.WILSON
    ref_gm = port.gm_field()
    P = O.SolverParams(prec=1e-20, cgmax=5000, solver=2)
    port.calc_fermion_force_eo(ref_gm, phih, g, kappa, mubar, act, P)
    ref_s, _ = port.calc_s_fermion_eo(phih, g, kappa, mubar, act, P)
    if precision == 64:  # the reference's semantics: |r|^2 < prec
        params = c2q.SolverParameters(solver="cg", prec=1e-20, cgmax=5000, precision=64)
    else:
        params = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-12, cgmax=5000, precision=16,
                                      use_rec12=True)
    gm = c2q.host.Gaugemomenta(system, L)
    rep = {}
    c2q.host.calc_fermion_force(gm, gf, phi, params, add, action, rep)
    got = gm.download()
    d = np.linalg.norm(got - ref_gm) / np.linalg.norm(ref_gm)
    assert d <= 1e-9, d
    s = c2q.host.calc_s_fermion(gf, phi, params, add, action)
    assert s == pytest.approx(ref_s, rel=1e-10)
