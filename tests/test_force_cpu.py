"""CPU: the HMC callers of the eo solvers in the oracle (test infrastructure).

* the eo fermion force (fermion_force_eo_0..3 of ocl_kernel/force_fermion_eo.cl)
  of both oracle builds against the known answers of
  physics/algorithms/fermion_force_test.cpp (cold 4^3x16 and conf.00200, at the
  reference's 0.01 % and, since both builds reproduce them to rounding, at 1e-10);
* the restatement ("port") against the reference's own kernel compiled as C
  ("reference") on non-trivial links with twisted boundary phases and chemical
  potentials, where every link and every generator component must agree;
* calc_fermion_force and calc_s_fermion (fermion_force.cpp, metropolis.cpp, CG
  branches) of the two builds against each other.
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KATS = json.load(open(os.path.join(GOLD, "reference_kats.json")))
CONF = np.load(os.path.join(GOLD, "conf00200.npz"))


def _oracle(request, kind):
    return request.getfixturevalue("port" if kind == "port" else "ref")


@pytest.mark.parametrize("kind", ["port", "reference"])
@pytest.mark.parametrize("case", range(len(KATS["fermion_force_eo"])))
def test_fermion_force_eo_kats(request, O, kind, case):
    o = _oracle(request, kind)
    kat = KATS["fermion_force_eo"][case]
    o.set_lattice(4, kat["nt"])
    g = CONF["gauge"] if kat["gauge"] == "conf.00200" else o.gauge_fill(False)
    sf1, sf2 = o.convert_to_eo(o.pseudo_randomize(o.vol, kat["seed"]))
    gm = o.gm_field()
    o.fermion_force_eo(gm, sf1, sf2, g, O.EVEN, kat["kappa"])
    even = o.gm_squarenorm(gm)
    o.fermion_force_eo(gm, sf1, sf2, g, O.ODD, kat["kappa"])
    both = o.gm_squarenorm(gm)
    assert even == pytest.approx(kat["refs"][0], rel=1e-4)
    assert both == pytest.approx(kat["refs"][1], rel=1e-4)
    assert even == pytest.approx(kat["refs"][0], rel=1e-10)
    assert both == pytest.approx(kat["refs"][1], rel=1e-10)


@pytest.mark.parametrize("kind", ["port", "reference"])
@pytest.mark.parametrize("case", range(len(KATS["fermion_force_full"])))
def test_fermion_force_full_kats(request, O, kind, case):
    """the non-eo force (case fermion_force): the reference's own kernel, and the
    restatement as the eo force of both parities"""
    o = _oracle(request, kind)
    kat = KATS["fermion_force_full"][case]
    o.set_lattice(4, kat["nt"])
    g = CONF["gauge"] if kat["gauge"] == "conf.00200" else o.gauge_fill(False)
    sf1 = o.pseudo_randomize(o.vol, kat["seeds"]["sf1"])
    sf2 = o.pseudo_randomize(o.vol, kat["seeds"]["sf2"])
    gm = o.gm_field()
    o.fermion_force_full(gm, sf1, sf2, g, kat["kappa"])
    assert o.gm_squarenorm(gm) == pytest.approx(kat["refs"][0], rel=1e-10)


@pytest.mark.parametrize("bc", [(1.0, 0.0, None, None), (0.5, 0.3, None, 0.2), (1.0, 0.0, 0.1, None)])
def test_force_port_matches_reference_kernel(port, ref, O, bc):
    tt, ts, cpr, cpi = bc
    for o in (port, ref):
        o.set_lattice(4, 8, tt, ts, cpr, cpi)
    g = port.gauge_fill(True)
    Y = port.pseudo_randomize(port.seo, 21)
    X = port.pseudo_randomize(port.seo, 22)
    gm0 = np.random.default_rng(23).standard_normal((4 * port.vol, 8))  # the force adds to what is there
    out = []
    for o in (port, ref):
        gm = gm0.copy()
        o.fermion_force_eo(gm, Y, X, g, O.EVEN, 0.15)
        o.fermion_force_eo(gm, X, Y, g, O.ODD, 0.15)
        out.append(gm)
    np.testing.assert_allclose(out[0], out[1], rtol=0, atol=1e-12 * np.abs(out[1]).max())


@pytest.mark.parametrize("action", ["twistedmass", "wilson"])
def test_calc_fermion_force_and_energy_port_vs_reference(port, ref, O, action):
    act = O.TWISTEDMASS if action == "twistedmass" else O.WILSON
    res = []
    for o in (port, ref):
        o.set_lattice(4, 4, 1.0, 0.0)
        g = CONF["gauge"]
        phi = o.pseudo_randomize(o.seo, 31)
        gm = o.gm_field()
        P = O.SolverParams(prec=1e-24, cgmax=2000, solver=2)
        it = o.calc_fermion_force_eo(gm, phi, g, 0.15, 2 * 0.15 * 0.01, act, P)
        s, it2 = o.calc_s_fermion_eo(phi, g, 0.15, 2 * 0.15 * 0.01, act, P)
        assert it > 0 and it2 == it
        res.append((gm, s))
    np.testing.assert_allclose(res[0][0], res[1][0], rtol=0, atol=1e-10 * np.abs(res[1][0]).max())
    assert res[0][1] == pytest.approx(res[1][1], rel=1e-10)
