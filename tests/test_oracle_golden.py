"""CPU: the oracle is pinned to the reference's own known answers.

Both oracle builds -- the C restatement ("port") and the reference's kernels
compiled as C ("reference") -- must reproduce the golden values that the
reference's tests hold for this path (tests/golden/reference_kats.json, taken
from hardware/code/fermions_test.cpp, physics/fermionmatrix/explicit_test.cpp
and fermionmatrix_test.cpp), at the reference's own tolerances, and agree with
each other to rounding.
"""
import json
import math
import os

import numpy as np
import pytest

from conftest import rel_l2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KATS = json.load(open(os.path.join(GOLD, "reference_kats.json")))
BACKENDS = ["port", "reference"]


def _oracle(request, kind):
    return request.getfixturevalue("port" if kind == "port" else "ref")


def closed_form(seo, ns, nt, th_t, th_s, cpr, cpi):
    c = KATS["dslash_eo_closed_form"]["coefficients"]
    aS, aT = math.pi * th_s / ns, cpi + math.pi * th_t / nt
    return seo * (c[0] * math.cos(aS) + c[1] * math.cos(aT) * math.cosh(cpr) + c[2] * math.sin(aS)
                  + c[3] * math.cosh(cpr) * math.sin(aT) + c[4] * math.cos(aT) * math.sinh(cpr)
                  + c[5] * math.sin(aT) * math.sinh(cpr))


# hardware/code/fermions_test.cpp:662-697 (DSLASH_EO_1/2, DSLASH_EO_BC_AND_CHEMPOT_1/2)
DSLASH_CASES = [(4, 4, 0, 0, 0, 0, 1), (4, 8, 0, 0, 0, 0, 0), (8, 8, 0.123456, 0.123456, 0.0, 0.123456, 1),
                (12, 12, 0.123456, 0.123456, 0.123456, 0.0, 0)]


@pytest.mark.parametrize("kind", BACKENDS)
@pytest.mark.parametrize("case", DSLASH_CASES)
def test_dslash_eo_closed_form(request, O, kind, case):
    o = _oracle(request, kind)
    ns, nt, tt, ts, cpr, cpi, even = case
    use_cp = (tt, ts) != (0, 0)
    o.set_lattice(ns, nt, tt, ts, cpr if use_cp else None, cpi if use_cp else None)
    g = o.gauge_fill(True)
    s = o.ascending_complex(o.seo)
    out = o.dslash_eo(s, g, O.EVEN if even else O.ODD, 0.123456)
    ref = closed_form(o.seo, ns, nt, tt, ts, cpr, cpi)
    assert abs(o.count_sf(out) - ref) <= 1e-9 * abs(ref)  # testPrecision 10e-8 %


@pytest.mark.parametrize("kind", BACKENDS)
def test_tm_sitediagonal_per_site(request, O, kind):
    o = _oracle(request, kind)
    o.set_lattice(4, 8)
    s = o.ascending_complex(o.seo)
    k = mu = 0.123456
    mubar = 2 * k * mu
    vals = KATS["tm_sitediagonal_per_site"]["values"]
    for name, which in [("mTmSitediagonal", O.DIAG_M), ("mTmSitediagonalMinus", O.DIAG_M_MINUS),
                        ("mTmInverseSitediagonal", O.DIAG_MINV),
                        ("mTmInverseSitediagonalMinus", O.DIAG_MINV_MINUS)]:
        out = o.tm_diag(s, mubar, which)
        assert abs(o.count_sf(out) - o.seo * vals[name]) <= 1e-9 * o.seo * vals[name], name


EXPLICIT = {"dslash": None, "M_tm_inverse_sitediagonal": "DIAG_MINV", "M_tm_sitediagnoal": "DIAG_M",
            "M_tm_inverse_sitediagonal_minus": "DIAG_MINV_MINUS", "M_tm_sitediagonal_minus": "DIAG_M_MINUS"}


@pytest.mark.parametrize("kind", BACKENDS)
@pytest.mark.parametrize("name", sorted(EXPLICIT))
def test_explicit_physics_kats(request, O, kind, name):
    """physics/fermionmatrix/explicit_test.cpp: 4^3x16, cold links, drand48 sources, kappa .125, mu .006."""
    o = _oracle(request, kind)
    kat = KATS["explicit"][name]
    o.set_lattice(4, kat["nt"])
    g = o.gauge_fill(False)
    src = o.pseudo_randomize(o.vol, kat["seed"])
    sf1, sf2 = o.convert_to_eo(src)
    mubar = 2 * 0.125 * 0.006
    if name == "dslash":
        sf2 = o.dslash_eo(sf1, g, O.EVEN, 0.125)
        a = o.squarenorm(sf2)
        sf1 = o.dslash_eo(sf2, g, O.ODD, 0.125)
    else:
        which = getattr(O, EXPLICIT[name])
        sf2 = o.tm_diag(sf1, mubar, which)
        a = o.squarenorm(sf2)
        sf1 = o.tm_diag(sf2, mubar, which)
    b = o.squarenorm(sf1)
    assert a == pytest.approx(kat["refs"][0], rel=1e-4)  # BOOST_CHECK_CLOSE 0.01 %
    assert b == pytest.approx(kat["refs"][1], rel=1e-4)


FM = {"Aee": "OP_AEE", "Aee_minus": "OP_AEE_MINUS", "Qplus_eo": "OP_QPLUS_EO", "Qminus_eo": "OP_QMINUS_EO",
      "QplusQminus_eo": "OP_QPQM_EO"}


@pytest.mark.parametrize("kind", BACKENDS)
@pytest.mark.parametrize("name", sorted(FM))
def test_fermionmatrix_eo_kats(request, O, kind, name):
    """physics/fermionmatrix/fermionmatrix_test.cpp, first (cold, 4^3x16) block; default action is Wilson."""
    o = _oracle(request, kind)
    kat = KATS["fermionmatrix_eo"][name]
    o.set_lattice(4, 16)
    g = o.gauge_fill(False)
    src = o.pseudo_randomize(o.vol, kat["seed"])
    sf1, sf2 = o.convert_to_eo(src)
    op = getattr(O, FM[name])
    sf2 = o.apply(op, sf1, g, 0.125, 0.0, action=O.WILSON)
    a = o.squarenorm(sf2)
    sf1 = o.apply(op, sf2, g, 0.125, 0.0, action=O.WILSON)
    b = o.squarenorm(sf1)
    assert a == pytest.approx(kat["refs"][0], rel=1e-4)
    assert b == pytest.approx(kat["refs"][1], rel=1e-4)


def test_port_matches_reference_kernels_fixture(port, O):
    """The restated oracle reproduces the committed outputs of the reference's own kernels."""
    d = np.load(os.path.join(GOLD, "ref_outputs.npz"))
    port.set_lattice(4, 4, 1.0, 0.3)
    g = np.zeros((4 * port.vol, 18))
    port.lib.c2qo_pseudo_randomize(g, g.size, int(d["lat4_gauge_seed"][0]))
    s = port.pseudo_randomize(port.seo, int(d["lat4_spinor_seed"][0]))
    assert rel_l2(port.dslash_eo(s, g, O.EVEN, 0.15), d["lat4_dslash_even"]) < 1e-14
    assert rel_l2(port.dslash_eo(s, g, O.ODD, 0.15), d["lat4_dslash_odd"]) < 1e-14
    assert rel_l2(port.apply(O.OP_QPQM_EO, s, g, 0.15, 0.03), d["lat4_qpqm"]) < 1e-14
    assert rel_l2(port.dslash_tm_inv_eo(s, g, O.ODD, 0.15, 0.03), d["lat4_dslash_tminv_odd"]) < 1e-14


@pytest.mark.parametrize("lat", [(4, 4, 1.0, 0.0), (6, 8, 1.0, 0.5), (8, 4, 0.0, 0.0)])
def test_port_vs_reference_random(port, ref, O, lat):
    res = {}
    for o in (port, ref):
        o.set_lattice(*lat)
        g = np.zeros((4 * o.vol, 18))
        o.lib.c2qo_pseudo_randomize(g, g.size, 11)
        s = o.pseudo_randomize(o.seo, 12)
        full = o.pseudo_randomize(o.vol, 13)
        res[o.kind] = [o.dslash_eo(s, g, O.EVEN, 0.16), o.apply(O.OP_QPQM_EO, s, g, 0.16, 0.01),
                       o.apply(O.OP_AEE, s, g, 0.16, 0.01), o.apply(O.OP_QMINUS_EO, s, g, 0.16, 0.01, merged=True),
                       o.m_tm_plus(full, g, 0.16, 0.01), o.m_tm_minus(full, g, 0.16, 0.01),
                       o.saxsbypz(0.3 - 0.2j, s, 1.1 + 0.4j, s * 2, s),
                       np.array([o.scalar_product(s, s * 1.5 + 0.1)])]
    for a, b in zip(res["port"], res["reference"]):
        assert rel_l2(a, b) < 1e-14


def test_oracle_solvers_port_vs_reference(port, ref, O):
    """Same algorithm, same iteration counts and solutions on both oracle builds."""
    out = {}
    for o in (port, ref):
        o.set_lattice(4, 4, 1.0, 0.0)
        g = np.zeros((4 * o.vol, 18))
        o.lib.c2qo_fill_gauge(g, 4 * o.vol, 0)
        g += 0.05 * o.pseudo_randomize(4 * o.vol, 3).reshape(4 * o.vol, 24)[:, :18]
        b = o.pseudo_randomize(o.seo, 5)
        x = np.zeros_like(b)
        P = O.SolverParams(prec=1e-20, cgmax=500, solver=1)
        it_cg = o.cg(x, O.OP_QPQM_EO, b, g, 0.12, 0.02, params=P)
        y = np.zeros_like(b)
        it_bi = o.bicgstab(y, O.OP_AEE, b, g, 0.12, 0.02, params=O.SolverParams(prec=1e-20, cgmax=500))
        z = np.zeros_like(b)
        it_sv = o.bicgstab(z, O.OP_AEE, b, g, 0.12, 0.02, params=O.SolverParams(prec=1e-20, cgmax=500, solver=3))
        out[o.kind] = (it_cg, x, it_bi, y, it_sv, z, o.apply(O.OP_QPQM_EO, x, g, 0.12, 0.02),
                       o.apply(O.OP_AEE, y, g, 0.12, 0.02), b)
    p, r = out["port"], out["reference"]
    assert p[0] == r[0] and p[0] > 0
    assert p[2] == r[2] and p[2] > 0
    assert p[4] == r[4] and p[4] > 0
    assert rel_l2(p[1], r[1]) < 1e-10 and rel_l2(p[3], r[3]) < 1e-10
    b = p[8]
    assert np.linalg.norm(p[6] - b) / np.linalg.norm(b) < 1e-9
    assert np.linalg.norm(p[7] - b) / np.linalg.norm(b) < 1e-9


def test_oracle_inversion_solves_full_system(port, O):
    """perform_inversion (eo) returns -M^{-1} b (the reference's sign conventions, inversion.cpp:165-221)."""
    port.set_lattice(4, 4, 1.0, 0.0)
    g = np.zeros((4 * port.vol, 18))
    port.lib.c2qo_fill_gauge(g, 4 * port.vol, 0)
    src = port.pseudo_randomize(port.vol, 21)
    kappa, mubar = 0.15, 2 * 0.15 * 0.4
    res, it, used_cg = port.perform_inversion_eo(src, g, kappa, mubar, params=O.SolverParams(prec=1e-24))
    assert it >= 0 and not used_cg
    m = port.m_tm_plus(-res, g, kappa, mubar)
    assert rel_l2(m, src) < 1e-10


@pytest.mark.parametrize("kind", BACKENDS)
def test_oracle_reproduces_inverter_integration_reference(request, O, kind):
    """executables/tests/inverter_test_ref with inverter_test_input_1: 4^4 cold gauge field,
    twisted mass kappa 0.15, mu 4, periodic boundaries, the 12 default point sources at
    the origin, eo perform_inversion, pseudoscalar correlator in the default direction
    z (testInverter.py compares at 0.1 %)."""
    ref = KATS["inverter"]["inverter_test_ref"]
    o = _oracle(request, kind)
    ns, nt = int(ref["input"]["nSpace"]), int(ref["input"]["nTime"])
    kappa, mu = float(ref["input"]["kappa"]), float(ref["input"]["mu"])
    o.set_lattice(ns, nt, 0.0, 0.0)
    g = np.zeros((4 * o.vol, 18))
    g[:, 0] = g[:, 8] = g[:, 16] = 1.0  # cold start
    C = np.zeros(nt)
    for k in range(12):
        src = np.zeros((o.vol, 24))
        src[0, 2 * (3 * (k % 4) + k // 4)] = 1.0
        phi, _, _ = o.perform_inversion_eo(src, g, kappa, 2 * kappa * mu, O.TWISTEDMASS,
                                           O.SolverParams(prec=1e-23, cgmax=1000, solver=2))
        # the inverter's default correlator direction is z (meta/parametersObs.cpp:72, correlator_ps_z)
        C += (phi ** 2).sum(axis=1).reshape(nt, ns, ns, ns).sum(axis=(0, 2, 3))
    C *= (2 * kappa) ** 2 / (ns * ns * nt)
    np.testing.assert_allclose(C, ref["ps_correlator"], rtol=ref["tolerance_percent"] / 100)
    np.testing.assert_allclose(C, ref["ps_correlator"], rtol=1e-9)  # far inside the reference's tolerance


def test_oracle_cg_zero_source_is_stuck(port, O):
    """A zero source with a zero start: the reference's CG forms alpha = (r, r) / (p, A p) = 0/0
    in its first iteration and reports the NaN residual as a stuck solver
    (physics/algorithms/solvers/cg.cpp:93-119)."""
    port.set_lattice(4, 4, 1.0, 0.0)
    g = np.zeros((4 * port.vol, 18))
    port.lib.c2qo_fill_gauge(g, 4 * port.vol, 0)
    b = np.zeros_like(port.pseudo_randomize(port.seo, 5))
    x = np.zeros_like(b)
    it = port.cg(x, O.OP_QPQM_EO, b, g, 0.12, 0.02, params=O.SolverParams(prec=1e-20, cgmax=50, solver=1))
    assert it == O.SOLVER_STUCK
