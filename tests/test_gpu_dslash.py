"""GPU parity of the dslash_eo family against the oracle (relative L2 <= 1e-12 in FP64)."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

LATTICES = [(4, 4, 0.0, 0.0, None, None), (8, 8, 1.0, 0.0, None, None), (6, 8, 1.0, 0.3, None, None),
            (8, 4, 0.7, 0.2, 0.1, 0.2), (4, 12, 1.0, 0.0, None, 0.3), (10, 6, 0.0, 1.0, 0.05, None)]


def setup(port, c2q, system, lat, seed=1, unitary=True):
    ns, nt, tt, ts, cpr, cpi = lat
    port.set_lattice(ns, nt, tt, ts, cpr, cpi)
    L = c2q.Lattice(ns, nt, tt, ts, cpr, cpi)
    if unitary:
        g = c2q.host.generate_gaugefield(L, 0.3, seed)
    else:
        g = np.zeros((4 * port.vol, 18))
        port.lib.c2qo_pseudo_randomize(g, g.size, seed)
    gf = c2q.Gaugefield(system, L, g)
    return L, g, gf


@pytest.mark.parametrize("lat", LATTICES)
@pytest.mark.parametrize("evenodd", [0, 1])
def test_dslash_eo_matches_oracle(port, system, O, lat, evenodd):
    import cl2qcd_b200 as c2q
    L, g, gf = setup(port, c2q, system, lat, unitary=False)
    s = port.pseudo_randomize(port.seo, 5)
    ref = port.dslash_eo(s, g, evenodd, 0.1573)
    a, b = c2q.Spinorfield_eo(system, L, s), c2q.Spinorfield_eo(system, L)
    c2q.host.dslash(b, gf, a, evenodd, 0.1573)
    assert rel_l2(b.dump(), ref) <= 1e-12


@pytest.mark.parametrize("lat", LATTICES[:3])
@pytest.mark.parametrize("minus", [False, True])
def test_dslash_AND_M_tm_inverse_sitediagonal(port, system, O, lat, minus):
    import cl2qcd_b200 as c2q
    L, g, gf = setup(port, c2q, system, lat)
    s = port.pseudo_randomize(port.seo, 6)
    for evenodd in (0, 1):
        ref = port.dslash_tm_inv_eo(s, g, evenodd, 0.16, 0.0016, minus)
        a, b = c2q.Spinorfield_eo(system, L, s), c2q.Spinorfield_eo(system, L)
        c2q.host.dslash_AND_M_tm_inverse_sitediagonal(b, gf, a, evenodd, 0.16, 0.0016, minus)
        assert rel_l2(b.dump(), ref) <= 1e-12


def test_dslash_closed_form_kat(system, O, port):
    """hardware/code/fermions_test.cpp DSLASH_EO_BC_AND_CHEMPOT_1 through the CUDA path."""
    import cl2qcd_b200 as c2q
    import json, math, os
    kats = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))
    c = kats["dslash_eo_closed_form"]["coefficients"]
    ns = nt = 8
    th = cpi = 0.123456
    L = c2q.Lattice(ns, nt, th, th, 0.0, cpi)
    port.set_lattice(ns, nt)
    gf = c2q.Gaugefield(system, L, port.gauge_fill(True))
    s = port.ascending_complex(port.seo)
    a, b = c2q.Spinorfield_eo(system, L, s), c2q.Spinorfield_eo(system, L)
    c2q.host.dslash(b, gf, a, 0, 0.123456)
    aS, aT = math.pi * th / ns, cpi + math.pi * th / nt
    ref = port.seo * (c[0] * math.cos(aS) + c[1] * math.cos(aT) + c[2] * math.sin(aS) + c[3] * math.sin(aT))
    assert abs(b.dump().sum() - ref) <= 1e-9 * abs(ref)


@pytest.mark.parametrize("lat", LATTICES[:4])
def test_rec12_matches_18real(port, system, O, lat):
    """12-real links (row 2 = conj(row0 x row1)) give the 18-real result on SU(3) fields."""
    import cl2qcd_b200 as c2q
    L, g, gf = setup(port, c2q, system, lat)
    b = port.pseudo_randomize(port.seo, 9)
    x64, x12 = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L)
    bb = c2q.Spinorfield_eo(system, L, b)
    add = c2q.AdditionalParameters(0.13, 0.01)
    A = c2q.host.QplusQminus_eo()
    r1, r2 = {}, {}
    c2q.host.cg(x64, A, gf, bb, c2q.SolverParameters(solver="cg", prec=0, rel_tol=1e-11, cgmax=2000), add, r1)
    c2q.host.cg(x12, A, gf, bb, c2q.SolverParameters(solver="cg", prec=0, rel_tol=1e-11, cgmax=2000,
                                                     use_rec12=True), add, r2)
    assert r2["true_resid_rel"] <= 1e-11
    assert rel_l2(x12.dump(), x64.dump()) < 1e-9


RP_LATTICES = [(4, 4, 0.0, 0.0, None, None), (8, 8, 1.0, 0.0, None, None), (6, 8, 1.0, 0.3, None, None),
               (8, 4, 0.7, 0.2, 0.1, 0.2), (4, 12, 1.0, 0.0, None, 0.3)]


@pytest.mark.parametrize("lat", RP_LATTICES)
@pytest.mark.parametrize("precision,rec12", [(32, False), (32, True), (16, True), (16, False)])
def test_reduced_precision_operators_match_oracle(port, system, O, lat, precision, rec12):
    """The FP32 / FP16 paired-site sweeps against the FP64 oracle: the dslash on
    both parities, the fused dslash + M_tm^{-1}, and Q+Q- (all four fused sweep
    kinds).  Bound: a few units of the storage rounding (FP32 2^-24, FP16 fixed
    point 2^-15 relative to the site norm) amplified by the stencil."""
    import cl2qcd_b200 as c2q
    tol = {32: 2e-6, 16: 2e-4}[precision]
    L, g, gf = setup(port, c2q, system, lat)
    system.set_link_format(rec12)
    try:
        s = port.pseudo_randomize(port.seo, 7)
        a = c2q.Spinorfield_eo(system, L, s, precision=precision)
        b = c2q.Spinorfield_eo(system, L, precision=precision)
        for evenodd in (0, 1):
            ref = port.dslash_eo(s, g, evenodd, 0.1573)
            c2q.host.dslash(b, gf, a, evenodd, 0.1573)
            assert rel_l2(b.dump(), ref) <= tol, ("dslash", evenodd)
            ref = port.dslash_tm_inv_eo(s, g, evenodd, 0.16, 0.0016, False)
            c2q.host.dslash_AND_M_tm_inverse_sitediagonal(b, gf, a, evenodd, 0.16, 0.0016, False)
            assert rel_l2(b.dump(), ref) <= tol, ("dslash_tm_inv", evenodd)
        ref = port.apply(O.OP_QPQM_EO, s, g, 0.16, 0.0016)
        c2q.host.QplusQminus_eo()(b, gf, a, c2q.AdditionalParameters(0.16, 0.0016))
        assert rel_l2(b.dump(), ref) <= 4 * tol, "QplusQminus_eo"
        # round trip of the storage itself
        assert rel_l2(a.dump(), s) <= tol / 4
    finally:
        system.set_link_format(False)


def test_reduced_precision_needs_nt_multiple_of_4(system):
    import cl2qcd_b200 as c2q
    with pytest.raises(c2q.InvalidParameters):
        c2q.Spinorfield_eo(system, c2q.Lattice(4, 6), precision=16)
