"""GPU: the inverter's measurement path against the reference's integration tests.

executables/tests/inverter_test_ref (inverter_test_input_1: 4^4 cold gauge field)
and inverter_test_ref2 (inverter_test_input_2: the ILDG configuration
conf.00200, decoded by this project's reader into tests/golden/conf00200.npz):
twisted mass kappa 0.15, mu 4, periodic boundaries, the 12 default point sources
at the origin, eo perform_inversion of each (result kept on the device), the
pseudoscalar correlator along z (the reference's default direction) contracted on
the GPU.  The reference's test compares at 0.1 %; the solvers it runs
(bicgstab, cg, bicgstab_save), each with useEO true and false (the
full-lattice solve of inversion.cpp:98-122) as its CMakeLists registers them,
are all checked here, at 1e-9.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KATS = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_kats.json")))


@pytest.mark.parametrize("use_eo", [True, False])
@pytest.mark.parametrize("solver", ["bicgstab", "cg", "bicgstab_save"])
@pytest.mark.parametrize("name", ["inverter_test_ref", "inverter_test_ref2"])
def test_ps_correlator_matches_inverter_reference(system, solver, name, use_eo):
    import cl2qcd_b200 as c2q
    ref = KATS["inverter"][name]
    ns, nt = int(ref["input"]["nSpace"]), int(ref["input"]["nTime"])
    kappa, mu = float(ref["input"]["kappa"]), float(ref["input"]["mu"])
    L = c2q.Lattice(ns, nt, 0.0, 0.0)
    if ref["input"]["startCondition"] == "cold":
        g = np.zeros((4 * L.vol, 18))
        g[:, 0] = g[:, 8] = g[:, 16] = 1.0
    else:  # initialConf=conf.00200
        g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "conf00200.npz"))["gauge"]
    gf = c2q.Gaugefield(system, L, g)
    params = c2q.SolverParameters(solver=solver, prec=1e-23, cgmax=1000)
    reps = []
    C = c2q.host.inverter_ps_correlator(system, gf, params, c2q.AdditionalParameters.from_mu(kappa, mu),
                                        reports=reps, use_eo=use_eo)
    assert len(reps) == 12
    np.testing.assert_allclose(C, ref["ps_correlator"], rtol=ref["tolerance_percent"] / 100)
    np.testing.assert_allclose(C, ref["ps_correlator"], rtol=1e-9)


def test_correlator_kernel_matches_numpy(system):
    """The contraction on random fields, along t and along z."""
    import cl2qcd_b200 as c2q
    L = c2q.Lattice(6, 8, 0.0, 0.0)
    rng = np.random.default_rng(5)
    fulls = [rng.standard_normal((L.vol, 24)) for _ in range(3)]
    ev, od = [], []
    for f in fulls:
        e, o = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L)
        c2q.host.convert_to_eoprec(e, o, f)
        ev.append(e)
        od.append(o)
    import ctypes as C
    lib = system.lib
    ae, ao = (C.c_void_p * 3)(*[e.h for e in ev]), (C.c_void_p * 3)(*[o.h for o in od])
    out = np.zeros(L.nt)
    assert lib.c2q_correlator_ps(ae, ao, 3, 0.13, 0, out) == 0
    n2 = [(f ** 2).sum(axis=1).reshape(L.nt, L.ns, L.ns, L.ns) for f in fulls]  # [t][z][y][x]
    expect = sum(a.sum(axis=(1, 2, 3)) for a in n2) * (0.26 ** 2) / L.ns ** 3
    np.testing.assert_allclose(out, expect, rtol=1e-13)
    out = np.zeros(L.ns)
    assert lib.c2q_correlator_ps(ae, ao, 3, 0.13, 3, out) == 0
    expect = sum(a.sum(axis=(0, 2, 3)) for a in n2) * (0.26 ** 2) / (L.ns ** 2 * L.nt)
    np.testing.assert_allclose(out, expect, rtol=1e-13)


FM = {"Aee": "OP_AEE", "Aee_minus": "OP_AEE_MINUS", "Qplus_eo": "OP_QPLUS_EO", "Qminus_eo": "OP_QMINUS_EO",
      "QplusQminus_eo": "OP_QPLUSQMINUS_EO"}


@pytest.mark.parametrize("name", sorted(FM))
def test_fermionmatrix_eo_kats_on_conf00200(system, port, name):
    """physics/fermionmatrix/fermionmatrix_test.cpp, second block (conf.00200, nTime 4,
    Wilson, kappa 0.125) through the GPU's c2q_apply_eo, at the reference's 0.01 %."""
    import cl2qcd_b200 as c2q
    from cl2qcd_b200 import _lib as L
    kat = KATS["fermionmatrix_eo"][name]
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "conf00200.npz"))["gauge"]
    port.set_lattice(4, 4)
    Lat = c2q.Lattice(4, 4)
    gf = c2q.Gaugefield(system, Lat, g)
    src = port.pseudo_randomize(port.vol, kat["seed"])
    e, o = port.convert_to_eo(src)
    sf1, sf2 = c2q.Spinorfield_eo(system, Lat, e), c2q.Spinorfield_eo(system, Lat, o)
    op = getattr(L, FM[name])
    lib = system.lib
    assert lib.c2q_apply_eo(op, sf2.h, gf.h, sf1.h, 0.125, 0.0, L.WILSON, 0) == 0
    assert c2q.host.squarenorm(sf2) == pytest.approx(kat["refs"][2], rel=1e-4)
    assert lib.c2q_apply_eo(op, sf1.h, gf.h, sf2.h, 0.125, 0.0, L.WILSON, 0) == 0
    assert c2q.host.squarenorm(sf1) == pytest.approx(kat["refs"][3], rel=1e-4)
