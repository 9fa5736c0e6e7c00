"""GPU: the inverter's measurement path against the reference's integration test.

executables/tests/inverter_test_ref (input inverter_test_input_1): 4^4 cold
gauge field, twisted mass kappa 0.15, mu 4, periodic boundaries, the 12 default
point sources at the origin, eo perform_inversion of each (result kept on the
device), pseudoscalar correlator in t contracted on the GPU.  The reference's
test compares at 0.1 %; the solvers it runs (bicgstab, cg, bicgstab_save) are
all checked here, and the correlator agrees with the oracle to 1e-9.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KATS = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_kats.json")))


@pytest.mark.parametrize("solver", ["bicgstab", "cg", "bicgstab_save"])
def test_ps_correlator_matches_inverter_reference(system, solver):
    import cl2qcd_b200 as c2q
    ref = KATS["inverter"]["inverter_test_ref"]
    ns, nt = int(ref["input"]["nSpace"]), int(ref["input"]["nTime"])
    kappa, mu = float(ref["input"]["kappa"]), float(ref["input"]["mu"])
    L = c2q.Lattice(ns, nt, 0.0, 0.0)
    g = np.zeros((4 * L.vol, 18))
    g[:, 0] = g[:, 8] = g[:, 16] = 1.0  # startCondition=cold
    gf = c2q.Gaugefield(system, L, g)
    params = c2q.SolverParameters(solver=solver, prec=1e-23, cgmax=1000)
    reps = []
    C = c2q.host.inverter_ps_correlator(system, gf, params, c2q.AdditionalParameters.from_mu(kappa, mu),
                                        reports=reps)
    assert len(reps) == 12
    np.testing.assert_allclose(C, ref["ps_correlator"], rtol=ref["tolerance_percent"] / 100)
    np.testing.assert_allclose(C, ref["ps_correlator"], rtol=1e-9)


def test_correlator_kernel_matches_numpy(system):
    """The contraction on random fields: C(t) = (2 kappa)^2 / NS^3 sum |phi|^2 per slice."""
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
    out = np.zeros(L.nt)
    lib = system.lib
    rc = lib.c2q_correlator_ps((C.c_void_p * 3)(*[e.h for e in ev]), (C.c_void_p * 3)(*[o.h for o in od]), 3, 0.13,
                               out)
    assert rc == 0
    expect = sum((f ** 2).sum(axis=1).reshape(L.nt, L.ns ** 3).sum(axis=1) for f in fulls) * (0.26 ** 2) / L.ns ** 3
    np.testing.assert_allclose(out, expect, rtol=1e-13)
