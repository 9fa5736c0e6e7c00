"""GPU: the temporal gauge of the mixed-precision inner solves.

The mixed-precision CG on QplusQminus_eo runs its inner iterations on the
gauge field transformed to the temporal gauge: every T link becomes the
identity except the one leaving the last time slice, and the T phases move
into the transformation.  The inner operator is unitarily equivalent to the
original one, so a solve with it must meet the same true FP64 residual bar on
the original field (checked with the oracle's operator) in about as many
iterations as without it, for every boundary condition that allows it
(antiperiodic, periodic and twisted T, an imaginary chemical potential).
With complex spatial phases it does not apply and the solver keeps the plain
inner sweeps (no transformed copy of the links is built).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    "antiperiodic": dict(theta_t=1.0, theta_s=0.0),
    "periodic": dict(theta_t=0.0, theta_s=0.0),
    "twisted_t": dict(theta_t=0.5, theta_s=0.0),
    "imaginary_cp": dict(theta_t=1.0, theta_s=0.0, cp_im=0.3),
    "spatial_phase": dict(theta_t=1.0, theta_s=0.5),
}


def _params(c2q, precision, tg, graph=False):
    return c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=5000, precision=precision,
                                use_rec12=True, use_graph=graph, temporal_gauge=tg)


@pytest.mark.parametrize("precision", [32, 16])
@pytest.mark.parametrize("case", sorted(CASES))
def test_solve_in_temporal_gauge(port, system, O, precision, case):
    import cl2qcd_b200 as c2q
    bc = CASES[case]
    ns, nt = 8, 8
    port.set_lattice(ns, nt, bc["theta_t"], bc["theta_s"], None, bc.get("cp_im"))
    L = c2q.Lattice(ns, nt, bc["theta_t"], bc["theta_s"], None, bc.get("cp_im"))
    g = c2q.host.generate_gaugefield(L, 0.3, 5)
    kappa, mubar = 0.15, 2 * 0.15 * 0.01
    add = c2q.AdditionalParameters(kappa, mubar)
    A = c2q.host.QplusQminus_eo()
    src = c2q.host.generate_source(L.seo, "gaussian", 21)
    out = {}
    for tg in (False, True):
        gf = c2q.Gaugefield(system, L, g)
        b = c2q.Spinorfield_eo(system, L, src)
        x = c2q.Spinorfield_eo(system, L)
        rep = {}
        before = gf.device_bytes
        c2q.host.cg(x, A, gf, b, _params(c2q, precision, tg), add, rep)
        grew = gf.device_bytes - before
        assert rep["true_resid_rel"] <= 1e-10, (tg, rep)
        r = port.apply(O.OP_QPQM_EO, x.dump(), g, kappa, mubar)
        assert np.linalg.norm(r - src) / np.linalg.norm(src) <= 1.5e-10
        out[tg] = (x.dump(), rep, grew)
    plain, tgd = out[False], out[True]
    if case == "spatial_phase":  # not applicable: the same sweeps, the same result
        assert tgd[2] == plain[2]
        assert tgd[1]["iterations"] == plain[1]["iterations"]
        assert np.array_equal(tgd[0], plain[0])
        return
    # the transformation (V FP64 3x3 complex matrices) was built, and the transformed
    # inner links in place of the plain ones
    assert tgd[2] >= plain[2] + ns ** 3 * nt * 144
    it0, it1 = plain[1]["iterations"], tgd[1]["iterations"]
    assert abs(it1 - it0) <= max(3, 0.05 * it0), (it0, it1)
    d = np.linalg.norm(tgd[0] - plain[0]) / np.linalg.norm(plain[0])
    assert d <= 1e-8, d


@pytest.mark.parametrize("precision", [32, 16])
def test_batch_in_temporal_gauge_matches_single(port, system, O, precision):
    """A batch of four sources in the temporal gauge (graph-captured) gives each
    source the result it gets alone."""
    import cl2qcd_b200 as c2q
    ns, nt = 8, 8
    port.set_lattice(ns, nt, 1.0, 0.0)
    L = c2q.Lattice(ns, nt, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, 0.25, 9)
    gf = c2q.Gaugefield(system, L, g)
    kappa, mubar = 0.16, 2 * 0.16 * 0.005
    add = c2q.AdditionalParameters(kappa, mubar)
    A = c2q.host.QplusQminus_eo()
    srcs = [c2q.host.generate_source(L.seo, "z2", 40 + k) for k in range(4)]
    bs = [c2q.Spinorfield_eo(system, L, s) for s in srcs]
    xs = [c2q.Spinorfield_eo(system, L) for _ in srcs]
    reps = []
    c2q.host.cg_multi(xs, A, gf, bs, _params(c2q, precision, True, graph=True), add, reps)
    for k, s in enumerate(srcs):
        assert reps[k]["true_resid_rel"] <= 1e-10, (k, reps[k])
        r = port.apply(O.OP_QPQM_EO, xs[k].dump(), g, kappa, mubar)
        assert np.linalg.norm(r - s) / np.linalg.norm(s) <= 1.5e-10
        x1 = c2q.Spinorfield_eo(system, L)
        rep1 = {}
        c2q.host.cg(x1, A, gf, bs[k], _params(c2q, precision, True), add, rep1)
        assert rep1["iterations"] == reps[k]["iterations"]
        d = np.linalg.norm(x1.dump() - xs[k].dump()) / np.linalg.norm(x1.dump())
        assert d <= 1e-12, (k, d)
