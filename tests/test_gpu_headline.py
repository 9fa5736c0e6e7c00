"""GPU parity at the sizes the performance is quoted on, against the reference's
own kernels compiled as C (the oracle; its restatement where that build is
absent).

* 32^3x64 (1,048,576 eo sites), the benchmark workload: seeded U = exp(i 0.25 H)
  links, one Gaussian source, kappa 0.16, mu 0.005, antiperiodic T.  FP64
  dslash_eo on both parities with 18- and 12-real links, the fused dslash +
  M_tm^-1, Aee and QplusQminus_eo (<= 1e-12 relative L2); the FP32 / FP16
  paired-site sweeps within their storage rounding (which exercises the slot
  fold at t = NT/2 at NT = 64); the mixed-precision CG solutions (FP16 and FP32
  inner, 12-real links, temporal gauge with lambda = c^64) with their true
  residual recomputed by the oracle's 18-real operator; the FP64 CG with the
  reference's stopping test needing exactly the iterations the reference's CG
  needed on this workload (oracle/workload_fp64_cg.json).
* 64^3x128 (16,777,216 eo sites, 19.3 GB of FP64 links): one FP64 dslash_eo
  sweep, and the mixed FP16 CG at kappa 0.1625, mu 0.003, eps 0.2 with its
  true residual recomputed by the oracle (lambda = c^128, 32-bit site indices
  near their largest values).

The inputs come from the oracle's own generators, which the CPU tests show to
be bit-identical to the library's.
"""
import json
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NS, NT, EPS, KAPPA, MU = 32, 64, 0.25, 0.16, 0.005
GAUGE_SEED, SOURCE_SEED = 20250, 777
MUBAR = 2 * KAPPA * MU


@pytest.fixture(scope="module")
def oc(O):
    """The checker: the reference's kernels where they were built, else the restatement."""
    return O.Oracle("reference" if O.available("reference") else "port")


@pytest.fixture(scope="module")
def w32(oc, system):
    import cl2qcd_b200 as c2q
    oc.set_lattice(NS, NT, 1.0, 0.0)
    g = oc.gauge_generate(NS, NT, EPS, GAUGE_SEED)
    b = oc.source_generate(oc.seo, "gaussian", SOURCE_SEED)
    L = c2q.Lattice(NS, NT, 1.0, 0.0)
    gf = c2q.Gaugefield(system, L, g)
    yield {"L": L, "g": g, "b": b, "gf": gf}
    system.set_link_format(False)
    del gf


def _at32(oc):
    oc.set_lattice(NS, NT, 1.0, 0.0)


@pytest.mark.parametrize("rec12", [False, True])
@pytest.mark.parametrize("evenodd", [0, 1])
def test_fp64_dslash_32c64(oc, system, w32, evenodd, rec12):
    import cl2qcd_b200 as c2q
    _at32(oc)
    ref = oc.dslash_eo(w32["b"], w32["g"], evenodd, KAPPA)
    system.set_link_format(rec12)
    try:
        a, out = c2q.Spinorfield_eo(system, w32["L"], w32["b"]), c2q.Spinorfield_eo(system, w32["L"])
        c2q.host.dslash(out, w32["gf"], a, evenodd, KAPPA)
        err = rel_l2(out.dump(), ref)
    finally:
        system.set_link_format(False)
    assert err <= 1e-12, err


@pytest.mark.parametrize("evenodd", [0, 1])
def test_fp64_dslash_tm_inverse_32c64(oc, system, w32, evenodd):
    import cl2qcd_b200 as c2q
    _at32(oc)
    ref = oc.dslash_tm_inv_eo(w32["b"], w32["g"], evenodd, KAPPA, MUBAR)
    a, out = c2q.Spinorfield_eo(system, w32["L"], w32["b"]), c2q.Spinorfield_eo(system, w32["L"])
    c2q.host.dslash_AND_M_tm_inverse_sitediagonal(out, w32["gf"], a, evenodd, KAPPA, MUBAR)
    assert rel_l2(out.dump(), ref) <= 1e-12


@pytest.mark.parametrize("name", ["Aee", "QplusQminus_eo"])
def test_fp64_fermionmatrix_32c64(oc, O, system, w32, name):
    import cl2qcd_b200 as c2q
    _at32(oc)
    op = {"Aee": O.OP_AEE, "QplusQminus_eo": O.OP_QPQM_EO}[name]
    ref = oc.apply(op, w32["b"], w32["g"], KAPPA, MUBAR)
    a, out = c2q.Spinorfield_eo(system, w32["L"], w32["b"]), c2q.Spinorfield_eo(system, w32["L"])
    getattr(c2q.host, name)()(out, w32["gf"], a, c2q.AdditionalParameters(KAPPA, MUBAR))
    assert rel_l2(out.dump(), ref) <= 1e-12


@pytest.mark.parametrize("precision,rec12,tol", [(32, False, 2e-6), (32, True, 2e-6), (16, True, 2e-4)])
@pytest.mark.parametrize("evenodd", [0, 1])
def test_reduced_precision_dslash_32c64(oc, system, w32, precision, rec12, tol, evenodd):
    """The paired-site sweeps against the FP64 oracle, within the storage rounding
    (FP32 spinors and links; FP16 fixed-point spinors with a per-site norm and
    FP16 12-real links)."""
    import cl2qcd_b200 as c2q
    _at32(oc)
    ref = oc.dslash_eo(w32["b"], w32["g"], evenodd, KAPPA)
    system.set_link_format(rec12)
    try:
        a = c2q.Spinorfield_eo(system, w32["L"], w32["b"], precision=precision)
        out = c2q.Spinorfield_eo(system, w32["L"], precision=precision)
        c2q.host.dslash(out, w32["gf"], a, evenodd, KAPPA)
        err = rel_l2(out.dump(), ref)
    finally:
        system.set_link_format(False)
    assert err <= tol, err


@pytest.mark.parametrize("precision", [16, 32])
def test_mixed_cg_32c64_true_residual_by_oracle(oc, O, system, w32, precision):
    """The headline solver: mixed-precision CG with 12-real links and the
    temporal gauge; the oracle recomputes ||b - A x|| / ||b|| with its 18-real
    FP64 operator, and the solver's own report agrees with it."""
    import cl2qcd_b200 as c2q
    _at32(oc)
    X, B = c2q.Spinorfield_eo(system, w32["L"]), c2q.Spinorfield_eo(system, w32["L"], w32["b"])
    rep = {}
    c2q.host.cg(X, c2q.host.QplusQminus_eo(), w32["gf"], B,
                c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=40000, precision=precision,
                                     use_rec12=True), c2q.AdditionalParameters(KAPPA, MUBAR), rep)
    b = w32["b"]
    r = oc.apply(O.OP_QPQM_EO, X.dump(), w32["g"], KAPPA, MUBAR) - b
    oracle_rel = np.linalg.norm(r) / np.linalg.norm(b)
    assert oracle_rel <= 1.0e-10 * (1 + 1e-6), (oracle_rel, rep)
    assert abs(oracle_rel - rep["true_resid_rel"]) <= 1e-3 * oracle_rel, (oracle_rel, rep)


def test_fp64_cg_iterations_match_reference_32c64(system, w32):
    """The reference's stopping test (|r|^2 < (1e-10)^2 |b|^2, checked every 10
    iterations, refresh every 100): the library's FP64 CG performs exactly the
    iterations the reference's CG on its own kernels performed on this workload."""
    import cl2qcd_b200 as c2q
    rec = json.load(open(os.path.join(ROOT, "oracle", "workload_fp64_cg.json")))
    w = rec["workload"]
    assert (w["ns"], w["nt"], w["eps"], w["kappa"], w["mu"], w["gauge_seed"], w["source_seed"]) == \
        (NS, NT, EPS, KAPPA, MU, GAUGE_SEED, SOURCE_SEED)
    b = w32["b"]
    X, B = c2q.Spinorfield_eo(system, w32["L"]), c2q.Spinorfield_eo(system, w32["L"], b)
    rep = {}
    ret = c2q.host.cg(X, c2q.host.QplusQminus_eo(), w32["gf"], B,
                      c2q.SolverParameters(solver="cg", prec=1e-20 * float((b * b).sum()), cgmax=10000,
                                           precision=64), c2q.AdditionalParameters(KAPPA, MUBAR), rep)
    assert ret == rec["cg_returned"], (ret, rec)
    assert abs(rep["true_resid_rel"] - rec["true_resid_rel"]) <= 1e-3 * rec["true_resid_rel"]


# ---------------------------------------------------------------- 64^3 x 128
@pytest.fixture(scope="module")
def w64(oc, system):
    import cl2qcd_b200 as c2q
    ns, nt = 64, 128
    oc.set_lattice(ns, nt, 1.0, 0.0)
    g = oc.gauge_generate(ns, nt, 0.2, 64128)
    b = oc.source_generate(oc.seo, "gaussian", 128)
    L = c2q.Lattice(ns, nt, 1.0, 0.0)
    gf = c2q.Gaugefield(system, L, g)
    yield {"L": L, "g": g, "b": b, "gf": gf, "ns": ns, "nt": nt}
    del gf


def test_fp64_dslash_64c128(oc, system, w64):
    import cl2qcd_b200 as c2q
    oc.set_lattice(w64["ns"], w64["nt"], 1.0, 0.0)
    ref = oc.dslash_eo(w64["b"], w64["g"], 1, 0.1625)
    a, out = c2q.Spinorfield_eo(system, w64["L"], w64["b"]), c2q.Spinorfield_eo(system, w64["L"])
    c2q.host.dslash(out, w64["gf"], a, 1, 0.1625)
    assert rel_l2(out.dump(), ref) <= 1e-12


def test_mixed_cg_64c128_true_residual_by_oracle(oc, O, system, w64):
    import cl2qcd_b200 as c2q
    kappa, mubar = 0.1625, 2 * 0.1625 * 0.003
    X, B = c2q.Spinorfield_eo(system, w64["L"]), c2q.Spinorfield_eo(system, w64["L"], w64["b"])
    rep = {}
    c2q.host.cg(X, c2q.host.QplusQminus_eo(), w64["gf"], B,
                c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=40000, precision=16,
                                     use_rec12=True), c2q.AdditionalParameters(kappa, mubar), rep)
    oc.set_lattice(w64["ns"], w64["nt"], 1.0, 0.0)
    b = w64["b"]
    r = oc.apply(O.OP_QPQM_EO, X.dump(), w64["g"], kappa, mubar)
    r -= b
    oracle_rel = np.linalg.norm(r) / np.linalg.norm(b)
    assert oracle_rel <= 1.0e-10 * (1 + 1e-6), (oracle_rel, rep)
    assert abs(oracle_rel - rep["true_resid_rel"]) <= 1e-3 * oracle_rel, (oracle_rel, rep)
