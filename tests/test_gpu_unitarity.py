"""GPU: FP64 unitarity measures and SU(3) projection (project_su3,
ocl_kernel/operations_gaugefield.cl:135-240) of an uploaded field, and solvers
on a field that is not SU(3) to rounding: links rounded to FP32 (as a 32-bit
ILDG file stores them), whose row 2 differs from conj(row0 x row1) by ~1e-7.
With 12-real links asked for, every solver must still report, and stop on, the
true residual of the operator on the links as uploaded, which the oracle
recomputes with its 18-real FP64 operator."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

NS, NT = 8, 16
KAPPA, MUBAR = 0.15, 2 * 0.15 * 0.01


def project_su3(g):
    """numpy restatement of project_su3 on every link of Matrixsu3[4V]."""
    U = (g[:, 0::2] + 1j * g[:, 1::2]).reshape(-1, 3, 3)
    a = U[:, :, 0] / np.linalg.norm(U[:, :, 0], axis=1)[:, None]
    b = U[:, :, 1] - np.sum(a.conj() * U[:, :, 1], axis=1)[:, None] * a
    b /= np.linalg.norm(b, axis=1)[:, None]
    c = np.conj(np.cross(a, b))
    P = np.stack([a, b, c], axis=2).reshape(-1, 9)
    out = np.empty_like(g)
    out[:, 0::2], out[:, 1::2] = P.real, P.imag
    return out


@pytest.fixture(scope="module")
def fields(port):
    port.set_lattice(NS, NT, 1.0, 0.0)
    g = port.gauge_generate(NS, NT, 0.3, 5)
    g32 = g.astype(np.float32).astype(np.float64)
    b = port.source_generate(port.seo, "gaussian", 6)
    return g, g32, b


def test_unitarity_of_su3_and_rounded_fields(system, fields):
    import cl2qcd_b200 as c2q
    g, g32, _ = fields
    L = c2q.Lattice(NS, NT, 1.0, 0.0)
    u = c2q.Gaugefield(system, L, g).unitarity()
    assert max(u.values()) <= 1e-14, u
    u32 = c2q.Gaugefield(system, L, g32).unitarity()
    assert 1e-9 <= u32["unitarity"] <= 1e-6 and 1e-9 <= u32["rec12"] <= 1e-6, u32
    # the same measures in numpy
    U = (g32[:, 0::2] + 1j * g32[:, 1::2]).reshape(-1, 3, 3)
    dev = np.abs(U @ U.conj().transpose(0, 2, 1) - np.eye(3)).max()
    assert abs(dev - u32["unitarity"]) <= 1e-3 * dev
    r12 = np.abs(U[:, 2, :] - np.conj(np.cross(U[:, 0, :], U[:, 1, :]))).max()
    assert abs(r12 - u32["rec12"]) <= 1e-3 * r12
    assert abs(np.abs(np.linalg.det(U) - 1).max() - u32["det"]) <= 1e-3 * u32["det"]


def test_reunitarize_matches_project_su3(system, fields):
    import cl2qcd_b200 as c2q
    _, g32, _ = fields
    L = c2q.Lattice(NS, NT, 1.0, 0.0)
    gf = c2q.Gaugefield(system, L, g32)
    before = gf.reunitarize()
    assert 1e-9 <= before <= 1e-6
    assert max(gf.unitarity().values()) <= 1e-14
    assert np.abs(gf.download() - project_su3(g32)).max() <= 1e-15


def test_non_finite_links_are_reported(system, fields):
    import cl2qcd_b200 as c2q
    g, _, _ = fields
    bad = g.copy()
    bad[123, 4] = np.nan
    L = c2q.Lattice(NS, NT, 1.0, 0.0)
    gf = c2q.Gaugefield(system, L, bad)
    assert np.isinf(gf.unitarity()["unitarity"])
    with pytest.raises(Exception):
        gf.reunitarize()


@pytest.mark.parametrize("precision", [64, 32, 16])
def test_cg_rec12_on_non_unitary_field_reports_uploaded_operator(port, O, system, fields, precision):
    import cl2qcd_b200 as c2q
    _, g32, b = fields
    port.set_lattice(NS, NT, 1.0, 0.0)
    L = c2q.Lattice(NS, NT, 1.0, 0.0)
    gf = c2q.Gaugefield(system, L, g32)
    X, B = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L, b)
    rep = {}
    c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, B,
                c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=20000, precision=precision,
                                     use_rec12=True), c2q.AdditionalParameters(KAPPA, MUBAR), rep)
    r = port.apply(O.OP_QPQM_EO, X.dump(), g32, KAPPA, MUBAR) - b
    oracle_rel = np.linalg.norm(r) / np.linalg.norm(b)
    assert oracle_rel <= 1e-10 * (1 + 1e-6), (oracle_rel, rep)
    assert abs(oracle_rel - rep["true_resid_rel"]) <= 1e-3 * oracle_rel, (oracle_rel, rep)


@pytest.mark.parametrize("precision", [32, 16])
def test_bicgstab_rec12_on_non_unitary_field_reports_uploaded_operator(port, O, system, fields, precision):
    import cl2qcd_b200 as c2q
    _, g32, b = fields
    port.set_lattice(NS, NT, 1.0, 0.0)
    L = c2q.Lattice(NS, NT, 1.0, 0.0)
    gf = c2q.Gaugefield(system, L, g32)
    kappa, mubar = 0.12, 2 * 0.12 * 0.01
    X, B = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L, b)
    rep = {}
    c2q.host.bicgstab(X, c2q.host.Aee(), gf, B,
                      c2q.SolverParameters(solver="bicgstab", prec=0.0, rel_tol=1e-10, cgmax=5000,
                                           precision=precision, use_rec12=True),
                      c2q.AdditionalParameters(kappa, mubar), rep)
    r = port.apply(O.OP_AEE, X.dump(), g32, kappa, mubar) - b
    oracle_rel = np.linalg.norm(r) / np.linalg.norm(b)
    assert oracle_rel <= 1e-10 * (1 + 1e-6), (oracle_rel, rep)
    assert abs(oracle_rel - rep["true_resid_rel"]) <= 1e-3 * oracle_rel, (oracle_rel, rep)


def test_rec12_exact_field_solves_agree(port, O, system, fields):
    """On an SU(3) field the 12-real and 18-real mixed solves reach the same solution."""
    import cl2qcd_b200 as c2q
    g, _, b = fields
    L = c2q.Lattice(NS, NT, 1.0, 0.0)
    gf = c2q.Gaugefield(system, L, g)
    B = c2q.Spinorfield_eo(system, L, b)
    xs = []
    for rec12 in (False, True):
        X = c2q.Spinorfield_eo(system, L)
        c2q.host.cg(X, c2q.host.QplusQminus_eo(), gf, B,
                    c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=20000, precision=16,
                                         use_rec12=rec12), c2q.AdditionalParameters(KAPPA, MUBAR))
        xs.append(X.dump())
    assert rel_l2(xs[1], xs[0]) <= 1e-8
