"""Known answers of the reference's eo BLAS and merged-kernel tests:
hardware/code/spinors_test.cpp (GLOBAL_SQUARENORM_EO, SCALAR_PRODUCT_EO, ZERO_EO,
COLD_EO, SAX_EO, SAXPY_EO, SAXSBYPZ_EO, CONVERT_EO),
hardware/code/fermions_merged_kernels_test.cpp (dslash_AND_M_tm_inverse_sitediagonal
(_minus), M_tm_sitediagonal(_minus)_AND_gamma5_eo, saxpy_AND_gamma5_eo) and
hardware/code/spinors_merged_kernels_test.cpp (saxpy_AND_squarenorm_eo), as
extracted into tests/golden/reference_kats.json by tests/golden/make_fixtures.py.

Each case fills its fields as the reference's test harness does (one:
every component 1; ascendingComplex: component k = (2k+1) + (2k+2) i) and
compares the same quantity (the squarenorm, the scalar product, or the sum of
all reals of the output field) at the reference's 1e-9 relative tolerance:
through both oracle builds on the CPU, and through the library's C ABI on the
GPU."""
import json
import os

import numpy as np
import pytest

KATS = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                   "reference_kats.json")))["blas_and_merged_eo"]
SPIN = KATS["spinors_eo"]
MERGED = KATS["merged_eo"]
TOL = 1e-9


def _fill(kind, n):
    a = np.zeros((n, 24))
    if kind == "one":
        a[:, 0::2] = 1.0
    elif kind == "ascendingComplex":
        a[:] = np.arange(1, 25, dtype=float)
    else:
        raise ValueError(kind)
    return a


def _close(got, want):
    scale = max(abs(want), 1.0)
    return abs(got - want) <= TOL * scale


def _parity_full(ns, nt, even):
    """a full field with every component (1, 0) on the sites of one parity (x+y+z+t even or odd)"""
    t, z, y, x = np.meshgrid(np.arange(nt), np.arange(ns), np.arange(ns), np.arange(ns), indexing="ij")
    par = ((x + y + z + t) % 2 == 0).reshape(-1)
    full = np.zeros((ns ** 3 * nt, 24))
    full[par == even, 0::2] = 1.0
    return full


# ------------------------------------------------------------------ CPU: the oracle
def _spin_oracle(o, c):
    o.set_lattice(c["ns"], c["nt"])
    n = o.seo
    f = [_fill(k, n) for k in c.get("fills") or ["ascendingComplex"]]
    t = c["test"]
    if t == "testEvenOddSquarenorm":
        return [o.squarenorm(f[0])]
    if t == "testEvenOddScalarProduct":
        z = o.scalar_product(f[0], f[1])
        return [z.real, z.imag]
    if t == "testEvenOddZero":
        return [o.squarenorm(o.eo_field())]
    if t == "testEvenOddCold":
        return [o.squarenorm(o.cold_eo())]
    a = [complex(*x) for x in c.get("coefficients", [])]
    x = f[0]
    if t == "testEvenOddSax":
        return [o.squarenorm(o.sax(a[0], x))]
    if t in ("testEvenOddSaxpy", "testEvenOddSaxpyArg"):
        return [o.squarenorm(o.saxpy(a[0], x, x))]
    if t == "testSaxsbypzEvenOdd":
        return [o.squarenorm(o.saxsbypz(a[0], x, a[1], x, x))]
    if t == "testConvertToEvenOdd":
        e, od = o.convert_to_eo(_parity_full(c["ns"], c["nt"], c["fill_even_sites"]))
        return [o.squarenorm(e), o.squarenorm(od)]
    raise ValueError(t)


def _merged_oracle(o, O, c):
    o.set_lattice(c["ns"], c["nt"])
    x = _fill(c["fills"][0], o.seo)
    t = c["test"]
    if t == "testSaxpyAndSquarenormEvenOdd":
        _, n = o.saxpy_squarenorm(complex(*c["coefficient"]), x, x)
        return n
    if t == "testSaxpyAndGamma5EvenOdd":
        return o.count_sf(o.saxpy_gamma5(complex(*c["coefficient"]), x, _fill(c["fills"][1], o.seo)))
    mubar = 2 * c["kappa"] * c["mu"]
    if t == "testMTmSitediagonalAndGamma5EvenOdd":
        return o.count_sf(o.tm_diag(x, mubar, O.DIAG_M_G5))
    if t == "testMTmSitediagonalMinusAndGamma5EvenOdd":
        return o.count_sf(o.tm_diag(x, mubar, O.DIAG_M_MINUS_G5))
    g = o.gauge_fill(c["gauge"] == "nonTrivial")
    return o.count_sf(o.dslash_tm_inv_eo(x, g, c["evenodd"], c["kappa"], mubar, t.endswith("Minus")))


def _expected_merged(c):
    if "expect_total" in c:
        return c["expect_total"]
    return c["per_site"] * (c["ns"] ** 3 * c["nt"] // 2)


@pytest.mark.parametrize("kind", ["port", "reference"])
@pytest.mark.parametrize("c", SPIN, ids=[c["case"] for c in SPIN])
def test_spinor_eo_kats_oracle(request, O, kind, c):
    if kind == "reference" and not O.available("reference"):
        pytest.skip("reference kernels not built")
    o = request.getfixturevalue("port" if kind == "port" else "ref")
    got = _spin_oracle(o, c)
    assert all(_close(g, w) for g, w in zip(got, c["expect"])), (got, c["expect"])


@pytest.mark.parametrize("kind", ["port", "reference"])
@pytest.mark.parametrize("c", MERGED, ids=[c["case"] for c in MERGED])
def test_merged_kats_oracle(request, O, kind, c):
    if kind == "reference" and not O.available("reference"):
        pytest.skip("reference kernels not built")
    o = request.getfixturevalue("port" if kind == "port" else "ref")
    got = _merged_oracle(o, O, c)
    assert _close(got, _expected_merged(c)), (got, _expected_merged(c))


# ------------------------------------------------------------------ GPU: the C ABI
def _sum(f):
    return float(f.dump().sum())


@pytest.mark.gpu
@pytest.mark.parametrize("c", SPIN, ids=[c["case"] for c in SPIN])
def test_spinor_eo_kats_gpu(system, c):
    import cl2qcd_b200 as c2q
    H = c2q.host
    L = c2q.Lattice(c["ns"], c["nt"])
    n = L.seo
    t = c["test"]
    F = lambda a=None: c2q.Spinorfield_eo(system, L, a)
    f = [F(_fill(k, n)) for k in c.get("fills") or ["ascendingComplex"]]
    a = [complex(*x) for x in c.get("coefficients", [])]
    out = F()
    if t == "testEvenOddSquarenorm":
        got = [H.squarenorm(f[0])]
    elif t == "testEvenOddScalarProduct":
        z = H.scalar_product(f[0], f[1])
        got = [z.real, z.imag]
    elif t == "testEvenOddZero":
        f[0].zero()
        got = [H.squarenorm(f[0])]
    elif t == "testEvenOddCold":
        f[0].cold()
        got = [H.squarenorm(f[0])]
    elif t == "testEvenOddSax":
        H.sax(out, a[0], f[0])
        got = [H.squarenorm(out)]
    elif t in ("testEvenOddSaxpy", "testEvenOddSaxpyArg"):
        H.saxpy(out, a[0], f[0], f[0])
        got = [H.squarenorm(out)]
    elif t == "testSaxsbypzEvenOdd":
        H.saxsbypz(out, a[0], f[0], a[1], f[0], f[0])
        got = [H.squarenorm(out)]
    elif t == "testConvertToEvenOdd":
        e, od = F(), F()
        H.convert_to_eoprec(e, od, _parity_full(c["ns"], c["nt"], c["fill_even_sites"]))
        got = [H.squarenorm(e), H.squarenorm(od)]
    else:
        raise ValueError(t)
    assert all(_close(g, w) for g, w in zip(got, c["expect"])), (got, c["expect"])


@pytest.mark.gpu
@pytest.mark.parametrize("c", MERGED, ids=[c["case"] for c in MERGED])
def test_merged_kats_gpu(system, port, c):
    import cl2qcd_b200 as c2q
    H = c2q.host
    L = c2q.Lattice(c["ns"], c["nt"])
    x = c2q.Spinorfield_eo(system, L, _fill(c["fills"][0], L.seo))
    out = c2q.Spinorfield_eo(system, L)
    t = c["test"]
    if t == "testSaxpyAndSquarenormEvenOdd":
        got = H.saxpy_AND_squarenorm(out, complex(*c["coefficient"]), x, x)
    elif t == "testSaxpyAndGamma5EvenOdd":
        y = c2q.Spinorfield_eo(system, L, _fill(c["fills"][1], L.seo))
        H.saxpy_AND_gamma5_eo(out, complex(*c["coefficient"]), x, y)
        got = _sum(out)
    elif t in ("testMTmSitediagonalAndGamma5EvenOdd", "testMTmSitediagonalMinusAndGamma5EvenOdd"):
        mubar = 2 * c["kappa"] * c["mu"]
        which = "M_tm_sitediagonal_AND_gamma5_eo" if "Minus" not in t else "M_tm_sitediagonal_minus_AND_gamma5_eo"
        getattr(H, which)(out, x, mubar)
        got = _sum(out)
    else:
        port.set_lattice(c["ns"], c["nt"])
        gf = c2q.Gaugefield(system, L, port.gauge_fill(c["gauge"] == "nonTrivial"))
        H.dslash_AND_M_tm_inverse_sitediagonal(out, gf, x, c["evenodd"], c["kappa"], 2 * c["kappa"] * c["mu"],
                                                t.endswith("Minus"))
        got = _sum(out)
    assert _close(got, _expected_merged(c)), (got, _expected_merged(c))
