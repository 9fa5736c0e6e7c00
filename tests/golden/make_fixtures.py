"""Regenerate the golden fixtures of tests/golden/ (run in a container that has the
reference tree and the oracle built; the fixtures themselves are committed).

1. reference_kats.json -- the known-answer values the reference's own tests
   hold for this path, extracted verbatim (by regex) from its test sources:
   * physics/fermionmatrix/fermionmatrix_test.cpp: Aee, Aee_minus, Qplus_eo,
     Qminus_eo, QplusQminus_eo (squarenorm after one and two applications,
     cold 4^3x16 block, seeds 5..9);
   * physics/fermionmatrix/explicit_test.cpp: dslash (seed 13) and the four
     M_tm_*sitediagonal* cases (seeds 5, 7, 9, 11);
   * physics/algorithms/fermion_force_test.cpp: the eo fermion force (squarenorm
     of the momenta, cold 4^3x16 and conf.00200);
   * hardware/code/fermions_test.cpp: the closed form of the dslash_eo
     kernel test in theta and the chemical potential, and the
     M_tm_sitediagonal family per-site constants.
2. conf00200.npz -- the reference's ILDG test configuration ildg_io/conf.00200
   decoded by this project's ILDG reader (Matrixsu3[4V], float64), for the
   known answers that are defined on it (the second blocks of explicit_test.cpp
   and fermionmatrix_test.cpp, inverter_test_ref2);
3. ref_outputs.npz -- outputs of the reference's own kernels (oracle/_ref/
   libc2q_ref.so, compiled from the reference sources) on small seeded
   inputs, used to pin the restated oracle and the CUDA path.

Usage:  python tests/golden/make_fixtures.py [/path/to/reference]
        (default: the directory named by the environment variable CL2QCD_REFERENCE)
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def _floats(s):
    return [float(x) for x in re.findall(r"[-+]?\d*\.\d+(?:[eE][-+]?\d+)?|[-+]?\d+\.(?:[eE][-+]?\d+)?", s)]


def extract_kats(ref: str) -> dict:
    out = {"source": "reference test sources, values copied by regex", "fermionmatrix_eo": {}, "explicit": {}}
    fm = open(os.path.join(ref, "physics/fermionmatrix/fermionmatrix_test.cpp")).read()
    for m in re.finditer(r"BOOST_AUTO_TEST_CASE\((\w+)\)\s*\{\s*const hmc_float refs\[4\] = \{([^}]*)\};\s*"
                         r"test_fermionmatrix<physics::fermionmatrix::(\w+)>\(refs, (\d+)\);", fm):
        name, vals, cls, seed = m.group(1), _floats(m.group(2)), m.group(3), int(m.group(4))
        if cls.endswith("_eo") or cls.startswith("Aee"):
            out["fermionmatrix_eo"][cls] = {"seed": seed, "refs": vals,
                                            "where": "physics/fermionmatrix/fermionmatrix_test.cpp"}
    ex = open(os.path.join(ref, "physics/fermionmatrix/explicit_test.cpp")).read()
    for m in re.finditer(r"BOOST_AUTO_TEST_CASE\((\w+)\)(.*?)(?=BOOST_AUTO_TEST_CASE|\Z)", ex, re.S):
        name, body = m.group(1), m.group(2)
        first = body.split("conf.00200")[0] if "conf.00200" in body else body
        seeds = re.findall(r"pseudo_randomize<Spinorfield, spinor>\(&src, (\d+)\)", first)
        refs = re.findall(r"BOOST_CHECK_CLOSE\(squarenorm\(\w+\), ([-+0-9.eE]+), 0\.01\)", first)
        nt = re.findall(r"--nTime=(\d+)", first)
        if seeds and refs and ("sitediag" in name or name == "dslash"):
            out["explicit"][name] = {"seed": int(seeds[0]), "refs": [float(r) for r in refs[:2]],
                                     "nt": int(nt[0]) if nt else None,
                                     "where": "physics/fermionmatrix/explicit_test.cpp"}
    ft = open(os.path.join(ref, "hardware/code/fermions_test.cpp")).read()
    m = re.search(r"calculateReferenceValuesDslashEvenOdd.*?return ReferenceValues\{(.*?)\};", ft, re.S)
    coeffs = _floats(m.group(1))
    out["dslash_eo_closed_form"] = {
        "coefficients": coeffs[:6],
        "form": "Seo*(c0*cos(pi thS/NS) + c1*cos(cpi + pi thT/NT)*cosh(cpr) + c2*sin(pi thS/NS) "
                "+ c3*cosh(cpr)*sin(cpi + pi thT/NT) + c4*cos(cpi + pi thT/NT)*sinh(cpr) "
                "+ c5*sin(cpi + pi thT/NT)*sinh(cpr)), signs included in the coefficients",
        "kappa": 0.123456, "fill": "ascendingComplex spinor, nonTrivial gauge",
        "where": "hardware/code/fermions_test.cpp:106-125",
    }
    # signs of the closed form terms as written in the source
    body = m.group(1)
    signs = []
    for term in re.finditer(r"([-+])?\s*([0-9.]+)\s*\*", body):
        signs.append(-1.0 if term.group(1) == "-" else 1.0)
    out["dslash_eo_closed_form"]["coefficients"] = [s * abs(c) for s, c in zip(signs, coeffs[:6])]
    diag = {}
    for fn in ["mTmSitediagonal", "mTmSitediagonalMinus", "mTmInverseSitediagonal", "mTmInverseSitediagonalMinus"]:
        mm = re.search(r"calculateReferenceValues_" + fn + r"\(.*?ReferenceValues\{latticeVolume \* ([0-9.]+)\}",
                       ft, re.S)
        diag[fn] = float(mm.group(1))
    out["tm_sitediagonal_per_site"] = {"values": diag, "kappa": 0.123456, "mu": 0.123456,
                                       "fill": "ascendingComplex", "lattice": [4, 8],
                                       "where": "hardware/code/fermions_test.cpp:69-104,483-507"}
    # first blocks of explicit_test.cpp for the full-lattice operators (cold gauge field)
    out["explicit_full_cold"] = {}
    for m in re.finditer(r"BOOST_AUTO_TEST_CASE\((\w+)\)(.*?)(?=BOOST_AUTO_TEST_CASE|\Z)", ex, re.S):
        name, body = m.group(1), m.group(2)
        first = body.split("conf.00200")[0]
        seeds = re.findall(r"pseudo_randomize<Spinorfield, spinor>\(&(sf\d), (\d+)\)", first)
        refs = re.findall(r"BOOST_CHECK_CLOSE\(squarenorm\(\w+\), ([-+0-9.eE]+), 0\.01\)", first)
        fn = re.findall(r"physics::fermionmatrix::(\w+)\(&sf2, gf, sf1", first)
        nt = re.findall(r"--nTime=(\d+)", first)
        if seeds and refs and fn and fn[0] in ("M_wilson", "M_tm_plus", "M_tm_minus"):
            out["explicit_full_cold"][name] = {"seeds": {k: int(v) for k, v in seeds},
                                               "refs": [float(r) for r in refs[:2]], "operator": fn[0],
                                               "kappa": 0.125, "mu": 0.006, "lattice": [4, int(nt[0]) if nt else 4],
                                               "where": "physics/fermionmatrix/explicit_test.cpp"}
    # second blocks of explicit_test.cpp: the full-lattice operators on the ILDG
    # configuration ildg_io/conf.00200 (nTime 4, default kappa 0.125, mu 0.006)
    out["explicit_conf00200"] = {}
    for m in re.finditer(r"BOOST_AUTO_TEST_CASE\((\w+)\)(.*?)(?=BOOST_AUTO_TEST_CASE|\Z)", ex, re.S):
        name, body = m.group(1), m.group(2)
        if "conf.00200" not in body:
            continue
        second = body.split("conf.00200", 1)[1]
        seeds = re.findall(r"pseudo_randomize<Spinorfield, spinor>\(&(sf\d), (\d+)\)", second)
        refs = re.findall(r"BOOST_CHECK_CLOSE\(squarenorm\(\w+\), ([-+0-9.eE]+), 0\.01\)", second)
        fn = re.findall(r"physics::fermionmatrix::(\w+)\(&sf2, gf, sf1", second)
        if seeds and refs and fn:
            out["explicit_conf00200"][name] = {"seeds": {k: int(v) for k, v in seeds},
                                               "refs": [float(r) for r in refs[:2]], "operator": fn[0],
                                               "kappa": 0.125, "mu": 0.006, "lattice": [4, 4],
                                               "where": "physics/fermionmatrix/explicit_test.cpp"}
    # physics/algorithms/fermion_force_test.cpp, case fermion_force_eo: squarenorm of the
    # momenta after F(sf1, sf2, EVEN) and after adding F(sf1, sf2, ODD), with sf1, sf2 the
    # eo halves of a drand48 full field; cold 4^3x16 and conf.00200 (4^4), kappa .125
    ff = open(os.path.join(ref, "physics/algorithms/fermion_force_test.cpp")).read()
    m = re.search(r"BOOST_AUTO_TEST_CASE\(fermion_force_eo\)(.*?)(?=BOOST_AUTO_TEST_CASE|\Z)", ff, re.S)
    out["fermion_force_eo"] = []
    for blk in m.group(1).split("using namespace physics::lattices;")[1:]:
        nt = re.findall(r"--nTime=(\d+)", blk)
        seed = re.findall(r"pseudo_randomize<Spinorfield, spinor>\(&src, (\d+)\)", blk)
        refs = re.findall(r"BOOST_CHECK_CLOSE\(squarenorm\(gm\), ([-+0-9.eE]+), 0\.01\)", blk)
        out["fermion_force_eo"].append({"nt": int(nt[0]), "gauge": "conf.00200" if "conf.00200" in blk else "cold",
                                        "seed": int(seed[0]), "refs": [float(r) for r in refs], "kappa": 0.125,
                                        "where": "physics/algorithms/fermion_force_test.cpp"})
    # the same file, case fermion_force: the non-eo force of two drand48 full fields
    m = re.search(r"BOOST_AUTO_TEST_CASE\(fermion_force\)(.*?)(?=BOOST_AUTO_TEST_CASE|\Z)", ff, re.S)
    out["fermion_force_full"] = []
    for blk in m.group(1).split("using namespace physics::lattices;")[1:]:
        nt = re.findall(r"--nTime=(\d+)", blk)
        seeds = re.findall(r"pseudo_randomize<Spinorfield, spinor>\(&(sf\d), (\d+)\)", blk)
        refs = re.findall(r"BOOST_CHECK_CLOSE\(squarenorm\(gm\), ([-+0-9.eE]+), 0\.01\)", blk)
        out["fermion_force_full"].append({"nt": int(nt[0]), "gauge": "conf.00200" if "conf.00200" in blk else "cold",
                                          "seeds": {k: int(v) for k, v in seeds}, "refs": [float(r) for r in refs],
                                          "kappa": 0.125, "where": "physics/algorithms/fermion_force_test.cpp"})
    # integration references of the inverter executable (executables/tests/testInverter.py:
    # the pseudoscalar correlator lines, compared at 0.1 %), with their input files
    out["inverter"] = {}
    for name, inp in (("inverter_test_ref", "inverter_test_input_1"), ("inverter_test_ref2", "inverter_test_input_2")):
        vals = _floats(open(os.path.join(ref, "executables/tests", name)).read())
        params = {}
        text = open(os.path.join(ref, "executables/tests", inp)).read()
        for line in text.splitlines():
            if "=" in line:
                k, v = line.strip().split("=", 1)
                params[k] = v
        out["inverter"][name] = {"ps_correlator": vals, "input": params, "input_text": text,
                                 "tolerance_percent": 0.1, "where": f"executables/tests/{name}, {inp}"}
    return out


def _extents(tok):
    m = re.search(r"LatticeExtents\{ns(\d+),\s*nt(\d+)\}", tok)
    return int(m.group(1)), int(m.group(2))


def _num(expr, ntp):
    return float(eval(expr.replace("nonTrivialParameter", repr(ntp)).replace(".*", "*")))


def _cases(src, suites):
    """(suite, case, call text) of every BOOST_AUTO_TEST_CASE inside the named suites."""
    out = []
    for sm in re.finditer(r"BOOST_AUTO_TEST_SUITE\((\w+)\)(.*?)BOOST_AUTO_TEST_SUITE_END\(\)", src, re.S):
        if sm.group(1) not in suites:
            continue
        for cm in re.finditer(r"BOOST_AUTO_TEST_CASE\((\w+)\)\s*\{(.*?)\}\s*(?=BOOST_AUTO_TEST_CASE|\Z)",
                              sm.group(2), re.S):
            out.append((sm.group(1), cm.group(1), " ".join(cm.group(2).split())))
    return out


def _reference_value_tables(src, ntp):
    """calculateReferenceValues_<name>: list of (python condition, value per lattice site)
    from its `if (...)` blocks returning `ReferenceValues{latticeVolume * (v)}`."""
    tables = {}
    for fm in re.finditer(r"calculateReferenceValues_(\w+)\([^)]*\)\s*\{(.*?)\n\}", src, re.S):
        stack, rows = [], []
        body = re.sub(r"\b(and|or)\s*\n\s*", r"\1 ", fm.group(2))  # conditions continued on the next line
        for line in body.splitlines():
            t = line.strip()
            m = re.match(r"(\}\s*else\s+)?if \((.*)\)\s*\{$", t)
            if m:
                if m.group(1):
                    stack.pop()
                stack.append(m.group(2))
                continue
            m = re.match(r"return ReferenceValues\{latticeVolume \* \(([-+0-9.eE]+)\)\};", t)
            if m:
                rows.append((" and ".join(f"({c})" for c in stack), float(m.group(1))))
                continue
            if t == "}" and stack:
                stack.pop()
        conv = []
        for cond, v in rows:
            c = (cond.replace("massParameters.kappa", "kappa").replace("massParameters.mu", "mu")
                 .replace("coefficient.re", "cre").replace("coefficient.im", "cim")
                 .replace("GaugefieldFillType::cold", "'cold'").replace("GaugefieldFillType::nonTrivial", "'nonTrivial'")
                 .replace("gF", "gf").replace("nonTrivialParameter", repr(ntp)))
            conv.append((c, v))
        tables[fm.group(1)] = conv
    return tables


def _lookup(table, **env):
    for cond, v in table:
        if eval(cond, {}, env):
            return v
    raise ValueError(f"no reference value for {env}")


def extract_blas_kats(ref: str) -> dict:
    """The eo BLAS suites of hardware/code/spinors_test.cpp, the merged kernels of
    fermions_merged_kernels_test.cpp and spinors_merged_kernels_test.cpp.  The
    cases (lattice, fills, coefficients, masses) are read from the test sources;
    the expected values are the tests' own: the closed forms of spinors_test.cpp:30-106
    (restated below) and the per-site constants of the merged-kernel tests (read
    from their calculateReferenceValues_* functions)."""
    ntp = float(re.search(r"nonTrivialParameter\s*=\s*([0-9.]+)",
                          open(os.path.join(ref, "hardware/code/kernelTester.hpp")).read()).group(1))
    sq24 = (2 * 24 ** 3 + 3 * 24 ** 2 + 24) / 6.0  # sumOfIntegersSquared(24), testUtilities.cpp:42-45
    odd, even = float(sum(range(1, 24, 2))), float(sum(range(2, 25, 2)))  # sumOfIntegers(1,23,2), (2,24,2)
    src = open(os.path.join(ref, "hardware/code/spinors_test.cpp")).read()
    out = {"spinors_eo": [], "merged_eo": [], "where": "hardware/code/spinors_test.cpp, "
           "fermions_merged_kernels_test.cpp, spinors_merged_kernels_test.cpp (tolerance 1e-9 relative, "
           "kernelTester.cpp)", "nonTrivialParameter": ntp}
    fills = lambda t: re.findall(r"SpinorFillType::(\w+)", t)
    coeffs = lambda t: [[float(a), float(b)] for a, b in re.findall(r"\{\s*([-0-9.]+),\s*([-0-9.]+)\s*\}", t)]
    for suite, case, call in _cases(src, {"GLOBAL_SQUARENORM_EO", "SCALAR_PRODUCT_EO", "ZERO_EO", "COLD_EO", "SAX_EO",
                                          "SAXPY_EO", "SAXSBYPZ_EO", "CONVERT_EO"}):
        fn = call.split("(")[0]
        ns, nt = _extents(call)
        seo = ns ** 3 * nt // 2
        e = {"suite": suite, "case": case, "test": fn, "ns": ns, "nt": nt}
        if fn == "testEvenOddSquarenorm":
            f = fills(call)
            e.update(fills=f, expect=[seo * (12.0 if f[0] == "one" else sq24)])
        elif fn == "testEvenOddScalarProduct":
            f = fills(call)
            val = {("one", "one"): (12.0, 0.0), ("one", "ascendingComplex"): (odd, even),
                   ("ascendingComplex", "one"): (odd, -even),
                   ("ascendingComplex", "ascendingComplex"): (sq24, 0.0)}[tuple(f)]
            e.update(fills=f, expect=[seo * val[0], seo * val[1]])
        elif fn in ("testEvenOddZero", "testEvenOddCold"):
            e.update(fills=fills(call), expect=[0.0 if fn == "testEvenOddZero" else 0.5])
        elif fn in ("testEvenOddSax", "testEvenOddSaxpy", "testEvenOddSaxpyArg", "testSaxsbypzEvenOdd"):
            c = coeffs(call.split("ComplexNumbers", 1)[1])
            if fn == "testEvenOddSax":
                k = complex(*c[0])
            elif fn == "testSaxsbypzEvenOdd":
                k = 1 + complex(*c[0]) + complex(*c[1])
            else:
                k = 1 - complex(*c[0])
            e.update(fills=["ascendingComplex"], coefficients=c, expect=[abs(k) ** 2 * seo * sq24])
        elif fn == "testConvertToEvenOdd":
            even_sites = "true" in call
            e.update(fill_even_sites=even_sites, expect=[12.0 * seo if even_sites else 0.0,
                                                         0.0 if even_sites else 12.0 * seo])
        else:
            continue
        out["spinors_eo"].append(e)
    msrc = open(os.path.join(ref, "hardware/code/fermions_merged_kernels_test.cpp")).read()
    tables = _reference_value_tables(msrc, ntp)
    kinds = {"testDslashEvenOddAndMTmInverseSitediagonal": "dslashEvenOddAndMTmInverseSitediagonal",
             "testDslashEvenOddAndMTmInverseSitediagonalMinus": "dslashEvenOddAndMTmInverseSitediagonalMinus",
             "testMTmSitediagonalAndGamma5EvenOdd": "mTmSitediagonalAndGamma5EvenOdd",
             "testMTmSitediagonalMinusAndGamma5EvenOdd": "mTmSitediagonalMinusAndGamma5EvenOdd",
             "testSaxpyAndGamma5EvenOdd": "saxpyAndGamma5EvenOdd"}
    for suite, case, call in _cases(msrc, {"DSLASH_AND_M_TM_INVERSE_SITEDIAGONAL_EO",
                                           "DSLASH_AND_M_TM_INVERSE_SITEDIAGONAL_MINUS_EO",
                                           "M_TM_SITEDIAGONAL_AND_GAMMA5_EO", "M_TM_SITEDIAGONAL_MINUS_AND_GAMMA5_EO",
                                           "SAXPY_AND_GAMMA5_EO"}):
        fn = call.split("(")[0]
        ns, nt = _extents(call)
        e = {"suite": suite, "case": case, "test": fn, "ns": ns, "nt": nt, "fills": fills(call)}
        if fn == "testSaxpyAndGamma5EvenOdd":
            a, b = re.search(r"hmc_complex\{([^,]+),([^}]+)\}", call).groups()
            cre, cim = _num(a, ntp), _num(b, ntp)
            e.update(coefficient=[cre, cim], per_site=_lookup(tables[kinds[fn]], cre=cre, cim=cim))
        else:
            a, b = re.search(r"TwistedMassMassParameters\{([^,]+),([^}]+)\}", call).groups()
            kappa, mu = _num(a, ntp), _num(b, ntp)
            gm = re.search(r"GaugefieldFillType::(\w+)", call)
            gf = gm.group(1) if gm else None
            e.update(kappa=kappa, mu=mu, gauge=gf,
                     per_site=_lookup(tables[kinds[fn]], kappa=kappa, mu=mu, gf=gf))
            if gf is not None:
                e["evenodd"] = 1 if call.rstrip(") ;").endswith("true") else 0
        out["merged_eo"].append(e)
    ssrc = open(os.path.join(ref, "hardware/code/spinors_merged_kernels_test.cpp")).read()
    for suite, case, call in _cases(ssrc, {"SF_SAXPY_AND_SQUARENORM_EO"}):
        ns, nt = _extents(call)
        cre, cim = [float(x) for x in re.search(r"hmc_complex\{([^,]+),([^}]+)\}", call).groups()]
        k = 1 - complex(cre, cim)
        out["merged_eo"].append({"suite": suite, "case": case, "test": "testSaxpyAndSquarenormEvenOdd", "ns": ns,
                                 "nt": nt, "fills": ["ascendingComplex"], "coefficient": [cre, cim],
                                 "expect_total": abs(k) ** 2 * (ns ** 3 * nt // 2) * sq24})
    return out


def extract_params_kats(ref: str) -> dict:
    """meta/inputparameters_test.cpp: the values its checkDefaults (empty input file,
    the double-precision branch), input_file2 (meta/test_input_2) and aliases
    (meta/test_input_aliases) cases require, with the input files' text verbatim."""
    src = open(os.path.join(ref, "meta/inputparameters_test.cpp")).read()
    blocks = {"defaults": src[src.index("void checkDefaults"):src.index("BOOST_AUTO_TEST_CASE(defaults)")],
              "input_file2": src[src.index("BOOST_AUTO_TEST_CASE(input_file2)"):
                                 src.index("BOOST_AUTO_TEST_CASE(command_line1)")],
              "aliases": src[src.index("BOOST_AUTO_TEST_CASE(aliases)"):src.index("BOOST_AUTO_TEST_CASE(help)")]}
    files = {"defaults": "test_input_1", "input_file2": "test_input_2", "aliases": "test_input_aliases"}
    out = {"where": "meta/inputparameters_test.cpp"}
    for name, body in blocks.items():
        body = body.split("#else")[0] + (body.split("#endif")[1] if "#endif" in body else "")
        expect = {}
        for getter, val in re.findall(r"BOOST_REQUIRE_EQUAL\(params\.(get_\w+|is_\w+)\(\)(?:\.size\(\))?,\s*([^;]+)\);",
                                      body):
            v = val.strip()[:-1].strip() if val.strip().endswith(")") else val.strip()
            if getter in expect:
                continue
            expect[getter] = v
        out[name] = {"input_file": f"meta/{files[name]}",
                     "input_text": open(os.path.join(ref, "meta", files[name])).read(), "expect": expect}
    return out


def make_ref_outputs(path):
    import oracle as O
    R = O.Oracle("reference")
    data = {}
    # 4^4, random (drand48) non-unitary gauge and spinor, antiperiodic T and a spatial phase
    R.set_lattice(4, 4, 1.0, 0.3)
    g = np.zeros((4 * R.vol, 18))
    R.lib.c2qo_pseudo_randomize(g, g.size, 3)
    s = R.pseudo_randomize(R.seo, 4)
    data["lat4_gauge_seed"] = np.array([3])
    data["lat4_spinor_seed"] = np.array([4])
    data["lat4_dslash_even"] = R.dslash_eo(s, g, O.EVEN, 0.15)
    data["lat4_dslash_odd"] = R.dslash_eo(s, g, O.ODD, 0.15)
    data["lat4_qpqm"] = R.apply(O.OP_QPQM_EO, s, g, 0.15, 0.03)
    data["lat4_dslash_tminv_odd"] = R.dslash_tm_inv_eo(s, g, O.ODD, 0.15, 0.03)
    np.savez_compressed(path, **data)


def decode_conf00200(ref: str) -> dict:
    """conf.00200 (4^4, the reference's ILDG test configuration) through this
    project's ILDG reader, stored as the reference's host layout Matrixsu3[4V]."""
    import cl2qcd_b200 as c2q
    ns, nt, aos, info = c2q.host.read_ildg(os.path.join(ref, "ildg_io/conf.00200"))
    np.savez_compressed(os.path.join(HERE, "conf00200.npz"), gauge=aos, ns=ns, nt=nt)
    plaq = re.findall(r"plaquette = ([0-9.]+)", info["xlf_info"])
    return {"ns": ns, "nt": nt, "precision": info["precision"], "suma": info["suma"], "sumb": info["sumb"],
            "checksum_status": info["checksum_status"],
            "plaquette_recorded": float(plaq[0]) if plaq else None,
            "plaquette": c2q.host.plaquette(c2q.Lattice(ns, nt), aos),
            "where": "ildg_io/conf.00200 (xlf-info, scidac-checksum records)"}


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CL2QCD_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("name the reference tree: make_fixtures.py /path/to/reference, or set CL2QCD_REFERENCE")
    kats = extract_kats(ref)
    kats["blas_and_merged_eo"] = extract_blas_kats(ref)
    kats["inputparameters"] = extract_params_kats(ref)
    kats["ildg_conf00200"] = decode_conf00200(ref)
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(kats, f, indent=1, sort_keys=True)
    make_ref_outputs(os.path.join(HERE, "ref_outputs.npz"))
    print("wrote", os.path.join(HERE, "reference_kats.json"), os.path.join(HERE, "ref_outputs.npz"))
