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
    kats["ildg_conf00200"] = decode_conf00200(ref)
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(kats, f, indent=1, sort_keys=True)
    make_ref_outputs(os.path.join(HERE, "ref_outputs.npz"))
    print("wrote", os.path.join(HERE, "reference_kats.json"), os.path.join(HERE, "ref_outputs.npz"))
