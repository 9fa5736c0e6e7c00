"""The C++ call surface (include/cl2qcd_b200.hpp) and the input-parameter parser
(c2q_params_from_kv): a program written against the reference's classes is
compiled with g++ and driven from the reference's own inverter input files
(executables/tests/inverter_test_input_1 / _2, kept verbatim in
tests/golden/reference_kats.json), with the overrides its CMakeLists passes on
the command line (useEO, solver).

CPU: compiling, parsing (values, defaults, aliases, sections, errors).
GPU: perform_inversion + the pseudoscalar correlator against
executables/tests/inverter_test_ref / ref2, and the SolverDidNotSolve mapping."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KATS = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_kats.json")))


@pytest.fixture(scope="module")
def adapter(lib, tmp_path_factory):
    d = tmp_path_factory.mktemp("adapter")
    exe = str(d / "adapter_inverter")
    libdir = os.path.join(ROOT, "cl2qcd_b200")
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "adapter_inverter.cpp"), "-L" + libdir, "-lc2q_b200",
                        "-Wl,-rpath," + libdir, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe, d


def run(adapter, mode, name, overrides="", gauge=None):
    exe, d = adapter
    inp = d / f"{name}.in"
    inp.write_text(KATS["inverter"][name]["input_text"])
    args = [exe, mode, str(inp), overrides] + ([gauge] if gauge else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    return r.returncode, json.loads(r.stdout.strip().splitlines()[-1])


def test_header_is_plain_cxx17(adapter):
    """The header compiles without CUDA headers (done by the fixture) and names
    the reference's classes."""
    src = open(os.path.join(ROOT, "include", "cl2qcd_b200.hpp")).read()
    for name in ("class Inputparameters", "class System", "class Gaugefield", "class Spinorfield_eo",
                 "class Fermionmatrix_eo", "QplusQminus_eo", "class SolverStuck", "class SolverDidNotSolve",
                 "inline int cg(", "inline int bicgstab(", "perform_inversion", "calculate_correlator"):
        assert name in src, name


def test_reference_input_file_parses(adapter):
    rc, p = run(adapter, "params", "inverter_test_ref", "useEO=false\\nsolver=cg")
    assert rc == 0, p
    assert (p["nspace"], p["ntime"], p["fermact"], p["use_eo"], p["solver"]) == (4, 4, 3, 0, 1)
    assert p["kappa"] == 0.15 and p["mu"] == 4.0 and p["mubar"] == pytest.approx(1.2, rel=1e-15)
    # the reference's defaults for what the file leaves out (meta/parametersSolver.cpp:74-91,
    # parametersSources.cpp:67-77, parametersObs.cpp:67-74)
    assert (p["prec"], p["cgmax"], p["iter_refresh"], p["check_every"]) == (1e-23, 1000, 100, 10)
    assert (p["start"], p["n_sources"], p["corr_dir"], p["theta_t"], p["rec12"]) == (0, 12, 3, 0.0, 0)
    rc, p = run(adapter, "params", "inverter_test_ref2")
    assert rc == 0 and p["start"] == 2 and p["initial_conf"] == "conf.00200" and p["solver"] == 2


def test_parser_rules(lib):
    from cl2qcd_b200 import _lib as L
    P = L.CParams()
    lib.c2q_params_default(C.byref(P))
    text = ("# comment line\n  NS = 8   # alias of nSpace\nNT=16\nThetaT=1\nuseEO=off\nsolver=BiCGStab_Save\n"
            "useReconstruct12=yes\nbeta=5.6\nnHmcSteps=10\n[b200]\ninnerPrecision=16\nrelativeTolerance=1e-10\n")
    assert lib.c2q_params_from_kv(text.encode(), C.byref(P)) == 0, lib.c2q_params_last_error()
    assert (P.lat.ns, P.lat.nt, P.lat.theta_t, P.use_eo, P.solver.solver) == (8, 16, 1.0, 0, 3)
    assert (P.solver.use_rec12, P.solver.precision, P.solver.rel_tol) == (1, 16, 1e-10)
    assert P.mubar == pytest.approx(2 * 0.125 * 0.006)  # defaults kappa 0.125, mu 0.006
    # a second text overrides the first
    assert lib.c2q_params_from_kv(b"kappa=0.16\nmu=0.005", C.byref(P)) == 0
    assert P.mubar == pytest.approx(0.0016) and P.lat.ns == 8
    for bad, why in ((b"nSpace=7", b"even"), (b"kappa=abc", b"invalid value"), (b"fermionAction=foo", b"invalid value"),
                     (b"noSuchKey=1", b"unknown option"), (b"mu=1\nmu=2", b"more than once"),
                     (b"precision=16", b"precision"), (b"justtext", b"name = value"),
                     (b"[b200]\ninnerPrecision=8", b"innerPrecision"), (b"startCondition=foo", b"invalid value")):
        before = bytes(P)
        assert lib.c2q_params_from_kv(bad, C.byref(P)) == L.BAD_ARG, bad
        assert why in lib.c2q_params_last_error(), (bad, lib.c2q_params_last_error())
        assert bytes(P) == before  # unchanged on error


def test_invalid_file_raises_invalid_parameters(adapter):
    rc, out = run(adapter, "params", "inverter_test_ref", "useEO=maybe")
    assert rc == 3 and "useEO" in out["invalid_parameters"]


@pytest.mark.gpu
@pytest.mark.parametrize("use_eo", ["true", "false"])
@pytest.mark.parametrize("solver", ["bicgstab", "cg", "bicgstab_save"])
@pytest.mark.parametrize("name", ["inverter_test_ref", "inverter_test_ref2"])
def test_inversion_driven_from_reference_input(adapter, name, solver, use_eo):
    ref = KATS["inverter"][name]
    gauge = None
    if name == "inverter_test_ref2":  # initialConf=conf.00200, decoded into the fixture
        g = np.load(os.path.join(ROOT, "tests", "golden", "conf00200.npz"))["gauge"]
        gauge = str(adapter[1] / "conf00200.raw")
        np.ascontiguousarray(g, dtype=np.float64).tofile(gauge)
    rc, out = run(adapter, "invert", name, f"useEO={use_eo}\\nsolver={solver}", gauge)
    assert rc == 0, out
    np.testing.assert_allclose(out["ps"], ref["ps_correlator"], rtol=ref["tolerance_percent"] / 100)
    np.testing.assert_allclose(out["ps"], ref["ps_correlator"], rtol=1e-9)
    assert out["did_not_solve_iterations"] >= 3  # SolverDidNotSolve carried the iterations
    assert out["cg_iterations"] > 0 and out["cg_true_resid_rel"] < 1e-8
