"""CPU: the input-parameter parser against the reference's own parser tests
(meta/inputparameters_test.cpp): the defaults of an empty input file, the values
of meta/test_input_2 and of meta/test_input_aliases (the files verbatim in
tests/golden/reference_kats.json), for every parameter this library keeps; and
the invalid values its command-line tests reject."""
import ctypes as C
import json
import os

import pytest

KATS = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                   "reference_kats.json")))["inputparameters"]

# getter of meta::Inputparameters -> field of c2q_params
FIELDS = {
    "get_precision": lambda p: p.precision,
    "get_nspace": lambda p: p.lat.ns,
    "get_ntime": lambda p: p.lat.nt,
    "get_use_chem_pot_re": lambda p: p.lat.use_cp_re,
    "get_use_chem_pot_im": lambda p: p.lat.use_cp_im,
    "get_chem_pot_re": lambda p: p.lat.cp_re,
    "get_chem_pot_im": lambda p: p.lat.cp_im,
    "get_theta_fermion_spatial": lambda p: p.lat.theta_s,
    "get_theta_fermion_temporal": lambda p: p.lat.theta_t,
    "get_startcondition": lambda p: p.start_condition,
    "get_sourcefile": lambda p: p.initial_conf.decode(),
    "get_ignore_checksum_errors": lambda p: p.ignore_checksum_errors,
    "get_fermact": lambda p: p.fermion_action,
    "get_kappa": lambda p: p.kappa,
    "get_mu": lambda p: p.mu,
    "get_cgmax": lambda p: p.solver.cgmax,
    "get_use_eo": lambda p: p.use_eo,
    "get_solver": lambda p: p.solver.solver,
    "get_num_sources": lambda p: p.n_sources,
    "get_source_x": lambda p: p.source_pos[0],
    "get_source_y": lambda p: p.source_pos[1],
    "get_source_z": lambda p: p.source_pos[2],
    "get_source_t": lambda p: p.source_pos[3],
    "get_solver_prec": lambda p: p.solver.prec,
    "get_iter_refresh": lambda p: p.solver.iter_refresh,
    "get_corr_dir": lambda p: p.correlator_direction,
    "get_use_merge_kernels_spinor": lambda p: p.use_merge_kernels_spinor,
    "get_use_merge_kernels_fermion": lambda p: p.use_merge_kernels_fermion,
    "get_use_rec12": lambda p: p.solver.use_rec12,
}
# the reference's enum values (common_header_files/types.hpp:197-204) -> the library's codes
ENUMS = {"common::cold_start": 0, "common::hot_start": 1, "common::start_from_source": 2,
         "common::action::wilson": 1, "common::action::clover": 2, "common::action::twistedmass": 3,
         "common::action::rooted_stagg": 7, "common::cg": 1, "common::bicgstab": 2, "common::bicgstab_save": 3}


def _value(v):
    if v in ENUMS:
        return ENUMS[v]
    if v in ("true", "false"):
        return int(v == "true")
    if v.startswith('"'):
        return v.strip('"')
    if v == "sizeof(double) * 8":
        return 64
    return float(v)


def _parse(lib, text):
    from cl2qcd_b200 import _lib as L
    P = L.CParams()
    lib.c2q_params_default(C.byref(P))
    rc = lib.c2q_params_from_kv(text.encode(), C.byref(P))
    return rc, P


@pytest.mark.parametrize("case", ["defaults", "input_file2", "aliases"])
def test_reference_parser_cases(lib, case):
    k = KATS[case]
    rc, P = _parse(lib, k["input_text"])
    assert rc == 0, lib.c2q_params_last_error()
    checked = 0
    for getter, v in k["expect"].items():
        if getter not in FIELDS:
            continue  # a parameter of the reference's other parts
        got, want = FIELDS[getter](P), _value(v)
        assert got == want, (case, getter, got, want)
        checked += 1
    assert checked >= (20 if case != "aliases" else 4)


@pytest.mark.parametrize("text", ["startCondition=foo", "fermionAction=foo", "integrator0=foo"])
def test_reference_rejects(lib, text):
    """command_line2..4 of inputparameters_test.cpp throw Invalid_Parameters; the
    integrator is a parameter of the HMC, outside this library, so an invalid
    value there is accepted and ignored here."""
    rc, _ = _parse(lib, text)
    if text.startswith("integrator0"):
        assert rc == 0
    else:
        assert rc == -5, text
