// params.cpp -- the reference's inverter input parameters (key = value text)
// mapped onto the library's structures.
//
// The reference reads its input file with boost::program_options'
// parse_config_file after a normaliser renames a few aliases
// (meta/inputparameters.cpp:150-196); the hot-path keys and their defaults are
// those of meta/parametersConfig.cpp:147-187 (nSpace, nTime, precision,
// useReconstruct12, startCondition, initialConf, ignoreChecksumErrors),
// meta/parametersFermion.cpp:106-150 (fermionAction, kappa, mu,
// thetaFermion*, chemical potential, useEO, kernel merging),
// meta/parametersSolver.cpp:74-107 (solver and its limits),
// meta/parametersSources.cpp:67-90 and meta/parametersObs.cpp:67-86 (inverter
// sources, correlators); mubar = 2 kappa mu (meta/util.cpp:56-59).
//
// The file format follows parse_config_file: one `name = value` per line,
// surrounding blanks ignored, `#` starts a comment, `[section]` prefixes the
// names after it with `section.`; a name that is not an option is an error, as
// is a name given twice; enum values are case-insensitive; booleans accept
// true/false, yes/no, on/off, 1/0 (an empty value is true).  Every other key
// the reference defines (gauge action, HMC, RHMC, I/O, observables outside the
// inverter) is accepted and ignored: it configures parts of the reference that
// lie outside this library.  Keys of this library (no counterpart in the
// reference) live in the section `b200`: innerPrecision, relativeTolerance,
// reliableDelta, useGraph, temporalGauge.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <sstream>
#include <string>

#include "../../include/cl2qcd_b200.h"

namespace {

thread_local std::string g_err;

int bad(const std::string& msg)
{
    g_err = msg;
    return C2Q_BAD_ARG;
}

std::string trim(const std::string& s)
{
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

std::string lower(std::string s)
{
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// The reference's option names that configure parts outside this path.
const std::set<std::string>& ignored_keys()
{
    static const std::set<std::string> k = {
        "PRNGPostfix", "PRNGPrefix", "beta", "confPostfix", "confPrefix", "conservative", "createCheckpointEvery",
        "csw", "cswMP", "deviceId", "disableOclCompilerOptimization", "enableProfiling", "fermObsCorrelatorsPostfix",
        "fermObsCorrelatorsPrefix", "fermObsInSingleFile", "fermObsPbpPostfix", "fermObsPbpPrefix", "fermionActionMP",
        "findminmaxMaxIterations", "findminmaxPrecision", "findminmaxResiduumCheckEvery", "gaugeAction",
        "gaugeObsInSingleFile", "gaugeObsPostfix", "gaugeObsPrefix", "hmcObsPostfix", "hmcObsPrefix",
        "hmcObsToSingleFile", "hostSeed", "initialPRNG", "integrationSteps0", "integrationSteps1",
        "integrationSteps2", "integrator0", "integrator1", "integrator2", "kappaMP", "lambda0", "lambda1", "lambda2",
        "logLevel", "mass", "measurePbp", "measureRectangles", "measureTransportCoefficientKappa", "muMP",
        "nBenchmarkIterations", "nDevices", "nDigitsInConfCheckpoint", "nHeatbathSteps", "nHmcSteps",
        "nOverrelaxationSteps", "nPseudoFermions", "nRhmcSteps", "nSmearingSteps", "nTastes", "nTastesDecimalDigits",
        "nThermalizationSteps", "nTimeScales", "onlineMeasureEvery", "overwriteTemporaryCheckpointEvery",
        "pbpMeasurements", "pbpVersion", "placeSourcesOnHost", "printToScreen", "profilingDataPostfix",
        "profilingDataPrefix", "rationalApproxFileHB", "rationalApproxFileMD", "rationalApproxFileMetropolis",
        "rationalApproxLowerBound", "rationalApproxOrderHBAndMD", "rationalApproxOrderMetropolis",
        "rationalApproxUpperBound", "readConfsEvery", "readFromConfNumber", "readMultipleConfs",
        "readRationalApproxFromFile", "readUntilConfNumber", "rectanglesFilename", "rhmcObsPostfix", "rhmcObsPrefix",
        "rhmcObsToSingleFile", "smearingFactor", "solverForcePrecision", "solverMP", "solverMaxIterationsMP",
        "solverUseAsyncCopy", "splitCPU", "tau", "testRefVal", "testRefVal2", "transportCoefficientKappaFilename",
        "useAnisotropy", "useCPU", "useGPU", "useGaugeOnly", "useMP", "useSameRandomNumbers", "useSmearing", "xi"};
    return k;
}

// meta/inputparameters.cpp:180-193 (add_option_aliases)
const std::map<std::string, std::string>& aliases()
{
    static const std::map<std::string, std::string> a = {
        {"NS", "nSpace"}, {"NT", "nTime"}, {"use_evenodd", "useEO"}, {"thermsteps", "nThermalizationSteps"},
        {"thermalizationsteps", "nThermalizationSteps"}, {"puregauge", "useGaugeOnly"}, {"PGT", "useGaugeOnly"},
        {"test_ref_value", "testRefVal"}, {"test_ref_value2", "testRefVal2"}, {"ThetaT", "thetaFermionTemporal"},
        {"ThetaS", "thetaFermionSpatial"}};
    return a;
}

bool to_double(const std::string& v, double* out)
{
    if (v.empty()) return false;
    char* end = nullptr;
    errno     = 0;
    const double d = std::strtod(v.c_str(), &end);
    if (errno || end != v.c_str() + v.size() || !std::isfinite(d)) return false;
    *out = d;
    return true;
}

bool to_int(const std::string& v, int* out)
{
    if (v.empty()) return false;
    char* end = nullptr;
    errno     = 0;
    const long x = std::strtol(v.c_str(), &end, 10);
    if (errno || end != v.c_str() + v.size() || x < -2147483647L || x > 2147483647L) return false;
    *out = (int)x;
    return true;
}

bool to_bool(const std::string& v, int* out)
{
    const std::string s = lower(v);
    if (s.empty() || s == "on" || s == "yes" || s == "1" || s == "true") {
        *out = 1;
        return true;
    }
    if (s == "off" || s == "no" || s == "0" || s == "false") {
        *out = 0;
        return true;
    }
    return false;
}

bool to_enum(const std::string& v, const std::map<std::string, int>& m, int* out)
{
    auto it = m.find(lower(v));
    if (it == m.end()) return false;
    *out = it->second;
    return true;
}

}  // namespace

extern "C" {

C2Q_EXPORT void c2q_params_default(c2q_params* p)
{
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->lat.ns = 4;  // meta/parametersConfig.cpp:147-169
    p->lat.nt = 8;
    p->fermion_action = C2Q_ACTION_WILSON;  // meta/parametersFermion.cpp:106-128
    p->kappa          = 0.125;
    p->mu             = 0.006;
    p->mubar          = 2.0 * p->kappa * p->mu;
    p->use_eo         = 1;
    p->precision      = 64;
    c2q_solver_params_default(&p->solver);  // meta/parametersSolver.cpp:74-91
    p->start_condition = C2Q_START_COLD;
    strcpy(p->initial_conf, "conf.00000");
    p->source_type          = C2Q_SOURCE_POINT;  // meta/parametersSources.cpp:67-77
    p->source_content       = C2Q_CONTENT_ONE;
    p->n_sources            = 12;
    p->correlator_direction = 3;  // meta/parametersObs.cpp:67-74
}

C2Q_EXPORT const char* c2q_params_last_error(void) { return g_err.c_str(); }

C2Q_EXPORT int c2q_params_from_kv(const char* text, c2q_params* p)
{
    g_err.clear();
    if (!text || !p) return bad("c2q_params_from_kv: null argument");
    static const std::map<std::string, int> solvers = {
        {"cg", C2Q_SOLVER_CG}, {"bicgstab", C2Q_SOLVER_BICGSTAB}, {"bicgstab_save", C2Q_SOLVER_BICGSTAB_SAVE}};
    // common::action (common_header_files/types.hpp:198): the fermion matrices
    // here take wilson and twistedmass; the others parse, and the calls reject them
    static const std::map<std::string, int> actions = {
        {"wilson", C2Q_ACTION_WILSON}, {"clover", 2}, {"twistedmass", C2Q_ACTION_TWISTEDMASS}, {"rooted_stagg", 7}};
    static const std::map<std::string, int> starts = {
        {"cold_start", C2Q_START_COLD}, {"cold", C2Q_START_COLD}, {"hot_start", C2Q_START_HOT},
        {"hot", C2Q_START_HOT}, {"start_from_source", C2Q_START_CONTINUE}, {"source", C2Q_START_CONTINUE},
        {"continue", C2Q_START_CONTINUE}};
    static const std::map<std::string, int> stypes = {{"point", C2Q_SOURCE_POINT},
                                                      {"volume", C2Q_SOURCE_VOLUME},
                                                      {"timeslice", C2Q_SOURCE_TIMESLICE},
                                                      {"zslice", C2Q_SOURCE_ZSLICE}};
    static const std::map<std::string, int> contents = {{"one", C2Q_CONTENT_ONE},
                                                        {"z4", C2Q_CONTENT_Z4},
                                                        {"gaussian", C2Q_CONTENT_GAUSSIAN},
                                                        {"z2", C2Q_CONTENT_Z2}};
    c2q_params q = *p;  // assigned only when the whole text is valid
    std::set<std::string> seen;
    std::istringstream in(text);
    std::string line, section;
    int lineno = 0;
    while (std::getline(in, line)) {
        ++lineno;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = trim(line);
        if (line.empty()) continue;
        const std::string where = "line " + std::to_string(lineno) + ": ";
        if (line.front() == '[') {
            if (line.back() != ']') return bad(where + "bad section header '" + line + "'");
            section = trim(line.substr(1, line.size() - 2));
            continue;
        }
        const size_t eq = line.find('=');
        if (eq == std::string::npos) return bad(where + "expected name = value, got '" + line + "'");
        std::string key       = trim(line.substr(0, eq));
        const std::string val = trim(line.substr(eq + 1));
        if (section.empty()) {
            auto al = aliases().find(key);
            if (al != aliases().end()) key = al->second;
        } else {
            key = section + "." + key;
        }
        if (!seen.insert(key).second) return bad(where + "option '" + key + "' given more than once");
        auto need = [&](bool ok) { return ok ? C2Q_OK : bad(where + "invalid value '" + val + "' for '" + key + "'"); };
        int rc    = C2Q_OK;
        int iv    = 0;
        if (key == "nSpace") rc = need(to_int(val, &q.lat.ns));
        else if (key == "nTime") rc = need(to_int(val, &q.lat.nt));
        else if (key == "precision") rc = need(to_int(val, &q.precision));
        else if (key == "useReconstruct12") rc = need(to_bool(val, &q.solver.use_rec12));
        else if (key == "startCondition") rc = need(to_enum(val, starts, &q.start_condition));
        else if (key == "initialConf") {
            if (val.size() >= sizeof q.initial_conf) return bad(where + "initialConf path too long");
            strcpy(q.initial_conf, val.c_str());
        } else if (key == "ignoreChecksumErrors") rc = need(to_bool(val, &q.ignore_checksum_errors));
        else if (key == "fermionAction") rc = need(to_enum(val, actions, &q.fermion_action));
        else if (key == "kappa") rc = need(to_double(val, &q.kappa));
        else if (key == "mu") rc = need(to_double(val, &q.mu));
        else if (key == "thetaFermionSpatial") rc = need(to_double(val, &q.lat.theta_s));
        else if (key == "thetaFermionTemporal") rc = need(to_double(val, &q.lat.theta_t));
        else if (key == "useChemicalPotentialRe") rc = need(to_bool(val, &q.lat.use_cp_re));
        else if (key == "useChemicalPotentialIm") rc = need(to_bool(val, &q.lat.use_cp_im));
        else if (key == "chemicalPotentialRe") rc = need(to_double(val, &q.lat.cp_re));
        else if (key == "chemicalPotentialIm") rc = need(to_double(val, &q.lat.cp_im));
        else if (key == "useEO") rc = need(to_bool(val, &q.use_eo));
        else if (key == "useKernelMergingFermionMatrix") rc = need(to_bool(val, &q.use_merge_kernels_fermion));
        else if (key == "useKernelMergingSpinor") rc = need(to_bool(val, &q.use_merge_kernels_spinor));
        else if (key == "solver") rc = need(to_enum(val, solvers, &q.solver.solver));
        else if (key == "solverPrecision") rc = need(to_double(val, &q.solver.prec));
        else if (key == "solverMaxIterations") rc = need(to_int(val, &q.solver.cgmax));
        else if (key == "solverMinIterations") rc = need(to_int(val, &q.solver.min_iter));
        else if (key == "solverRestartEvery") rc = need(to_int(val, &q.solver.iter_refresh));
        else if (key == "solverResiduumCheckEvery") rc = need(to_int(val, &q.solver.resid_check_every));
        else if (key == "sourceType") rc = need(to_enum(val, stypes, &q.source_type));
        else if (key == "sourceContent") rc = need(to_enum(val, contents, &q.source_content));
        else if (key == "nSources") rc = need(to_int(val, &q.n_sources));
        else if (key == "sourceX") rc = need(to_int(val, &q.source_pos[0]));
        else if (key == "sourceY") rc = need(to_int(val, &q.source_pos[1]));
        else if (key == "sourceZ") rc = need(to_int(val, &q.source_pos[2]));
        else if (key == "sourceT") rc = need(to_int(val, &q.source_pos[3]));
        else if (key == "measureCorrelators") rc = need(to_bool(val, &q.measure_correlators));
        else if (key == "correlatorDirection") rc = need(to_int(val, &q.correlator_direction));
        else if (key == "b200.innerPrecision") rc = need(to_int(val, &q.solver.precision));
        else if (key == "b200.relativeTolerance") rc = need(to_double(val, &q.solver.rel_tol));
        else if (key == "b200.reliableDelta") rc = need(to_double(val, &q.solver.reliable_delta));
        else if (key == "b200.useGraph") rc = need(to_bool(val, &q.solver.use_graph));
        else if (key == "b200.temporalGauge") rc = need(to_bool(val, &q.solver.use_temporal_gauge));
        else if (!ignored_keys().count(key)) return bad(where + "unknown option '" + key + "'");
        if (rc) return rc;
    }
    // checks of this path (the reference checks these when it builds the lattice and the kernels)
    if (q.lat.ns < 2 || q.lat.nt < 2 || (q.lat.ns & 1) || (q.lat.nt & 1))
        return bad("nSpace and nTime must be even and at least 2");
    if (q.precision != 64 && q.precision != 32) return bad("precision must be 64 or 32 (bits)");
    if (q.solver.precision != 64 && q.solver.precision != 32 && q.solver.precision != 16)
        return bad("b200.innerPrecision must be 64, 32 or 16");
    if (q.solver.cgmax < 0 || q.solver.iter_refresh <= 0 || q.solver.resid_check_every <= 0)
        return bad("solverMaxIterations must be >= 0, solverRestartEvery and solverResiduumCheckEvery > 0");
    if (q.correlator_direction < 0 || q.correlator_direction > 3) return bad("correlatorDirection must be 0..3");
    if (q.n_sources < 0) return bad("nSources must be >= 0");
    q.mubar = 2.0 * q.kappa * q.mu;
    *p      = q;
    return C2Q_OK;
}

}  // extern "C"
