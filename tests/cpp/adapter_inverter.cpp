// adapter_inverter.cpp -- a program written against the reference's C++
// classes (through include/cl2qcd_b200.hpp) that drives the inverter path
// from a reference input file: parameters, gauge field, the 12 point sources
// at the origin, perform_inversion and the pseudoscalar correlator; plus a CG
// call that must throw SolverDidNotSolve.  Test infrastructure: built and run
// by tests/test_cpp_adapter.py.
//
//   adapter_inverter params  <input file> [overrides]          (no GPU)
//   adapter_inverter invert  <input file> [overrides] [gauge]  (GPU; gauge: raw Matrixsu3[4V] doubles)
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "cl2qcd_b200.hpp"

using namespace cl2qcd_b200;

static std::string slurp(const char* path)
{
    std::ifstream f(path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

static std::string unescape(std::string s)  // "\n" in a shell argument separates overrides
{
    for (size_t i; (i = s.find("\\n")) != std::string::npos;) s.replace(i, 2, "\n");
    return s;
}

static int params_mode(const meta::Inputparameters& p)
{
    std::printf("{\"nspace\": %d, \"ntime\": %d, \"kappa\": %.17g, \"mu\": %.17g, \"mubar\": %.17g, "
                "\"fermact\": %d, \"use_eo\": %d, \"solver\": %d, \"prec\": %.17g, \"cgmax\": %d, "
                "\"iter_refresh\": %d, \"check_every\": %d, \"theta_t\": %.17g, \"theta_s\": %.17g, "
                "\"start\": %d, \"initial_conf\": \"%s\", \"n_sources\": %d, \"corr_dir\": %d, \"rec12\": %d, "
                "\"inner_precision\": %d, \"rel_tol\": %.17g}\n",
                p.get_nspace(), p.get_ntime(), p.get_kappa(), p.get_mu(), meta::get_mubar(p), (int)p.get_fermact(),
                (int)p.get_use_eo(), (int)p.get_solver(), p.get_solver_prec(), p.get_cgmax(), p.get_iter_refresh(),
                p.get_cg_iteration_block_size(), p.get_theta_fermion_temporal(), p.get_theta_fermion_spatial(),
                (int)p.get_startcondition(), p.get_sourcefile().c_str(), p.get_num_sources(), p.get_corr_dir(),
                (int)p.get_use_rec12(), p.c().solver.precision, p.c().solver.rel_tol);
    return 0;
}

static int invert_mode(const meta::Inputparameters& params, const char* gauge_path)
{
    hardware::System system(params);
    physics::InterfacesHandler ih(params);
    const int ns = params.get_nspace(), nt = params.get_ntime();
    const size_t vol = (size_t)ns * ns * ns * nt;
    std::vector<double> aos;
    if (gauge_path) {
        aos.resize(4 * vol * 18);
        std::ifstream f(gauge_path, std::ios::binary);
        f.read(reinterpret_cast<char*>(aos.data()), (std::streamsize)(aos.size() * sizeof(double)));
        if (!f) throw Invalid_Parameters("short gauge file");
    }
    physics::lattices::Gaugefield gf = gauge_path ? physics::lattices::Gaugefield(system, aos.data())
                                                  : physics::lattices::Gaugefield(system);
    // the 12 point sources at the origin: spin k % 4, colour k / 4, value 1
    std::vector<physics::lattices::Spinorfield*> sources, results;
    for (int k = 0; k < params.get_num_sources(); ++k) {
        std::vector<double> full(vol * 24, 0.0);
        full[2 * (3 * (k % 4) + k / 4)] = 1.0;
        sources.push_back(new physics::lattices::Spinorfield(system));
        sources.back()->load(full.data());
        results.push_back(new physics::lattices::Spinorfield(system));
    }
    physics::algorithms::perform_inversion(&results, &gf, sources, system, ih);
    const std::vector<hmc_float> corr =
        physics::observables::wilson::calculate_correlator("ps", results, sources, system, ih);
    std::printf("{\"ps\": [");
    for (size_t i = 0; i < corr.size(); ++i) std::printf("%s%.17g", i ? ", " : "", corr[i]);
    std::printf("]");
    // an eo CG with too few iterations: SolverDidNotSolve with its iteration count
    physics::lattices::Spinorfield_eo x(system), b(system);
    std::vector<double> src(b.get_elements() * 24, 0.0);
    for (size_t i = 0; i < src.size(); i += 7) src[i] = 1.0;
    b.load(src.data());
    x.zero();
    physics::fermionmatrix::QplusQminus_eo qpqm(system, ih);
    physics::WilsonAdditionalParameters add(params);
    meta::Inputparameters few(std::string(), "solverMaxIterations=3\nsolver=cg");
    physics::InterfacesHandler ih_few(few);
    int thrown = -1;
    try {
        physics::algorithms::solvers::cg(&x, qpqm, gf, b, system, ih_few, 1e-30, add);
    } catch (const physics::algorithms::solvers::SolverDidNotSolve& e) {
        thrown = e.get_iterations();
    }
    // and a full solve through the same call, with the reference's stopping test
    x.zero();
    c2q_solve_report rep{};
    const int it = physics::algorithms::solvers::cg(&x, qpqm, gf, b, system, ih, 1e-20, add, &rep);
    std::printf(", \"did_not_solve_iterations\": %d, \"cg_iterations\": %d, \"cg_true_resid_rel\": %.6g}\n", thrown, it,
                rep.true_resid_rel);
    for (auto* f : sources) delete f;
    for (auto* f : results) delete f;
    return 0;
}

int main(int argc, char** argv)
{
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s params|invert <input file> [overrides] [gauge]\n", argv[0]);
        return 2;
    }
    try {
        const meta::Inputparameters params(slurp(argv[2]), argc > 3 ? unescape(argv[3]) : std::string());
        if (!std::strcmp(argv[1], "params")) return params_mode(params);
        return invert_mode(params, argc > 4 ? argv[4] : nullptr);
    } catch (const Invalid_Parameters& e) {
        std::printf("{\"invalid_parameters\": \"%s\"}\n", e.what());
        return 3;
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 4;
    }
}
