/*
 * cl2qcd_b200.hpp -- the reference's C++ call surface of the even-odd inverter
 * path, header-only, on top of the C ABI of cl2qcd_b200.h.
 *
 * Code written against CL2QCD's classes compiles against these after
 * `using namespace cl2qcd_b200;` (or a namespace alias): the same namespaces,
 * class names, constructor arguments where they carry meaning here, solver
 * signatures and exception types.
 *
 *   meta::Inputparameters, meta::get_mubar      meta/inputparameters.hpp, meta/util.cpp:56-59
 *   hardware::System                            hardware/system.hpp:70-84
 *   physics::AdditionalParameters,
 *   physics::WilsonAdditionalParameters         physics/additionalParameters.hpp:29-36,
 *                                               interfaceImplementations/physicsParameters.hpp:35-55
 *   physics::InterfacesHandler                  physics/interfacesHandler.hpp (the solver parameters)
 *   physics::lattices::Gaugefield, Spinorfield_eo, Spinorfield
 *                                               physics/lattices/gaugefield.hpp, spinorfield_eo.hpp:48-305,
 *                                               spinorfield.hpp
 *   physics::fermionmatrix::Fermionmatrix_eo, Aee, Aee_minus, Qplus_eo,
 *   Qminus_eo, QplusQminus_eo                   physics/fermionmatrix/fermionmatrix.hpp:121-310
 *   physics::algorithms::solvers::cg, bicgstab  physics/algorithms/solvers/cg.hpp:53-56, bicgstab.hpp:54-57
 *   physics::algorithms::solvers::SolverException, SolverStuck, SolverDidNotSolve
 *                                               physics/algorithms/solvers/exceptions.hpp:35-62
 *   physics::algorithms::perform_inversion      physics/algorithms/inversion.hpp:40-43
 *   physics::observables::wilson::calculate_correlator ("ps")
 *                                               physics/observables/wilsonTwoFlavourCorrelators.hpp:36-39
 *   Invalid_Parameters                          executables/exceptions.hpp
 *
 * Objects own their device memory (RAII, not copyable) and must not outlive
 * the System they were created on.  Errors of the library that have no
 * reference exception type throw cl2qcd_b200::Error with the status code.
 */
#ifndef CL2QCD_B200_HPP
#define CL2QCD_B200_HPP

#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cl2qcd_b200.h"

namespace cl2qcd_b200 {

typedef double hmc_float;

class Error : public std::runtime_error {
  public:
    Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const noexcept { return code_; }

  private:
    int code_;
};

class Invalid_Parameters : public std::invalid_argument {
  public:
    explicit Invalid_Parameters(const std::string& what) : std::invalid_argument(what) {}
};

namespace common {
    enum action { wilson = C2Q_ACTION_WILSON, twistedmass = C2Q_ACTION_TWISTEDMASS };
    enum solver { cg = C2Q_SOLVER_CG, bicgstab = C2Q_SOLVER_BICGSTAB, bicgstab_save = C2Q_SOLVER_BICGSTAB_SAVE };
    enum startcondition { cold_start = C2Q_START_COLD, hot_start = C2Q_START_HOT,
                          start_from_source = C2Q_START_CONTINUE };
}  // namespace common

namespace detail {
    inline void check(int rc, const c2q_ctx* ctx, const char* what)
    {
        if (rc == C2Q_OK) return;
        std::string msg = std::string(what) + ": ";
        if (ctx && c2q_last_error(ctx)) msg += c2q_last_error(ctx);
        if (rc == C2Q_BAD_ARG) throw Invalid_Parameters(msg);
        throw Error(rc, msg);
    }
}  // namespace detail

// ---------------------------------------------------------------- meta
namespace meta {
    class Inputparameters {
      public:
        Inputparameters() { c2q_params_default(&p_); }
        /* key = value text as in an input file; `overrides` (the same format)
         * take precedence, as the reference's command-line options do */
        explicit Inputparameters(const std::string& text, const std::string& overrides = "")
        {
            c2q_params_default(&p_);
            parse(text);
            if (!overrides.empty()) parse(overrides);
        }
        static Inputparameters from_file(const std::string& path, const std::string& overrides = "")
        {
            std::ifstream f(path);
            if (!f) throw Invalid_Parameters("Invalid config file " + path);
            std::stringstream ss;
            ss << f.rdbuf();
            return Inputparameters(ss.str(), overrides);
        }
        int get_nspace() const noexcept { return p_.lat.ns; }
        int get_ntime() const noexcept { return p_.lat.nt; }
        size_t get_precision() const noexcept { return (size_t)p_.precision; }
        bool get_use_rec12() const noexcept { return p_.solver.use_rec12 != 0; }
        common::action get_fermact() const noexcept { return (common::action)p_.fermion_action; }
        hmc_float get_kappa() const noexcept { return p_.kappa; }
        hmc_float get_mu() const noexcept { return p_.mu; }
        hmc_float get_theta_fermion_spatial() const noexcept { return p_.lat.theta_s; }
        hmc_float get_theta_fermion_temporal() const noexcept { return p_.lat.theta_t; }
        bool get_use_chem_pot_re() const noexcept { return p_.lat.use_cp_re != 0; }
        bool get_use_chem_pot_im() const noexcept { return p_.lat.use_cp_im != 0; }
        hmc_float get_chem_pot_re() const noexcept { return p_.lat.cp_re; }
        hmc_float get_chem_pot_im() const noexcept { return p_.lat.cp_im; }
        bool get_use_eo() const noexcept { return p_.use_eo != 0; }
        bool get_use_merge_kernels_fermion() const noexcept { return p_.use_merge_kernels_fermion != 0; }
        common::solver get_solver() const noexcept { return (common::solver)p_.solver.solver; }
        hmc_float get_solver_prec() const noexcept { return p_.solver.prec; }
        int get_cgmax() const noexcept { return p_.solver.cgmax; }
        int get_iter_refresh() const noexcept { return p_.solver.iter_refresh; }
        int get_cg_iteration_block_size() const noexcept { return p_.solver.resid_check_every; }
        int get_cg_minimum_iteration_count() const noexcept { return p_.solver.min_iter; }
        common::startcondition get_startcondition() const noexcept
        {
            return (common::startcondition)p_.start_condition;
        }
        std::string get_sourcefile() const { return p_.initial_conf; }
        bool get_ignore_checksum_errors() const noexcept { return p_.ignore_checksum_errors != 0; }
        int get_num_sources() const noexcept { return p_.n_sources; }
        int get_corr_dir() const noexcept { return p_.correlator_direction; }
        const c2q_params& c() const noexcept { return p_; }
        c2q_params& c() noexcept { return p_; }

      private:
        void parse(const std::string& text)
        {
            if (c2q_params_from_kv(text.c_str(), &p_) != C2Q_OK) throw Invalid_Parameters(c2q_params_last_error());
        }
        c2q_params p_;
    };
    inline hmc_float get_mubar(const Inputparameters& p) { return 2. * p.get_kappa() * p.get_mu(); }
}  // namespace meta

// ---------------------------------------------------------------- hardware
namespace hardware {
    class System {
      public:
        explicit System(const meta::Inputparameters& params, int device = 0, void* cuda_stream = nullptr)
            : params_(params)
        {
            detail::check(c2q_ctx_create(&ctx_, device, cuda_stream), nullptr, "c2q_ctx_create");
        }
        ~System() { c2q_ctx_destroy(ctx_); }
        System(const System&)            = delete;
        System& operator=(const System&) = delete;
        const meta::Inputparameters& get_inputparameters() const noexcept { return params_; }
        c2q_ctx* ctx() const noexcept { return ctx_; }
        void synchronize() const { detail::check(c2q_ctx_synchronize(ctx_), ctx_, "synchronize"); }

      private:
        meta::Inputparameters params_;
        c2q_ctx* ctx_ = nullptr;
    };
}  // namespace hardware

// ---------------------------------------------------------------- physics
namespace physics {
    class AdditionalParameters {
      public:
        virtual ~AdditionalParameters() {}
        virtual hmc_float getKappa() const = 0;
        virtual hmc_float getMubar() const = 0;
    };

    class WilsonAdditionalParameters final : public AdditionalParameters {
      public:
        WilsonAdditionalParameters(const meta::Inputparameters& params, const bool /*withMassPreconditioning*/ = false)
            : kappa_(params.get_kappa()), mubar_(meta::get_mubar(params))
        {
        }
        hmc_float getKappa() const override { return kappa_; }
        hmc_float getMubar() const override { return mubar_; }

      private:
        hmc_float kappa_, mubar_;
    };

    /* The parameter interfaces the solvers and matrices read, built from the
     * input parameters (what InterfacesHandlerImplementation provides). */
    class InterfacesHandler {
      public:
        explicit InterfacesHandler(const meta::Inputparameters& params) : params_(params) {}
        const meta::Inputparameters& parameters() const noexcept { return params_; }
        c2q_solver_params solver_parameters() const noexcept { return params_.c().solver; }

      private:
        meta::Inputparameters params_;
    };

    namespace lattices {
        inline c2q_lattice lattice_of(const meta::Inputparameters& p) { return p.c().lat; }

        class Gaugefield {
          public:
            /* startCondition: cold (unit links) or continue (the ILDG file initialConf). */
            explicit Gaugefield(const hardware::System& system) : system_(system)
            {
                const meta::Inputparameters& p = system.get_inputparameters();
                create();
                const size_t n = (size_t)4 * vol() * 18;
                std::vector<double> aos(n, 0.0);
                if (p.get_startcondition() == common::cold_start) {
                    for (size_t l = 0; l < n / 18; ++l) aos[18 * l] = aos[18 * l + 8] = aos[18 * l + 16] = 1.0;
                } else if (p.get_startcondition() == common::start_from_source) {
                    int ns = 0, nt = 0, prec = 0, status = 0;
                    unsigned a = 0, b = 0;
                    detail::check(c2q_ildg_read(p.get_sourcefile().c_str(), aos.data(), aos.size(), &ns, &nt, &prec,
                                                nullptr, 0, &a, &b, &status),
                                  system.ctx(), "reading initialConf");
                    if (ns != p.get_nspace() || nt != p.get_ntime())
                        throw Invalid_Parameters("initialConf has another lattice size than nSpace / nTime");
                    if (status == 0 && !p.get_ignore_checksum_errors())
                        throw Error(C2Q_BAD_ARG, "checksum of " + p.get_sourcefile() + " does not match");
                } else {
                    throw Invalid_Parameters("startCondition hot needs the reference's PRNG, outside this library");
                }
                upload(aos.data());
            }
            Gaugefield(const hardware::System& system, const double* aos) : system_(system)
            {
                create();
                upload(aos);
            }
            ~Gaugefield() { c2q_gauge_destroy(g_); }
            Gaugefield(const Gaugefield&)            = delete;
            Gaugefield& operator=(const Gaugefield&) = delete;
            void upload(const double* aos) { detail::check(c2q_gauge_upload(g_, aos), system_.ctx(), "gauge upload"); }
            const c2q_gauge* get() const noexcept { return g_; }
            const hardware::System& system() const noexcept { return system_; }

          private:
            void create()
            {
                const c2q_lattice lat = lattice_of(system_.get_inputparameters());
                detail::check(c2q_gauge_create(system_.ctx(), &lat, &g_), system_.ctx(), "c2q_gauge_create");
            }
            long long vol() const
            {
                const meta::Inputparameters& p = system_.get_inputparameters();
                return (long long)p.get_nspace() * p.get_nspace() * p.get_nspace() * p.get_ntime();
            }
            const hardware::System& system_;
            c2q_gauge* g_ = nullptr;
        };

        class Spinorfield_eo {
          public:
            explicit Spinorfield_eo(const hardware::System& system) : system_(system)
            {
                const c2q_lattice lat = lattice_of(system.get_inputparameters());
                detail::check(c2q_spinor_eo_create(system.ctx(), &lat, &f_), system.ctx(), "c2q_spinor_eo_create");
            }
            ~Spinorfield_eo() { c2q_spinor_eo_destroy(f_); }
            Spinorfield_eo(const Spinorfield_eo&)            = delete;
            Spinorfield_eo& operator=(const Spinorfield_eo&) = delete;
            size_t get_elements() const
            {
                const meta::Inputparameters& p = system_.get_inputparameters();
                return (size_t)p.get_nspace() * p.get_nspace() * p.get_nspace() * p.get_ntime() / 2;
            }
            /* Spinor::load / dump: spinor[Seo], 24 doubles each, eo index order */
            void load(const double* aos) const
            {
                detail::check(c2q_spinor_eo_upload(f_, aos), system_.ctx(), "spinor upload");
            }
            void dump(double* aos) const
            {
                detail::check(c2q_spinor_eo_download(f_, aos), system_.ctx(), "spinor download");
            }
            void zero() const { detail::check(c2q_spinor_eo_zero(f_), system_.ctx(), "zero"); }
            void cold() const { detail::check(c2q_spinor_eo_cold(f_), system_.ctx(), "cold"); }
            c2q_spinor_eo* get() const noexcept { return f_; }
            const hardware::System& system() const noexcept { return system_; }

          private:
            const hardware::System& system_;
            c2q_spinor_eo* f_ = nullptr;
        };

        /* A full lattice field, held as its two parities on the device. */
        class Spinorfield {
          public:
            explicit Spinorfield(const hardware::System& system) : even_(system), odd_(system) {}
            size_t get_elements() const { return 2 * even_.get_elements(); }
            void load(const double* full) const
            {
                detail::check(c2q_convert_to_eoprec(even_.get(), odd_.get(), full), even_.system().ctx(), "load");
            }
            void dump(double* full) const
            {
                detail::check(c2q_convert_from_eoprec(full, even_.get(), odd_.get()), even_.system().ctx(), "dump");
            }
            const Spinorfield_eo& even() const noexcept { return even_; }
            const Spinorfield_eo& odd() const noexcept { return odd_; }

          private:
            Spinorfield_eo even_, odd_;
        };

        inline hmc_float squarenorm(const Spinorfield_eo& x)
        {
            double r = 0;
            detail::check(c2q_squarenorm(x.get(), &r), x.system().ctx(), "squarenorm");
            return r;
        }
    }  // namespace lattices

    namespace fermionmatrix {
        class Fermionmatrix_eo {
          public:
            virtual ~Fermionmatrix_eo() {}
            virtual void operator()(const lattices::Spinorfield_eo* out, const lattices::Gaugefield& gf,
                                    const lattices::Spinorfield_eo& in,
                                    const AdditionalParameters& additionalParameters) const
            {
                detail::check(c2q_apply_eo(op_, out->get(), gf.get(), in.get(), additionalParameters.getKappa(),
                                           additionalParameters.getMubar(), action_, merged_),
                              system_.ctx(), "fermion matrix");
            }
            bool isHermitian() const noexcept { return herm_; }
            int op() const noexcept { return op_; }
            int action() const noexcept { return action_; }

          protected:
            Fermionmatrix_eo(bool herm, const hardware::System& system, int op)
                : system_(system), herm_(herm), op_(op),
                  action_(system.get_inputparameters().get_fermact()),
                  merged_(system.get_inputparameters().get_use_merge_kernels_fermion() ? 1 : 0)
            {
            }

          private:
            const hardware::System& system_;
            bool herm_;
            int op_, action_, merged_;
        };
#define C2Q_EO_MATRIX(NAME, HERM, OP)                                                                      \
    class NAME : public Fermionmatrix_eo {                                                                 \
      public:                                                                                              \
        explicit NAME(const hardware::System& system) : Fermionmatrix_eo(HERM, system, OP) {}              \
        NAME(const hardware::System& system, const InterfacesHandler&) : Fermionmatrix_eo(HERM, system, OP) {} \
    };
        C2Q_EO_MATRIX(Aee, false, C2Q_OP_AEE)
        C2Q_EO_MATRIX(Aee_minus, false, C2Q_OP_AEE_MINUS)
        C2Q_EO_MATRIX(Qplus_eo, false, C2Q_OP_QPLUS_EO)
        C2Q_EO_MATRIX(Qminus_eo, false, C2Q_OP_QMINUS_EO)
        C2Q_EO_MATRIX(QplusQminus_eo, true, C2Q_OP_QPLUSQMINUS_EO)
#undef C2Q_EO_MATRIX
    }  // namespace fermionmatrix

    namespace algorithms {
        namespace solvers {
            class SolverException : public std::runtime_error {
              public:
                int get_iterations() const noexcept { return iterations_; }

              protected:
                SolverException(const std::string& message, int iterations)
                    : std::runtime_error(message), iterations_(iterations)
                {
                }

              private:
                int iterations_;
            };
            class SolverStuck : public SolverException {
              public:
                explicit SolverStuck(int iterations, const std::string& why = "Solver got stuck.")
                    : SolverException(why, iterations)
                {
                }
            };
            class SolverDidNotSolve : public SolverException {
              public:
                explicit SolverDidNotSolve(int iterations) : SolverException("Solver did not solve.", iterations) {}
            };

            namespace detail_ {
                inline int finish(int rc, const c2q_solve_report& rep, c2q_ctx* ctx)
                {
                    if (rc == C2Q_SOLVER_STUCK)
                        throw SolverStuck(rep.iterations, ctx && c2q_last_error(ctx) ? c2q_last_error(ctx) : "");
                    if (rc == C2Q_DID_NOT_SOLVE) throw SolverDidNotSolve(rep.iterations);
                    if (rc < 0) cl2qcd_b200::detail::check(rc, ctx, "solver");
                    return rc;
                }
            }  // namespace detail_

            /* Solves A x = b (x holds the start vector); returns the iterations
             * performed, throws SolverStuck / SolverDidNotSolve.  The limits
             * come from interfacesHandler; prec is the stopping threshold on
             * |r|^2.  `report` (optional) receives the library's report. */
            inline int cg(const lattices::Spinorfield_eo* x, const fermionmatrix::Fermionmatrix_eo& A,
                          const lattices::Gaugefield& gf, const lattices::Spinorfield_eo& b,
                          const hardware::System& system, InterfacesHandler& interfacesHandler, hmc_float prec,
                          const AdditionalParameters& additionalParameters, c2q_solve_report* report = nullptr)
            {
                c2q_solver_params P = interfacesHandler.solver_parameters();
                P.solver            = C2Q_SOLVER_CG;
                P.prec              = prec;
                c2q_solve_report rep{};
                const int rc = c2q_cg(x->get(), A.op(), gf.get(), b.get(), additionalParameters.getKappa(),
                                      additionalParameters.getMubar(), A.action(), &P, &rep);
                if (report) *report = rep;
                return detail_::finish(rc, rep, system.ctx());
            }
            inline int bicgstab(const lattices::Spinorfield_eo* x, const fermionmatrix::Fermionmatrix_eo& A,
                                const lattices::Gaugefield& gf, const lattices::Spinorfield_eo& b,
                                const hardware::System& system, InterfacesHandler& interfacesHandler, hmc_float prec,
                                const AdditionalParameters& additionalParameters,
                                c2q_solve_report* report = nullptr)
            {
                c2q_solver_params P = interfacesHandler.solver_parameters();
                if (P.solver != C2Q_SOLVER_BICGSTAB_SAVE) P.solver = C2Q_SOLVER_BICGSTAB;
                P.prec = prec;
                c2q_solve_report rep{};
                const int rc = c2q_bicgstab(x->get(), A.op(), gf.get(), b.get(), additionalParameters.getKappa(),
                                            additionalParameters.getMubar(), A.action(), &P, &rep);
                if (report) *report = rep;
                return detail_::finish(rc, rep, system.ctx());
            }
        }  // namespace solvers

        /* perform_inversion (inversion.cpp:44-242): result[k] = M^-1-type solution
         * of sources[k] with the input parameters' solver, useEO branch and
         * the reference's sign conventions. */
        inline void perform_inversion(const std::vector<lattices::Spinorfield*>* result,
                                      const lattices::Gaugefield* gaugefield,
                                      const std::vector<lattices::Spinorfield*>& sources,
                                      const hardware::System& system, InterfacesHandler& interfacesHandler)
        {
            const meta::Inputparameters& p = interfacesHandler.parameters();
            const c2q_solver_params P      = interfacesHandler.solver_parameters();
            if (!result || result->size() != sources.size())
                throw Invalid_Parameters("perform_inversion: one result field per source");
            for (size_t k = 0; k < sources.size(); ++k) {
                std::vector<double> src(sources[k]->get_elements() * 24), out(src.size());
                sources[k]->dump(src.data());
                c2q_solve_report rep{};
                int rc;
                if (p.get_use_eo()) {
                    rc = c2q_perform_inversion_eo_fields(system.ctx(), (*result)[k]->even().get(),
                                                         (*result)[k]->odd().get(), gaugefield->get(), src.data(),
                                                         p.get_kappa(), meta::get_mubar(p), p.get_fermact(), &P, &rep);
                } else {
                    rc = c2q_perform_inversion_full(system.ctx(), out.data(), gaugefield->get(), src.data(),
                                                    p.get_kappa(), meta::get_mubar(p), p.get_fermact(), &P, &rep);
                    if (rc >= 0) (*result)[k]->load(out.data());
                }
                solvers::detail_::finish(rc, rep, system.ctx());
            }
        }
    }  // namespace algorithms

    namespace observables {
        namespace wilson {
            /* The pseudoscalar correlator ("ps") of point-source solutions, along
             * correlatorDirection (0: t, 3: z). */
            inline std::vector<hmc_float> calculate_correlator(const std::string& type,
                                                               const std::vector<lattices::Spinorfield*>& corr,
                                                               const std::vector<lattices::Spinorfield*>& /*sources*/,
                                                               const hardware::System& system,
                                                               InterfacesHandler& interfacesHandler)
            {
                if (type != "ps") throw Invalid_Parameters("correlator type " + type + " is outside this library");
                const meta::Inputparameters& p = interfacesHandler.parameters();
                std::vector<c2q_spinor_eo*> ev, od;
                for (auto* f : corr) {
                    ev.push_back(f->even().get());
                    od.push_back(f->odd().get());
                }
                std::vector<hmc_float> out(p.get_corr_dir() == 0 ? p.get_ntime() : p.get_nspace());
                cl2qcd_b200::detail::check(c2q_correlator_ps(ev.data(), od.data(), (int)corr.size(), p.get_kappa(),
                                                             p.get_corr_dir(), out.data()),
                                           system.ctx(), "correlator");
                return out;
            }
        }  // namespace wilson
    }      // namespace observables
}  // namespace physics

}  // namespace cl2qcd_b200

#endif
