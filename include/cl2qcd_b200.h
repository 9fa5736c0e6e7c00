/*
 * cl2qcd_b200.h -- C ABI of the B200-native twisted-mass Wilson even-odd
 * inverter hot path (CL2QCD's dslash_eo / M_tm sitediagonal / eo BLAS /
 * CG / BiCGStab / eo inversion), implemented in hand-written sm_100a CUDA.
 *
 * Plain C: opaque handles, plain pointers and sizes, integer status codes.
 * Every entry point names the reference interface it replaces (file:line in
 * the CL2QCD tree).
 *
 * Host data formats are the reference's:
 *   eo spinor field : double[Seo][24], eo index order (site/2), each spinor
 *                     [spin 0..3][colour 0..2][re, im]
 *                     (common_header_files/types_fermions.hpp:31-55,
 *                      hardware/buffers/spinor.cpp:83-106);
 *   full spinor     : double[V][24] in site order x + NS y + NS^2 z + NS^3 t
 *                     (geometry/index.cpp:46-70);
 *   gauge field     : double[4 V][18], Matrixsu3 at link mu + 4*site with
 *                     TDIR = 0, XDIR = 1, YDIR = 2, ZDIR = 3, row-major
 *                     (re, im) (hardware/code/gaugefield.cpp:533,
 *                      geometry/latticeExtents.hpp:28).
 *
 * Threading: one CUDA stream per context; calls on a context are ordered on
 * that stream.  Calls that return host scalars or reports synchronise the
 * stream.  A context is thread-compatible (one host thread at a time), not
 * thread-safe.  Different contexts may be used from different threads.
 */
#ifndef CL2QCD_B200_H
#define CL2QCD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define C2Q_EXPORT __attribute__((visibility("default")))
#else
#define C2Q_EXPORT
#endif

/* ---- status codes (the C++ mirror maps them back to the reference's
 *      exception types, physics/algorithms/solvers/exceptions.hpp:35-62) ---- */
#define C2Q_OK 0
#define C2Q_SOLVER_STUCK -1   /* SolverStuck: NaN residual or |rho| < 1e-25 */
#define C2Q_DID_NOT_SOLVE -2  /* SolverDidNotSolve: iteration limit reached */
#define C2Q_TIMEOUT -3
#define C2Q_OOM -4
#define C2Q_BAD_ARG -5        /* Invalid_Parameters / std::invalid_argument */
#define C2Q_CUDA_ERROR -6
#define C2Q_NO_DEVICE -7

/* evenodd argument of c2q_dslash_eo, with the reference's meaning
 * (common_header_files/globaldefs.hpp:38-39; ocl_kernel/fermionmatrix_eo_dslash.cl:50-58):
 * ODD writes the sites with x+y+z+t even, EVEN writes the odd sites. */
#define C2Q_EVEN 0
#define C2Q_ODD 1

/* fermion actions (common_header_files/types.hpp:198, the subset on this path) */
#define C2Q_ACTION_WILSON 1
#define C2Q_ACTION_TWISTEDMASS 3

/* eo fermion matrices (physics/fermionmatrix/fermionmatrix.hpp:194-310) */
#define C2Q_OP_AEE 0
#define C2Q_OP_AEE_MINUS 1
#define C2Q_OP_QPLUS_EO 2
#define C2Q_OP_QMINUS_EO 3
#define C2Q_OP_QPLUSQMINUS_EO 4
#define C2Q_OP_AEE_AND_GAMMA5_EO 5
#define C2Q_OP_AEE_MINUS_AND_GAMMA5_EO 6

/* site-diagonal tm factors (physics/fermionmatrix/fermionmatrix.hpp:50-57;
 * ocl_kernel/fermionmatrix_eo_m.cl:22-109, fermionmatrix_eo_m_merged.cl:22-64) */
#define C2Q_DIAG_M_TM 0              /* M_tm_sitediagonal:               1 + i mubar g5 */
#define C2Q_DIAG_M_TM_INVERSE 1      /* M_tm_inverse_sitediagonal:       (1 - i mubar g5)/(1+mubar^2) */
#define C2Q_DIAG_M_TM_MINUS 2        /* M_tm_sitediagonal_minus:         1 - i mubar g5 */
#define C2Q_DIAG_M_TM_INVERSE_MINUS 3/* M_tm_inverse_sitediagonal_minus: (1 + i mubar g5)/(1+mubar^2) */
#define C2Q_DIAG_M_TM_AND_GAMMA5 4   /* M_tm_sitediagonal_AND_gamma5_eo */
#define C2Q_DIAG_M_TM_MINUS_AND_GAMMA5 5

/* solvers (common_header_files/types.hpp:199 common::solver) */
#define C2Q_SOLVER_CG 1
#define C2Q_SOLVER_BICGSTAB 2
#define C2Q_SOLVER_BICGSTAB_SAVE 3

/* inner precision of the Krylov iteration */
#define C2Q_PREC_FP64 64   /* plain FP64, the reference's arithmetic */
#define C2Q_PREC_FP32 32   /* FP32 inner solve inside FP64 reliable updates */
#define C2Q_PREC_FP16 16   /* FP16 fixed-point spinors (per-site norm) + FP32 arithmetic, FP64 reliable updates */

typedef struct c2q_ctx c2q_ctx;
typedef struct c2q_gauge c2q_gauge;
typedef struct c2q_spinor_eo c2q_spinor_eo;

/* Lattice and boundary conditions.  Replaces the lattice/BC parameters the
 * reference bakes into its kernels as build options
 * (hardware/code/opencl_module.cpp:61-224; meta/parametersFermion.cpp:106-150):
 * nSpace, nTime, thetaFermionTemporal/Spatial (units of pi; phase theta*pi/N
 * on every hop), useChemicalPotentialRe/Im and chemicalPotentialRe/Im. */
typedef struct {
    int ns, nt;            /* both even */
    double theta_t, theta_s;
    int use_cp_re, use_cp_im;
    double cp_re, cp_im;
} c2q_lattice;

/* Solver parameters.  Replaces SolversParametersInterface
 * (physics/algorithms/algorithmsInterfaces.hpp:28-37; defaults of
 * meta/parametersSolver.cpp:74-107). */
typedef struct {
    int solver;               /* C2Q_SOLVER_* (solver) */
    double prec;              /* solverPrecision: stop when |r|^2 < prec (absolute, reference semantics); <= 0 disables */
    double rel_tol;           /* additionally stop when ||b - A x|| / ||b|| <= rel_tol (true residual); <= 0 disables */
    int cgmax;                /* solverMaxIterations */
    int iter_refresh;         /* solverRestartEvery */
    int resid_check_every;    /* solverResiduumCheckEvery (CG) */
    int min_iter;             /* solverMinIterations (CG) */
    int precision;            /* C2Q_PREC_*: inner arithmetic */
    double reliable_delta;    /* mixed precision: reliable update when |r_inner| < delta * max|r| since the last one (default 0.003) */
    int use_rec12;            /* inner operator uses 12-real links */
    int use_graph;            /* CG: replay the iterations between residual refreshes as a captured CUDA graph */
    int use_temporal_gauge;   /* mixed precision on QplusQminus_eo: inner iterations on the field in the
                                 temporal gauge (T links the identity but on the last slice), where the
                                 T weights are pure phases and the spatial ones real (default 1) */
} c2q_solver_params;

/* What a solve reports (replaces the reference's log lines,
 * physics/algorithms/solvers/cg.cpp:195-275). */
typedef struct {
    int status;               /* >= 0 iterations, else C2Q_* status */
    int iterations;           /* inner Krylov iterations */
    int reliable_updates;     /* FP64 residual recomputations (mixed precision) */
    double resid_sq;          /* last iterated |r|^2 */
    double true_resid_rel;    /* ||b - A x|| / ||b|| recomputed in FP64 at the end */
    double seconds;           /* device time of the solve (CUDA events) */
    double dslash_applications; /* dslash launches (each = one parity sweep over the lattice) */
} c2q_solve_report;

/* ---------------- input parameters ----------------
 * The reference's input-file keys of the inverter path (meta::Inputparameters,
 * meta/inputparameters.cpp:150-196, read by boost's parse_config_file):
 *   nSpace, nTime, precision, useReconstruct12, startCondition, initialConf,
 *   ignoreChecksumErrors (meta/parametersConfig.cpp:147-187);
 *   fermionAction, kappa, mu, thetaFermionSpatial/Temporal,
 *   useChemicalPotentialRe/Im, chemicalPotentialRe/Im, useEO,
 *   useKernelMergingFermionMatrix/Spinor (meta/parametersFermion.cpp:106-150);
 *   solver, solverPrecision, solverMaxIterations, solverMinIterations,
 *   solverRestartEvery, solverResiduumCheckEvery (meta/parametersSolver.cpp:74-107);
 *   sourceType, sourceContent, nSources, sourceX/Y/Z/T
 *   (meta/parametersSources.cpp:67-90); measureCorrelators,
 *   correlatorDirection (meta/parametersObs.cpp:67-86);
 * with the aliases NS, NT, use_evenodd, ThetaT, ThetaS
 * (meta/inputparameters.cpp:180-193) and mubar = 2 kappa mu (meta/util.cpp:56-59).
 * Keys of this library, without a counterpart in the reference, sit in the
 * section [b200]: innerPrecision (64, 32, 16), relativeTolerance,
 * reliableDelta, useGraph, temporalGauge. */
#define C2Q_START_COLD 0      /* startCondition cold / cold_start */
#define C2Q_START_HOT 1       /* hot / hot_start */
#define C2Q_START_CONTINUE 2  /* continue / source / start_from_source */
#define C2Q_SOURCE_POINT 0    /* sourceType (common::sourcetypes) */
#define C2Q_SOURCE_VOLUME 1
#define C2Q_SOURCE_TIMESLICE 2
#define C2Q_SOURCE_ZSLICE 3
#define C2Q_CONTENT_ONE 0     /* sourceContent (common::sourcecontents) */
#define C2Q_CONTENT_Z4 1
#define C2Q_CONTENT_GAUSSIAN 2
#define C2Q_CONTENT_Z2 3
typedef struct {
    c2q_lattice lat;              /* nSpace, nTime, thetaFermion*, chemical potential */
    int fermion_action;           /* fermionAction as common::action: C2Q_ACTION_WILSON (1), clover (2),
                                     C2Q_ACTION_TWISTEDMASS (3), rooted_stagg (7); the fermion
                                     matrices here take the wilson and twisted-mass actions */
    double kappa, mu;             /* kappa, mu */
    double mubar;                 /* 2 kappa mu */
    int use_eo;                   /* useEO */
    int precision;                /* precision in bits (64 or 32; this library's FP64 path needs 64) */
    int use_merge_kernels_fermion, use_merge_kernels_spinor;
    c2q_solver_params solver;     /* solver keys; use_rec12 = useReconstruct12; [b200] keys */
    int start_condition;          /* C2Q_START_* */
    char initial_conf[1024];      /* initialConf */
    int ignore_checksum_errors;   /* ignoreChecksumErrors */
    int source_type, source_content, n_sources;
    int source_pos[4];            /* sourceX, sourceY, sourceZ, sourceT */
    int measure_correlators;      /* measureCorrelators */
    int correlator_direction;     /* correlatorDirection (0 = t .. 3 = z; c2q_correlator_ps takes 0 and 3) */
} c2q_params;
/* The reference's defaults (the constructors of meta/parameters*.cpp). */
C2Q_EXPORT void c2q_params_default(c2q_params* p);
/* Parses input-file text onto p (start from c2q_params_default; a second call
 * overrides what the first set, as the reference's command-line options
 * override its input file).  Format of parse_config_file: `name = value` per
 * line, `#` comments, `[section]` headers; unknown names and a name given twice
 * are errors; every other key the reference defines (HMC, RHMC, gauge, I/O) is
 * accepted and ignored.  Returns C2Q_OK, or C2Q_BAD_ARG with p unchanged and the
 * reason in c2q_params_last_error() (per thread). */
C2Q_EXPORT int c2q_params_from_kv(const char* key_value_text, c2q_params* p);
C2Q_EXPORT const char* c2q_params_last_error(void);

/* ---------------- context ---------------- */
/* Creates a context on `device`.  `cuda_stream` (a cudaStream_t) is borrowed
 * if non-NULL, else the context creates its own.  Replaces hardware::System /
 * hardware::Device (hardware/system.cpp:117-200, hardware/device.cpp:79). */
C2Q_EXPORT int c2q_ctx_create(c2q_ctx** out, int device, void* cuda_stream);
/* Every gauge and spinor object created on a context must be destroyed before
 * the context (they use its stream). */
C2Q_EXPORT int c2q_ctx_destroy(c2q_ctx* ctx);
C2Q_EXPORT const char* c2q_last_error(const c2q_ctx* ctx);
C2Q_EXPORT int c2q_ctx_synchronize(c2q_ctx* ctx);
/* Kernels this library launched on the context since creation (all of them are this library's own). */
C2Q_EXPORT long long c2q_ctx_launch_count(const c2q_ctx* ctx);
/* Per-launch timing of the dslash sweeps with CUDA events on the context's
 * stream (off by default; replaces the reference's enableProfiling,
 * hardware/device.cpp:181-241).  c2q_ctx_profile(ctx, 1) clears and starts;
 * c2q_ctx_profile_read synchronises and returns, for sweeps of storage
 * precision `prec` (64, 32, 16), the number of timed launches, their summed
 * device time in milliseconds and their summed algorithmic bytes (per output
 * site: 8 links, the input and output spinors, and the spinors an epilogue or
 * a fused reduction reads at the output site). */
C2Q_EXPORT int c2q_ctx_profile(c2q_ctx* ctx, int enable);
C2Q_EXPORT int c2q_ctx_profile_read(c2q_ctx* ctx, int prec, long long* launches, double* total_ms,
                                    double* bytes);

/* ---------------- gauge field ---------------- */
/* Gaugefield device layout + import (physics/lattices/gaugefield.hpp:44-139;
 * hardware/code/gaugefield.cpp:533 importGaugefield).  `aos` is Matrixsu3[4V]. */
C2Q_EXPORT int c2q_gauge_create(c2q_ctx* ctx, const c2q_lattice* lat, c2q_gauge** out);
C2Q_EXPORT int c2q_gauge_upload(c2q_gauge* g, const double* aos);
C2Q_EXPORT int c2q_gauge_download(const c2q_gauge* g, double* aos);
C2Q_EXPORT int c2q_gauge_destroy(c2q_gauge* g);
/* Device bytes held by the gauge object (all precisions built so far). */
C2Q_EXPORT size_t c2q_gauge_device_bytes(const c2q_gauge* g);
/* FP64 unitarity of the uploaded links, measured on the device (no
 * counterpart in the reference, which takes SU(3) for granted wherever it
 * reconstructs a link): dev[0] = max over links of max_ij |(U U^dagger - 1)_ij|,
 * dev[1] = max |det U - 1|, dev[2] = max_j |U_2j - conj(row0 x row1)_j| (what
 * 12-real storage changes).  Non-finite links give infinity.  The solvers use
 * 12-real FP64 links for intermediate residuals only when dev[2] <= 1e-13; the
 * residual that stops a mixed-precision solve, and every reported true
 * residual, use the links as uploaded. */
C2Q_EXPORT int c2q_gauge_unitarity(const c2q_gauge* g, double* dev);
/* project_su3 (ocl_kernel/operations_gaugefield.cl:135-240; applied by the
 * reference after every link update, md_update_gaugefield.cl:44) on every link,
 * in FP64 on the device, in place: column 0 normalised, column 1
 * orthogonalised against it and normalised, column 2 = conj(col0 x col1).
 * dev_before (may be NULL) receives c2q_gauge_unitarity's dev[0] before the
 * projection.  Copies derived from the links are rebuilt on next use. */
C2Q_EXPORT int c2q_gauge_reunitarize(c2q_gauge* g, double* dev_before);

/* ---------------- eo spinor fields ---------------- */
/* physics::lattices::Spinorfield_eo (physics/lattices/spinorfield_eo.hpp:48-305). */
C2Q_EXPORT int c2q_spinor_eo_create(c2q_ctx* ctx, const c2q_lattice* lat, c2q_spinor_eo** out);
C2Q_EXPORT int c2q_spinor_eo_destroy(c2q_spinor_eo* f);
/* Spinor::load / dump (hardware/buffers/spinor.cpp:83-106): spinor[Seo] in eo index order. */
C2Q_EXPORT int c2q_spinor_eo_upload(c2q_spinor_eo* f, const double* aos);
C2Q_EXPORT int c2q_spinor_eo_download(const c2q_spinor_eo* f, double* aos);
/* (no counterpart in the reference: its Spinor::load / dump wait) The same
 * transfers enqueued without waiting, FP64 fields only, on `stream` (a
 * cudaStream_t of the same device; NULL: the context's stream).  The host array
 * must stay valid, and a download's must not be read, until the stream has
 * passed the copy.  With pinned host memory and a copy stream ordered against
 * the context's stream by events, the transfers of one solve overlap another
 * solve.  The context's transfers share one staging buffer: keep them on one
 * stream (or order them by events). */
C2Q_EXPORT int c2q_spinor_eo_upload_async(c2q_spinor_eo* f, const double* aos, void* stream);
C2Q_EXPORT int c2q_spinor_eo_download_async(const c2q_spinor_eo* f, double* aos, void* stream);
/* Spinorfield_eo::zero / cold (physics/lattices/spinorfield_eo.cpp:147-165) */
C2Q_EXPORT int c2q_spinor_eo_zero(c2q_spinor_eo* f);
C2Q_EXPORT int c2q_spinor_eo_cold(c2q_spinor_eo* f);
/* Reduced-precision eo fields (no counterpart in the reference, which is FP64
 * only; CMakeLists.txt:127-132): C2Q_PREC_FP32 or C2Q_PREC_FP16 storage, the
 * inner fields of the mixed-precision solvers.  NT must be a multiple of 4
 * (the device layout pairs the sites at t and t + NT/2).  upload / download /
 * zero / BLAS / the explicit operators accept them; upload rounds on the device.
 * Fields passed together to one call must have the same precision. */
C2Q_EXPORT int c2q_spinor_eo_create_precision(c2q_ctx* ctx, const c2q_lattice* lat, int precision,
                                              c2q_spinor_eo** out);
C2Q_EXPORT int c2q_spinor_eo_precision(const c2q_spinor_eo* f);
/* out = in, rounded (or widened) to out's precision. */
C2Q_EXPORT int c2q_spinor_eo_convert(c2q_spinor_eo* out, const c2q_spinor_eo* in);
/* Link storage the explicit operator calls (dslash, dslash_AND_M_tm_inverse_sitediagonal,
 * apply_eo) read: 0 = 18-real (the reference's), 1 = 12-real with row-2
 * reconstruction.  FP16 operators always use 12-real FP16 links. */
C2Q_EXPORT int c2q_ctx_set_link_format(c2q_ctx* ctx, int rec12);
/* Autotuner of the reduced-precision sweeps (no counterpart in the reference):
 * on by default (environment C2Q_AUTOTUNE=0 turns it off for new contexts);
 * the first sweep of each launch shape times the kernel's launch
 * configurations and keeps the fastest.  tune_report writes one line per
 * shape into buf (NUL-terminated, truncated to len) and returns the length
 * needed including the NUL. */
C2Q_EXPORT int c2q_ctx_set_autotune(c2q_ctx* ctx, int enable);
/* (no counterpart in the reference) Pins the launch choice of every
 * reduced-precision sweep on the context instead of the autotuner's: 0..3 =
 * launch configuration (choice & 1) with one block per tile (choice >> 1 = 0)
 * or a grid-stride grid (1); 4 = two right-hand sides per thread, for FP16
 * batches of two or more in the temporal gauge (elsewhere choice 0); -1 = the
 * autotuner decides (default).  Every choice gives bitwise the same results. */
C2Q_EXPORT int c2q_ctx_set_sweep_choice(c2q_ctx* ctx, int choice);
C2Q_EXPORT int c2q_ctx_tune_report(const c2q_ctx* ctx, char* buf, int len);
/* convert_to_eoprec / convert_from_eoprec (physics/lattices/spinorfield_eo.cpp:372-410):
 * `full` is a host spinor[V]; `even` gets the sites with x+y+z+t even (FP64 fields). */
C2Q_EXPORT int c2q_convert_to_eoprec(c2q_spinor_eo* even, c2q_spinor_eo* odd, const double* full);
C2Q_EXPORT int c2q_convert_from_eoprec(double* full, const c2q_spinor_eo* even, const c2q_spinor_eo* odd);

/* ---------------- explicit fermion operations ---------------- */
/* physics::fermionmatrix::dslash (physics/fermionmatrix/explicit.cpp:185-222) */
C2Q_EXPORT int c2q_dslash_eo(c2q_spinor_eo* out, const c2q_gauge* g, const c2q_spinor_eo* in, int evenodd,
                             double kappa);
/* Fermions::dslash_AND_M_tm_inverse_sitediagonal(_minus)_eo_device (hardware/code/fermions.cpp:550-623) */
C2Q_EXPORT int c2q_dslash_AND_M_tm_inverse_sitediagonal_eo(c2q_spinor_eo* out, const c2q_gauge* g,
                                                           const c2q_spinor_eo* in, int evenodd, double kappa,
                                                           double mubar, int minus);
/* M_tm_(inverse_)sitediagonal(_minus) (physics/fermionmatrix/explicit.cpp:88-183) and the merged
 * M_tm_sitediagonal(_minus)_AND_gamma5_eo (hardware/code/fermions.cpp): `which` = C2Q_DIAG_* */
C2Q_EXPORT int c2q_tm_sitediagonal(c2q_spinor_eo* out, const c2q_spinor_eo* in, double mubar, int which);
/* Spinorfield_eo::gamma5 (physics/lattices/spinorfield_eo.cpp:412-418) */
C2Q_EXPORT int c2q_gamma5_eo(c2q_spinor_eo* inout);

/* Fermionmatrix_eo::operator() (physics/fermionmatrix/fermionmatrix.hpp:121-136,
 * fermionmatrix.cpp:224-664): out = A(in) for op = C2Q_OP_*, action = C2Q_ACTION_*.
 * `merged` = useKernelMergingFermionMatrix (fermionmatrix.cpp:596). */
C2Q_EXPORT int c2q_apply_eo(int op, c2q_spinor_eo* out, const c2q_gauge* g, const c2q_spinor_eo* in, double kappa,
                            double mubar, int action, int merged);
/* Full-lattice (non-eo) fermion matrices (physics/fermionmatrix/fermionmatrix.cpp:41-222,
 * explicit.cpp:36-87) on a field held as its two parities: M_tm_plus / M_tm_minus
 * (= M_wilson for the Wilson action), Qplus / Qminus = g5 M_tm_plus / minus,
 * QplusQminus = Qplus Qminus.  The output must not alias the input. */
#define C2Q_FULL_M_TM_PLUS 0
#define C2Q_FULL_M_TM_MINUS 1
#define C2Q_FULL_QPLUS 2
#define C2Q_FULL_QMINUS 3
#define C2Q_FULL_QPLUSQMINUS 4
C2Q_EXPORT int c2q_apply_full(int op, c2q_spinor_eo* out_even, c2q_spinor_eo* out_odd, const c2q_gauge* g,
                              const c2q_spinor_eo* in_even, const c2q_spinor_eo* in_odd, double kappa, double mubar,
                              int action);

/* ---------------- eo BLAS (physics/lattices/spinorfield_eo.hpp:148-305) ---------------- */
C2Q_EXPORT int c2q_saxpy(c2q_spinor_eo* out, double alpha_re, double alpha_im, const c2q_spinor_eo* x,
                         const c2q_spinor_eo* y);                         /* out = y - alpha x */
C2Q_EXPORT int c2q_saxpy_AND_gamma5_eo(c2q_spinor_eo* out, double alpha_re, double alpha_im,
                                       const c2q_spinor_eo* x, const c2q_spinor_eo* y); /* out = g5 (y - alpha x) */
C2Q_EXPORT int c2q_sax(c2q_spinor_eo* out, double alpha_re, double alpha_im, const c2q_spinor_eo* x);
C2Q_EXPORT int c2q_saxsbypz(c2q_spinor_eo* out, double alpha_re, double alpha_im, const c2q_spinor_eo* x,
                            double beta_re, double beta_im, const c2q_spinor_eo* y, const c2q_spinor_eo* z);
C2Q_EXPORT int c2q_copyData(c2q_spinor_eo* to, const c2q_spinor_eo* from);
C2Q_EXPORT int c2q_scalar_product(const c2q_spinor_eo* x, const c2q_spinor_eo* y, double* re, double* im);
C2Q_EXPORT int c2q_squarenorm(const c2q_spinor_eo* x, double* result);
C2Q_EXPORT int c2q_saxpy_AND_squarenorm(c2q_spinor_eo* out, double alpha_re, double alpha_im,
                                        const c2q_spinor_eo* x, const c2q_spinor_eo* y, double* squarenorm);

/* Scalar product sum conj(x) y of two FP64 eo spinor fields, for callers that
 * cannot allocate device memory (their memory pool owns the GPU, they cannot
 * afford the synchronisation an allocation may cause, or their host program
 * forbids plugins from allocating).  No counterpart in the reference: it is an
 * addition of this library.
 *   x_soa, y_soa : caller-owned device buffers in the library's FP64 field
 *                  layout: 12 complex lanes of double2, component k of site i
 *                  at element k*stride + i (stride >= n_sites);
 *   result_dev   : caller-owned device memory for 2 doubles (re, im);
 *   cuda_stream  : the cudaStream_t to run on (NULL = legacy default stream).
 * Asynchronous: the result is in result_dev when the stream reaches it.
 * Allocates nothing: the reduction scratch is a fixed array inside the library
 * (about 256 KiB per device, held until the process exits); more than
 * C2Q_NOALLOC_MAX_SITES sites is rejected with C2Q_BAD_ARG (and a message on
 * stderr), and so are x_soa / y_soa not 16-byte aligned or result_dev not
 * 8-byte aligned.  The first call on a device looks up the scratch's device
 * address, so make that call before any stream capture; the address is kept
 * for the life of the process, so a process that resets a device
 * (cudaDeviceReset) must not call this entry point on it afterwards.  Calls
 * share the scratch: calls that overlap on the GPU (other streams or host
 * threads) race. */
#define C2Q_NOALLOC_MAX_SITES 4194304
C2Q_EXPORT int c2q_scalar_product_eo_noalloc(const void* x_soa, const void* y_soa, int n_sites, int stride,
                                             double* result_dev, void* cuda_stream);

/* ---------------- solvers ---------------- */
C2Q_EXPORT void c2q_solver_params_default(c2q_solver_params* p);
/* solvers::cg (physics/algorithms/solvers/cg.hpp:41-56, cg.cpp:158-170, 277-400):
 * solves A x = b for op (normally C2Q_OP_QPLUSQMINUS_EO), x holds the start
 * vector on entry.  Returns iterations (>= 0) or C2Q_SOLVER_STUCK /
 * C2Q_DID_NOT_SOLVE / other status. */
C2Q_EXPORT int c2q_cg(c2q_spinor_eo* x, int op, const c2q_gauge* g, const c2q_spinor_eo* b, double kappa,
                      double mubar, int action, const c2q_solver_params* p, c2q_solve_report* report);
/* solvers::bicgstab (physics/algorithms/solvers/bicgstab.hpp:42-57, bicgstab.cpp:384-733);
 * p->solver selects the fast (C2Q_SOLVER_BICGSTAB) or save (C2Q_SOLVER_BICGSTAB_SAVE) variant.
 * With p->precision 32 or 16 (no counterpart in the reference): the BiCGStab
 * iteration on FP32 / FP16 fields and links with reliable updates (whenever its
 * iterated residual has dropped by reliable_delta, x takes the accumulated
 * increment in FP64 and the FP64 true residual replaces the iterated one; the
 * search direction and shadow residual are kept); the stopping test applies to
 * the FP64 true residual and report->reliable_updates counts the updates. */
C2Q_EXPORT int c2q_bicgstab(c2q_spinor_eo* x, int op, const c2q_gauge* g, const c2q_spinor_eo* b, double kappa,
                            double mubar, int action, const c2q_solver_params* p, c2q_solve_report* report);
/* Multi-right-hand-side CG on one operator: x[k], b[k] for k < nrhs (each
 * right-hand side converges on its own; the dslash reads each link once per
 * batch).  Same semantics per right-hand side as c2q_cg. */
C2Q_EXPORT int c2q_cg_multi(c2q_spinor_eo* const* x, int op, const c2q_gauge* g, const c2q_spinor_eo* const* b,
                            int nrhs, double kappa, double mubar, int action, const c2q_solver_params* p,
                            c2q_solve_report* reports);

/* physics::algorithms::perform_inversion, eo branch of invert_M_nf2_upperflavour
 * (physics/algorithms/inversion.cpp:44-76, 78-242), one source: `source` and
 * `result` are host full fields spinor[V].  Reproduces the reference
 * literally, including its parity-role swap (inversion.cpp:141-149) and sign
 * conventions (inversion.cpp:165-169, 204-221), which make the returned
 * field equal to -M^{-1} source. */
C2Q_EXPORT int c2q_perform_inversion_eo(c2q_ctx* ctx, double* result, const c2q_gauge* g, const double* source,
                                        double kappa, double mubar, int action, const c2q_solver_params* p,
                                        c2q_solve_report* report);
/* The same inversion with the result left on the device: out_even / out_odd
 * receive the sites with x+y+z+t even / odd of the full result (FP64 fields). */
C2Q_EXPORT int c2q_perform_inversion_eo_fields(c2q_ctx* ctx, c2q_spinor_eo* out_even, c2q_spinor_eo* out_odd,
                                               const c2q_gauge* g, const double* source, double kappa, double mubar,
                                               int action, const c2q_solver_params* p, c2q_solve_report* report);
/* Pseudoscalar correlator from point sources
 * (physics/observables/wilsonTwoFlavourCorrelators.cpp:162-415 with
 * ocl_kernel/fermionobservables/correlator_ps_point.cl correlator_ps_t / _z):
 * direction 0: out[t] = (2 kappa)^2 / NS^3 * sum_k sum_{x in slice t} |phi_k(x)|^2;
 * direction 3 (the reference's default correlatorDirection, meta/parametersObs.cpp:72):
 * out[z] = (2 kappa)^2 / (NS^2 NT) * sum_k sum_{x with that z} |phi_k(x)|^2,
 * over the n full solutions phi_k = (even[k], odd[k]); out is a host array of
 * NT (direction 0) or NS (direction 3) doubles. */
C2Q_EXPORT int c2q_correlator_ps(const c2q_spinor_eo* const* even, const c2q_spinor_eo* const* odd, int n,
                                 double kappa, int direction, double* out);

/* Full-lattice (useEO=false) solves: solvers::cg / bicgstab on
 * physics::lattices::Spinorfield (physics/algorithms/inversion.cpp:98-122), x
 * and b held as their two parities (c2q_convert_to_eoprec), op a C2Q_FULL_*
 * matrix; FP64, the reference's semantics, x holds the start vector. */
C2Q_EXPORT int c2q_cg_full(c2q_spinor_eo* x_even, c2q_spinor_eo* x_odd, int op, const c2q_gauge* g,
                           const c2q_spinor_eo* b_even, const c2q_spinor_eo* b_odd, double kappa, double mubar,
                           int action, const c2q_solver_params* p, c2q_solve_report* report);
C2Q_EXPORT int c2q_bicgstab_full(c2q_spinor_eo* x_even, c2q_spinor_eo* x_odd, int op, const c2q_gauge* g,
                                 const c2q_spinor_eo* b_even, const c2q_spinor_eo* b_odd, double kappa, double mubar,
                                 int action, const c2q_solver_params* p, c2q_solve_report* report);
/* perform_inversion, non-eo branch of invert_M_nf2_upperflavour (inversion.cpp:98-122):
 * cold start; solver CG: QplusQminus y = gamma5 source, result = Qminus y;
 * otherwise BiCGStab (p->solver fast / save) on M.  Host full fields spinor[V];
 * result = M^{-1} source. */
C2Q_EXPORT int c2q_perform_inversion_full(c2q_ctx* ctx, double* result, const c2q_gauge* g, const double* source,
                                          double kappa, double mubar, int action, const c2q_solver_params* p,
                                          c2q_solve_report* report);

/* ---------------- HMC callers of the eo solvers ----------------
 * Gauge momenta (physics::lattices::Gaugemomenta, physics/lattices/gaugemomenta.hpp):
 * 8 reals (the su(3) algebra element ae, common_header_files/types.hpp:178-188)
 * per link; host format ae[4 V] at link mu + 4 site, TDIR = 0. */
typedef struct c2q_gaugemomenta c2q_gaugemomenta;
C2Q_EXPORT int c2q_gaugemomenta_create(c2q_ctx* ctx, const c2q_lattice* lat, c2q_gaugemomenta** out);
C2Q_EXPORT int c2q_gaugemomenta_destroy(c2q_gaugemomenta* gm);
/* Gaugemomenta::zero (gaugemomentum_zero.cl) */
C2Q_EXPORT int c2q_gaugemomenta_zero(c2q_gaugemomenta* gm);
C2Q_EXPORT int c2q_gaugemomenta_upload(c2q_gaugemomenta* gm, const double* aos);
C2Q_EXPORT int c2q_gaugemomenta_download(const c2q_gaugemomenta* gm, double* aos);
/* squarenorm(const Gaugemomenta&) (gaugemomentum_squarenorm.cl): sum of e_k^2 over every link */
C2Q_EXPORT int c2q_gaugemomenta_squarenorm(const c2q_gaugemomenta* gm, double* out);
/* physics::algorithms::fermion_force(gm, Y, X, evenodd, gf, params) on eo fields
 * (physics/algorithms/fermion_force.cpp:699-730; kernels fermion_force_eo_0..3,
 * ocl_kernel/force_fermion_eo.cl, via hardware/code/molecular_dynamics.cpp:543-625):
 * gm += the force of Y on the sites evenodd selects (C2Q_ODD: x+y+z+t even) and X
 * on the other parity; FP64. */
C2Q_EXPORT int c2q_fermion_force_eo(c2q_gaugemomenta* gm, const c2q_gauge* g, const c2q_spinor_eo* Y,
                                    const c2q_spinor_eo* X, int evenodd, double kappa);

/* ---------------- inputs ---------------- */
/* Seeded synthetic gauge field U = exp(i eps H), H traceless Hermitian with
 * N(0,1) entries, reunitarised in FP64 (host computation, no GPU needed).
 * Writes Matrixsu3[4V] in the reference's AoS layout. */
C2Q_EXPORT int c2q_gauge_generate(double* aos, int ns, int nt, double eps, unsigned long long seed);
/* Seeded sources into host arrays of n_sites spinors:
 * kind 0 = Z2 noise ((+-1 +-i)/sqrt 2 per component), 1 = Gaussian (complex N(0,1) per component). */
C2Q_EXPORT int c2q_source_generate(double* aos, size_t n_sites, int kind, unsigned long long seed);
/* Gauge configuration in ILDG format in a LIME file (what the reference reads
 * with ildg_io/ildgIo_gaugefield.cpp:44-76, copy_gaugefield_from_ildg_format
 * :158-221): aos receives Matrixsu3[4V] (link mu + 4*site, mu 0 = time); with
 * aos = NULL only ns / nt / precision are read.  info (may be NULL) receives the
 * xlf-info text; checksum_status: 1 the recorded SciDAC checksum matches the
 * data, 0 it does not, -1 none recorded; suma / sumb: the checksum of the data. */
C2Q_EXPORT int c2q_ildg_read(const char* path, double* aos, size_t aos_len, int* ns, int* nt, int* precision,
                             char* info, int info_len, unsigned* suma, unsigned* sumb, int* checksum_status);
/* The same sources generated in place on the device into an FP64 eo field
 * (Z2 bit-identical to c2q_source_generate; Gaussian equal to rounding). */
C2Q_EXPORT int c2q_spinor_eo_source(c2q_spinor_eo* f, int kind, unsigned long long seed);

/* Library version string. */
C2Q_EXPORT const char* c2q_version(void);

/* ---------------- serving (no counterpart in the reference) ----------------
 * A request loop on one GPU.  The server owns `slots` worker threads, each with
 * its own context and stream; queued requests are admitted, first fit in
 * arrival order, as soon as a slot is free and their HBM footprint fits the
 * budget, so their work overlaps on the device with the running requests.
 * Gauge fields are registered once and stay resident.  Each request solves
 * QplusQminus_eo x_k = b_k (twisted mass, mubar = 2 kappa mu) for nsrc seeded
 * sources generated on the device, with the multi-right-hand-side mixed-
 * precision CG at the server's inner precision and link format. */
typedef struct c2q_server c2q_server;
typedef struct {
    c2q_lattice lat;                  /* must equal the registered gauge field's lattice */
    unsigned long long gauge_id;
    double kappa, mu;
    int nsrc;                         /* 1..64 sources */
    int source_kind;                  /* 0 Z2, 1 Gaussian (c2q_source_generate) */
    unsigned long long source_seed;   /* source k uses seed + k */
    c2q_solver_params params;         /* stopping test and limits; precision / use_rec12 come from the server */
    double* solutions;                /* optional host array nsrc * Seo * 24 (eo AoS per source), or NULL */
} c2q_request;
typedef struct {
    int status;                       /* C2Q_OK or the worst solver status; C2Q_OOM if it can never fit */
    int nsrc;
    double t_submit, t_admit, t_done; /* seconds since the server was created */
    int iterations_max;
    double true_resid_rel_max;        /* max over sources of ||b - A x|| / ||b|| in FP64 */
    double solution_norm2;            /* sum over sources of |x|^2 (a checksum) */
    long long footprint_bytes;
} c2q_request_result;
typedef struct {
    long long budget_bytes, gauge_bytes, reserved_bytes;
    int queued, running, slots;
    long long completed;
    double seconds;
} c2q_server_stats;
/* hbm_budget 0: 85% of the free device memory; precision 32 or 16 (inner CG). */
C2Q_EXPORT int c2q_server_create(c2q_server** out, int device, int slots, size_t hbm_budget, int precision,
                                 int rec12);
C2Q_EXPORT int c2q_server_add_gauge(c2q_server* s, unsigned long long gauge_id, const c2q_lattice* lat,
                                    const double* aos);
/* A request with eo sites x sources >= heavy_site_rhs fills the GPU by itself;
 * at most max_heavy such requests run at a time (two side by side share SMs and
 * L2 and finish later than one after the other), while lighter requests are
 * admitted beside them.  Default 2^19 site-sources, 1 at a time; max_heavy =
 * slots lifts the limit. */
C2Q_EXPORT int c2q_server_set_heavy_limit(c2q_server* s, long long heavy_site_rhs, int max_heavy);
C2Q_EXPORT int c2q_server_submit(c2q_server* s, const c2q_request* req, long long* ticket);
/* Blocks until the request has finished (or failed); each ticket is waited on once. */
C2Q_EXPORT int c2q_server_wait(c2q_server* s, long long ticket, c2q_request_result* out);
C2Q_EXPORT int c2q_server_get_stats(c2q_server* s, c2q_server_stats* out);
/* Finishes the running requests, cancels the queued ones (status C2Q_TIMEOUT). */
C2Q_EXPORT int c2q_server_destroy(c2q_server* s);
/* Device bytes one request holds while it runs (the admission footprint). */
C2Q_EXPORT size_t c2q_request_footprint(const c2q_lattice* lat, int nsrc, int precision);

#ifdef __cplusplus
}
#endif

#endif
