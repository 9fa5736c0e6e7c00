/*
 * c2q_oracle.c -- TEST INFRASTRUCTURE ONLY (oracle control flow).
 *
 * A C restatement of the reference's eo fermion-matrix, solver and inversion
 * control flow, running on the kernel interface of oracle_kernels.h.  Linked
 * with oracle_kernels_port.c it is the "port" oracle; linked with
 * oracle_kernels_ref.c (the reference's own kernels) it is the "reference"
 * CPU path.  Only tests/, the smoke check and bench.py's CPU-baseline leg load
 * it; the product never does.
 *
 * Followed:
 *   operators   physics/fermionmatrix/fermionmatrix.cpp:224-664
 *   cg          physics/algorithms/solvers/cg.cpp:277-400 (cg_singledev)
 *   bicgstab    physics/algorithms/solvers/bicgstab.cpp:401-564 (save), :566-733 (fast)
 *   inversion   physics/algorithms/inversion.cpp:78-242 (eo branch)
 *   fills       meta/type_ops.cpp:27-66, hardware/code/GaugefieldTester.cpp:52-78,
 *               hardware/code/SpinorTester.cpp:280-296
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_kernels.h"

#define C2QO_API __attribute__((visibility("default")))

/* status codes shared with the product's C ABI */
#define C2QO_SOLVER_STUCK -1
#define C2QO_DID_NOT_SOLVE -2

enum { C2QO_WILSON = 0, C2QO_TWISTEDMASS = 1 };
enum {
    C2QO_OP_AEE          = 0,
    C2QO_OP_AEE_MINUS    = 1,
    C2QO_OP_QPLUS_EO     = 2,
    C2QO_OP_QMINUS_EO    = 3,
    C2QO_OP_QPQM_EO      = 4,
    C2QO_OP_AEE_G5       = 5, /* Aee_AND_gamma5_eo */
    C2QO_OP_AEE_MINUS_G5 = 6  /* Aee_minus_AND_gamma5_eo */
};

typedef struct {
    double prec;           /* solverPrecision: stop when |r|^2 < prec (absolute) */
    int cgmax;             /* solverMaxIterations */
    int iter_refresh;      /* solverRestartEvery */
    int resid_check_every; /* solverResiduumCheckEvery (CG only) */
    int min_iter;          /* solverMinIterations (CG only) */
    int merge_spinor;      /* useKernelMergingSpinor */
    int merge_fermion;     /* useKernelMergingFermionMatrix */
    int solver;            /* 1 cg, 2 bicgstab, 3 bicgstab_save (common::solver) */
} c2qo_solver_params;

static const c2qo_complex ONE  = {1., 0.};
static const c2qo_complex MONE = {-1., 0.};

static c2qo_complex cdiv(c2qo_complex n, c2qo_complex d)
{
    double norm = d.re * d.re + d.im * d.im;
    return (c2qo_complex){(n.re * d.re + n.im * d.im) / norm, (n.im * d.re - n.re * d.im) / norm};
}
static c2qo_complex cmul(c2qo_complex a, c2qo_complex b)
{
    return (c2qo_complex){a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im};
}

static double* field_alloc(void) { return calloc(ok_seo() * 24, sizeof(double)); }

/* --------------------------- thin kernel exports --------------------------- */
C2QO_API const char* c2qo_backend(void) { return ok_backend_name(); }

C2QO_API void c2qo_set_lattice(int ns, int nt, double theta_t, double theta_s, int use_cp_re, double cp_re,
                               int use_cp_im, double cp_im)
{
    c2qo_lattice l = {ns, nt, theta_t, theta_s, use_cp_re, use_cp_im, cp_re, cp_im};
    ok_set_lattice(&l);
}
C2QO_API void c2qo_dslash_eo(double* out, const double* in, const double* g, int evenodd, double kappa)
{
    ok_dslash_eo(out, in, g, evenodd, kappa);
}
C2QO_API void c2qo_dslash_tm_inv_eo(double* out, const double* in, const double* g, int evenodd, double kappa,
                                    double mubar, int minus)
{
    ok_dslash_tm_inv_eo(out, in, g, evenodd, kappa, mubar, minus);
}
C2QO_API void c2qo_tm_diag(double* out, const double* in, double mubar, int which) { ok_tm_diag(out, in, mubar, which); }
C2QO_API void c2qo_gamma5_eo(double* inout) { ok_gamma5_eo(inout); }
C2QO_API void c2qo_saxpy(double* out, double are, double aim, const double* x, const double* y)
{
    ok_saxpy(out, (c2qo_complex){are, aim}, x, y);
}
C2QO_API void c2qo_saxpy_gamma5(double* out, double are, double aim, const double* x, const double* y)
{
    ok_saxpy_gamma5(out, (c2qo_complex){are, aim}, x, y);
}
C2QO_API void c2qo_sax(double* out, double are, double aim, const double* x) { ok_sax(out, (c2qo_complex){are, aim}, x); }
C2QO_API void c2qo_saxsbypz(double* out, double are, double aim, const double* x, double bre, double bim,
                            const double* y, const double* z)
{
    ok_saxsbypz(out, (c2qo_complex){are, aim}, x, (c2qo_complex){bre, bim}, y, z);
}
C2QO_API void c2qo_scalar_product(const double* x, const double* y, double* re, double* im)
{
    c2qo_complex r = ok_scalar_product(x, y);
    *re            = r.re;
    *im            = r.im;
}
C2QO_API double c2qo_squarenorm(const double* x) { return ok_squarenorm(x); }
C2QO_API double c2qo_squarenorm_full(const double* x) { return ok_squarenorm_full(x); }
C2QO_API double c2qo_saxpy_squarenorm(double* out, double are, double aim, const double* x, const double* y)
{
    return ok_saxpy_squarenorm(out, (c2qo_complex){are, aim}, x, y);
}
C2QO_API void c2qo_cold(double* x) { ok_cold(x); }
C2QO_API void c2qo_zero(double* x) { ok_zero(x); }
C2QO_API void c2qo_convert_to_eo(double* even, double* odd, const double* full) { ok_convert_to_eo(even, odd, full); }
C2QO_API void c2qo_convert_from_eo(double* full, const double* even, const double* odd)
{
    ok_convert_from_eo(full, even, odd);
}
C2QO_API void c2qo_m_tm_plus(double* out, const double* in, const double* g, double kappa, double mubar)
{
    ok_m_tm_plus(out, in, g, kappa, mubar);
}
C2QO_API void c2qo_m_tm_minus(double* out, const double* in, const double* g, double kappa, double mubar)
{
    ok_m_tm_minus(out, in, g, kappa, mubar);
}
C2QO_API void c2qo_gamma5_full(double* inout) { ok_gamma5_full(inout); }

/* ------------------------------ operators ------------------------------ */
/* Aee family, fermionmatrix.cpp:224-591.  "minus" selects Aee_minus, "g5" the
 * _AND_gamma5_eo variant (merged saxpy+gamma5 at the end). */
static void aee_family(double* out, const double* in, const double* g, double kappa, double mubar, int action,
                       int minus, int g5)
{
    double* tmp  = field_alloc();
    double* tmp2 = field_alloc();
    if (action == C2QO_WILSON) {
        ok_dslash_eo(tmp, in, g, 1 /*ODD*/, kappa);
        ok_dslash_eo(out, tmp, g, 0 /*EVEN*/, kappa);
        if (g5)
            ok_saxpy_gamma5(out, ONE, out, in);
        else
            ok_saxpy(out, ONE, out, in);
    } else {
        ok_dslash_eo(tmp, in, g, 1, kappa);
        ok_tm_diag(tmp2, tmp, mubar, minus ? C2QO_DIAG_MINV_MINUS : C2QO_DIAG_MINV);
        ok_dslash_eo(out, tmp2, g, 0, kappa);
        ok_tm_diag(tmp, in, mubar, minus ? C2QO_DIAG_M_MINUS : C2QO_DIAG_M);
        if (g5)
            ok_saxpy_gamma5(out, ONE, out, tmp);
        else
            ok_saxpy(out, ONE, out, tmp);
    }
    free(tmp);
    free(tmp2);
}

/* fermionmatrix.cpp:592-664 */
C2QO_API void c2qo_apply(int op, double* out, const double* in, const double* g, double kappa, double mubar,
                         int action, int merged)
{
    switch (op) {
        case C2QO_OP_AEE: aee_family(out, in, g, kappa, mubar, action, 0, 0); break;
        case C2QO_OP_AEE_MINUS: aee_family(out, in, g, kappa, mubar, action, 1, 0); break;
        case C2QO_OP_AEE_G5: aee_family(out, in, g, kappa, mubar, action, 0, 1); break;
        case C2QO_OP_AEE_MINUS_G5: aee_family(out, in, g, kappa, mubar, action, 1, 1); break;
        case C2QO_OP_QPLUS_EO:
        case C2QO_OP_QMINUS_EO: {
            const int minus = op == C2QO_OP_QMINUS_EO;
            if (!merged) {
                aee_family(out, in, g, kappa, mubar, action, minus, 0);
                ok_gamma5_eo(out);
            } else {
                aee_family(out, in, g, kappa, mubar, action, minus, 1);
            }
            break;
        }
        case C2QO_OP_QPQM_EO: {
            double* tmp = field_alloc();
            c2qo_apply(C2QO_OP_QMINUS_EO, tmp, in, g, kappa, mubar, action, merged);
            c2qo_apply(C2QO_OP_QPLUS_EO, out, tmp, g, kappa, mubar, action, merged);
            free(tmp);
            break;
        }
        default: abort();
    }
}

/* ------------------------------ solvers ------------------------------ */
typedef struct {
    int op, action, merged;
    const double* g;
    double kappa, mubar;
} opctx;

static void opapply(const opctx* A, double* out, const double* in)
{
    c2qo_apply(A->op, out, in, A->g, A->kappa, A->mubar, A->action, A->merged);
}

/* cg.cpp:277-400 */
static int cg_eo(double* x, const opctx* A, const double* b, const c2qo_solver_params* P)
{
    double* p  = field_alloc();
    double* rn = field_alloc();
    double* v  = field_alloc();
    c2qo_complex omega = {0, 0}, rho, alpha, beta, rho_next = {0, 0};
    int iter, ret = C2QO_DID_NOT_SOLVE;
    for (iter = 0; iter < P->cgmax || iter < P->min_iter; iter++) {
        if (iter % P->iter_refresh == 0) {
            opapply(A, rn, x);
            ok_saxpy(rn, ONE, rn, b);
            ok_copy(p, rn);
            omega = ok_scalar_product(rn, rn);
        } else {
            omega = rho_next;
        }
        opapply(A, v, p);
        rho   = ok_scalar_product(p, v);
        alpha = cdiv(omega, rho);
        c2qo_complex tmp1 = cmul(MONE, alpha);
        ok_saxpy(x, tmp1, p, x);
        if (P->merge_spinor) {
            double n = ok_saxpy_squarenorm(rn, alpha, v, rn);
            rho_next = (c2qo_complex){n, 0.};
        } else {
            ok_saxpy(rn, alpha, v, rn);
            rho_next = ok_scalar_product(rn, rn);
        }
        if (iter % P->resid_check_every == 0) {
            double resid = rho_next.re;
            if (resid != resid) {
                ret = C2QO_SOLVER_STUCK;
                goto done;
            }
            if (resid < P->prec && iter >= P->min_iter) {
                ret = iter;
                goto done;
            }
        }
        beta = cdiv(rho_next, omega);
        c2qo_complex tmp2 = cmul(MONE, beta);
        ok_saxpy(p, tmp2, p, rn);
    }
done:
    free(p);
    free(rn);
    free(v);
    return ret;
}

/* bicgstab.cpp:566-733 */
static int bicgstab_fast(double* x, const opctx* A, const double* b, const c2qo_solver_params* P)
{
    double *p = field_alloc(), *rn = field_alloc(), *rhat = field_alloc(), *s = field_alloc(), *t = field_alloc(),
           *v = field_alloc();
    c2qo_complex alpha = {0, 0}, beta, omega = {0, 0}, rho = {0, 0}, rho_next, tmp1, tmp2;
    int iter, ret = C2QO_DID_NOT_SOLVE;
    for (iter = 0; iter < P->cgmax; iter++) {
        if (iter % P->iter_refresh == 0) {
            opapply(A, rn, x);
            ok_saxpy(p, ONE, rn, b);
            ok_copy(rhat, p);
            ok_copy(rn, p);
            rho = ok_scalar_product(rhat, rn);
        }
        double resid = ok_squarenorm(rn);
        if (resid != resid) {
            ret = C2QO_SOLVER_STUCK;
            goto done;
        }
        if (resid < P->prec) {
            ret = iter;
            goto done;
        }
        opapply(A, v, p);
        tmp1  = ok_scalar_product(rhat, v);
        alpha = cdiv(rho, tmp1);
        ok_saxpy(s, alpha, v, rn);
        opapply(A, t, s);
        tmp1  = ok_scalar_product(t, s);
        tmp2  = ok_scalar_product(t, t);
        omega = cdiv(tmp1, tmp2);
        ok_saxsbypz(x, alpha, p, omega, s, x);
        ok_saxpy(rn, omega, t, s);
        rho_next = ok_scalar_product(rhat, rn);
        if (fabs(rho_next.re) < 1e-25 && fabs(rho_next.im) < 1e-25) {
            ret = C2QO_SOLVER_STUCK;
            goto done;
        }
        tmp1 = cdiv(rho_next, rho);
        tmp2 = cdiv(alpha, omega);
        beta = cmul(tmp1, tmp2);
        tmp1 = cmul(beta, omega);
        tmp2 = cmul(MONE, tmp1);
        ok_saxsbypz(p, beta, p, tmp2, v, rn);
        rho = rho_next;
    }
done:
    free(p);
    free(rn);
    free(rhat);
    free(s);
    free(t);
    free(v);
    return ret;
}

/* bicgstab.cpp:401-564 */
static int bicgstab_save(double* x, const opctx* A, const double* b, const c2qo_solver_params* P)
{
    double *s = field_alloc(), *t = field_alloc(), *v = field_alloc(), *p = field_alloc(), *rn = field_alloc(),
           *rhat = field_alloc(), *aux = field_alloc();
    c2qo_complex alpha = ONE, beta, omega = ONE, rho = ONE, rho_next, tmp1, tmp2;
    int iter, ret = C2QO_DID_NOT_SOLVE;
    for (iter = 0; iter < P->cgmax; iter++) {
        if (iter % P->iter_refresh == 0) {
            ok_zero(v);
            ok_zero(p);
            opapply(A, rn, x);
            ok_saxpy(rn, ONE, rn, b);
            ok_copy(rhat, rn);
            alpha = ONE;
            omega = ONE;
            rho   = ONE;
        }
        rho_next = ok_scalar_product(rhat, rn);
        if (fabs(rho_next.re) < 1e-25 && fabs(rho_next.im) < 1e-25) {
            ret = C2QO_SOLVER_STUCK;
            goto done;
        }
        tmp1 = cdiv(rho_next, rho);
        rho  = rho_next;
        tmp2 = cdiv(alpha, omega);
        beta = cmul(tmp1, tmp2);
        tmp1 = cmul(beta, omega);
        tmp2 = cmul(MONE, tmp1);
        ok_saxsbypz(p, beta, p, tmp2, v, rn);
        opapply(A, v, p);
        tmp1  = ok_scalar_product(rhat, v);
        alpha = cdiv(rho, tmp1);
        ok_saxpy(s, alpha, v, rn);
        opapply(A, t, s);
        tmp1  = ok_scalar_product(t, s);
        tmp2  = ok_scalar_product(t, t);
        omega = cdiv(tmp1, tmp2);
        ok_saxpy(rn, omega, t, s);
        ok_saxsbypz(x, alpha, p, omega, s, x);
        double resid = ok_squarenorm(rn);
        if (resid != resid) {
            ret = C2QO_SOLVER_STUCK;
            goto done;
        }
        if (resid < P->prec) {
            opapply(A, aux, x);
            ok_saxpy(aux, ONE, aux, b);
            double trueresid = ok_squarenorm(aux);
            if (trueresid < P->prec) {
                ret = iter;
                goto done;
            }
        }
    }
done:
    free(s);
    free(t);
    free(v);
    free(p);
    free(rn);
    free(rhat);
    free(aux);
    return ret;
}

C2QO_API int c2qo_cg(double* x, int op, const double* b, const double* g, double kappa, double mubar, int action,
                     const c2qo_solver_params* P)
{
    opctx A = {op, action, P->merge_fermion, g, kappa, mubar};
    return cg_eo(x, &A, b, P);
}

C2QO_API int c2qo_bicgstab(double* x, int op, const double* b, const double* g, double kappa, double mubar, int action,
                           const c2qo_solver_params* P)
{
    opctx A = {op, action, P->merge_fermion, g, kappa, mubar};
    return P->solver == 3 ? bicgstab_save(x, &A, b, P) : bicgstab_fast(x, &A, b, P);
}

/* ------------------------------ HMC callers ------------------------------ */
/* physics::algorithms::fermion_force(gm, Y, X, evenodd, ...) on the eo fields
 * (fermion_force.cpp:699-730 -> molecular_dynamics.cpp:543-625) */
C2QO_API void c2qo_fermion_force_eo(double* gm, const double* Y, const double* X, const double* g, int evenodd,
                                    double kappa)
{
    ok_fermion_force_eo(gm, Y, X, g, evenodd, kappa);
}

/* physics::algorithms::fermion_force(gm, Y, X, ...) on full fields
 * (fermion_force.cpp:672-697 -> force_fermion.cl) */
C2QO_API void c2qo_fermion_force_full(double* gm, const double* Y, const double* X, const double* g, double kappa)
{
    ok_fermion_force_full(gm, Y, X, g, kappa);
}

/* squarenorm of gauge momenta ae[4V] (gaugemomentum_squarenorm.cl: the sum of
 * e_k^2 over every link) */
C2QO_API double c2qo_gm_squarenorm(const double* gm)
{
    const size_t n = 4 * 8 * ok_vol();
    double s       = 0.;
    for (size_t k = 0; k < n; ++k) s += gm[k] * gm[k];
    return s;
}

/* calc_fermion_force on eo fields, CG branch (fermion_force.cpp:37-80, 131-175):
 * X = (Q+Q-)^-1 phi from a cold start, Y = Q- X, then
 *   X_odd = -M^-1_minus D(ODD) X,  F += F(Y, X_odd, EVEN),
 *   Y_odd = -M^-1 D(ODD) Y,        F += F(Y_odd, X, ODD)
 * (Wilson: the site-diagonal inverse is 1).  Returns the CG's iteration count. */
C2QO_API int c2qo_calc_fermion_force_eo(double* gm, const double* phi, const double* g, double kappa, double mubar,
                                        int action, const c2qo_solver_params* P)
{
    double *x = field_alloc(), *y = field_alloc(), *tmp1 = field_alloc(), *tmp2 = field_alloc();
    ok_cold(x);
    const int it = c2qo_cg(x, C2QO_OP_QPQM_EO, phi, g, kappa, mubar, action, P);
    c2qo_apply(C2QO_OP_QMINUS_EO, y, x, g, kappa, mubar, action, P->merge_fermion);
    const c2qo_complex m1 = {-1., 0.};
    ok_dslash_eo(tmp1, x, g, 1 /*ODD*/, kappa);
    if (action == C2QO_TWISTEDMASS) {
        ok_tm_diag(tmp2, tmp1, mubar, C2QO_DIAG_MINV_MINUS);
        ok_sax(tmp1, m1, tmp2);
    } else {
        ok_sax(tmp1, m1, tmp1);
    }
    ok_fermion_force_eo(gm, y, tmp1, g, 0 /*EVEN*/, kappa);
    ok_dslash_eo(tmp1, y, g, 1 /*ODD*/, kappa);
    if (action == C2QO_TWISTEDMASS) {
        ok_tm_diag(tmp2, tmp1, mubar, C2QO_DIAG_MINV);
        ok_sax(tmp1, m1, tmp2);
    } else {
        ok_sax(tmp1, m1, tmp1);
    }
    ok_fermion_force_eo(gm, tmp1, x, g, 1 /*ODD*/, kappa);
    free(x);
    free(y);
    free(tmp1);
    free(tmp2);
    return it;
}

/* calc_s_fermion on eo fields, CG branch (metropolis.cpp:79-121): X = (Q+Q-)^-1
 * phi from a cold start, S_f = |Q- X|^2.  *iters receives the CG's count. */
C2QO_API double c2qo_calc_s_fermion_eo(const double* phi, const double* g, double kappa, double mubar, int action,
                                       const c2qo_solver_params* P, int* iters)
{
    double *x = field_alloc(), *y = field_alloc();
    ok_cold(x);
    const int it = c2qo_cg(x, C2QO_OP_QPQM_EO, phi, g, kappa, mubar, action, P);
    if (iters) *iters = it;
    c2qo_apply(C2QO_OP_QMINUS_EO, y, x, g, kappa, mubar, action, P->merge_fermion);
    const double s2 = ok_squarenorm(y);
    free(x);
    free(y);
    return s2;
}

/* Eo branch of invert_M_nf2_upperflavour, inversion.cpp:129-236, including the
 * parity-role swap (issue #387 workaround, :141-149) and the sign convention of
 * the prepared source and the odd reconstruction (:165-169, :204-221).
 * Returns the solver's iteration count or a negative status; *used_cg tells
 * whether the CG fallback ran. */
C2QO_API int c2qo_perform_inversion_eo(double* result, const double* source, const double* g, double kappa,
                                       double mubar, int action, const c2qo_solver_params* P, int* used_cg)
{
    double *src_even = field_alloc(), *src_odd = field_alloc(), *tmp1 = field_alloc(), *tmp2 = field_alloc(),
           *res_eo = field_alloc();
    int converged;
    ok_convert_to_eo(src_odd, src_even, source);
    if (action == C2QO_WILSON) {
        ok_dslash_eo(tmp1, src_odd, g, 0 /*EVEN*/, kappa);
        ok_saxpy(src_even, ONE, src_even, tmp1);
    } else {
        ok_tm_diag(tmp1, src_odd, mubar, C2QO_DIAG_MINV);
        ok_dslash_eo(tmp2, tmp1, g, 0, kappa);
        ok_saxpy(src_even, ONE, src_even, tmp2);
    }
    ok_cold(res_eo);
    if (used_cg) *used_cg = 0;
    c2qo_solver_params Pb = *P;
    if (P->solver == 1) Pb.solver = 2; /* solver=cg first tries BiCGStab (inversion.cpp:176-181) */
    converged = c2qo_bicgstab(res_eo, C2QO_OP_AEE, src_even, g, kappa, mubar, action, &Pb);
    if (converged < 0 && P->solver == 1) {
        /* CG fallback on QplusQminus_eo with source gamma5 b, then x = Qminus_eo y (inversion.cpp:182-195) */
        if (used_cg) *used_cg = 1;
        ok_gamma5_eo(src_even);
        converged = c2qo_cg(res_eo, C2QO_OP_QPQM_EO, src_even, g, kappa, mubar, action, P);
        c2qo_apply(C2QO_OP_QMINUS_EO, src_even, res_eo, g, kappa, mubar, action, P->merge_fermion);
        ok_copy(res_eo, src_even);
    }
    if (action == C2QO_WILSON) {
        ok_dslash_eo(tmp1, res_eo, g, 1 /*ODD*/, kappa);
        ok_saxpy(tmp1, MONE, tmp1, src_odd);
        ok_sax(tmp1, MONE, tmp1);
    } else {
        ok_dslash_eo(tmp2, res_eo, g, 1, kappa);
        ok_tm_diag(tmp1, tmp2, mubar, C2QO_DIAG_MINV);
        ok_tm_diag(tmp2, src_odd, mubar, C2QO_DIAG_MINV);
        ok_saxpy(tmp1, MONE, tmp1, tmp2);
        ok_sax(tmp1, MONE, tmp1);
    }
    ok_convert_from_eo(result, tmp1, res_eo);
    free(src_even);
    free(src_odd);
    free(tmp1);
    free(tmp2);
    free(res_eo);
    return converged;
}

/* ------------------------------ test fills ------------------------------ */
/* pseudo_randomize: srand48(seed) then one drand48() per real, in memory order
 * (meta/type_ops.cpp:27-66; physics/lattices/util.hpp:83-91). */
C2QO_API void c2qo_pseudo_randomize(double* a, size_t n_reals, int seed)
{
    srand48(seed);
    for (size_t i = 0; i < n_reals; ++i) a[i] = drand48();
}

/* GaugefieldFillType::nonTrivial: one fixed matrix on every link
 * (hardware/code/GaugefieldTester.cpp:52-78); cold: identity. */
C2QO_API void c2qo_fill_gauge(double* g, size_t n_links, int nontrivial)
{
    static const double NT[18] = {.130189,  .260378,  .260378,  .390567,  .520756,    .650945,
                                  .572742,  .403041,  .371222,  .321726,  -.449002,   -.258088,
                                  1.11022e-16, .651751, .0271563, -.733219, -.0271563, .190094};
    static const double ID[18] = {1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0};
    for (size_t l = 0; l < n_links; ++l) memcpy(g + 18 * l, nontrivial ? NT : ID, sizeof NT);
}

/* SpinorFillType::ascendingComplex: component k (0..11) = (2k+1, 2k+2)
 * (hardware/code/SpinorTester.cpp:280-296). */
C2QO_API void c2qo_fill_ascending_complex(double* s, size_t n_sites)
{
    for (size_t i = 0; i < n_sites; ++i)
        for (int k = 0; k < 24; ++k) s[24 * i + k] = (double)(k + 1);
}

/* count_sf: sum of all re and im parts (hardware/code/SpinorTester.cpp:343-353). */
C2QO_API double c2qo_count_sf(const double* s, size_t n_sites)
{
    double sum = 0.;
    for (size_t i = 0; i < n_sites; ++i) {
        double site = 0.;
        for (int k = 0; k < 24; ++k) site += s[24 * i + k];
        sum += site;
    }
    return sum;
}
