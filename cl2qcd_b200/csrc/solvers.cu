// solvers.cu -- CG (FP64 and mixed precision with FP64 reliable updates),
// BiCGStab (fast and save variants) and the eo Schur-complement inversion,
// on top of the fused sweeps of fields.cu.
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <limits>
#include <vector>

#include "blas.cuh"
#include "c2q_host.h"
#include "mixed.cuh"

namespace c2q {

namespace {

struct Cx {
    double re, im;
};
inline Cx cdiv(Cx n, Cx d)
{
    // complexdivide, common_header_files/operations_complex.hpp:59-66
    const double norm = d.re * d.re + d.im * d.im;
    return {(n.re * d.re + n.im * d.im) / norm, (n.im * d.re - n.re * d.im) / norm};
}
inline Cx cmulx(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im}; }

// RAII group of scratch fields
struct Fields {
    std::vector<c2q_spinor_eo> f;
    ~Fields()
    {
        for (auto& x : f) field_free(&x);
    }
};

int make_fields(c2q_ctx* ctx, const c2q_lattice& lat, int prec, int n, Fields& F, size_t first)
{
    F.f.resize(first + n);
    for (int k = 0; k < n; ++k) {
        int rc = field_alloc(ctx, lat, prec, &F.f[first + k]);
        if (rc) return rc;
    }
    return C2Q_OK;
}

struct SolveClock {
    c2q_ctx* ctx;
    explicit SolveClock(c2q_ctx* c) : ctx(c) { cudaEventRecord(ctx->ev0, ctx->stream); }
    double seconds()
    {
        cudaEventRecord(ctx->ev1, ctx->stream);
        cudaEventSynchronize(ctx->ev1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        return ms * 1e-3;
    }
};

int read_sc(c2q_ctx* ctx, SolverScalars* h)
{
    int rc = pinned_copy(ctx, ctx->host_pinned_dev, 0, ctx->scalars, 0, sizeof(SolverScalars));
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(h, ctx->host_pinned, sizeof(SolverScalars));
    return C2Q_OK;
}

int write_sc(c2q_ctx* ctx, const SolverScalars& h)
{
    memcpy(ctx->host_pinned, &h, sizeof(SolverScalars));
    int rc = pinned_copy(ctx, ctx->scalars, 0, ctx->host_pinned_dev, 0, sizeof(SolverScalars));
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

// out = y - a x with |out|^2 into the reduction result (or a finisher); returns via read if asked
int saxpy_norm(c2q_ctx* ctx, c2q_spinor_eo* out, Cx a, const c2q_spinor_eo* x, const c2q_spinor_eo* y, int fin,
               double* norm_out)
{
    BlasSpec s;
    s.op  = B_SAXPY;
    s.out = out;
    s.x   = x;
    s.y   = y;
    s.a   = coef_host(a.re, a.im);
    s.dot = 2;
    s.fin = fin;
    int rc = launch_blas(ctx, s);
    if (rc || !norm_out) return rc;
    double h[2];
    rc        = read_scalars(ctx, ctx->red_result, 2, h);
    *norm_out = h[0];
    return rc;
}

int dot_read(c2q_ctx* ctx, const c2q_spinor_eo* x, const c2q_spinor_eo* y, Cx* out)
{
    BlasSpec s;
    s.x   = x;
    s.y   = y;
    s.dot = 1;
    int rc = launch_blas(ctx, s);
    if (rc) return rc;
    double h[2];
    rc   = read_scalars(ctx, ctx->red_result, 2, h);
    *out = {h[0], h[1]};
    return rc;
}

// <x,y> and <x,x> in one pass over x and y (read back together)
int dot2_read(c2q_ctx* ctx, const c2q_spinor_eo* x, const c2q_spinor_eo* y, Cx* xy, Cx* xx)
{
    BlasSpec s;
    s.x    = x;
    s.y    = y;
    s.dot  = 3;
    int rc = launch_blas(ctx, s);
    if (rc) return rc;
    double h[4];
    rc  = read_scalars(ctx, ctx->red_result, 4, h);
    *xy = {h[0], h[1]};
    *xx = {h[2], h[3]};
    return rc;
}

int copy_field(c2q_ctx* ctx, c2q_spinor_eo* to, const c2q_spinor_eo* from)
{
    BlasSpec s;
    s.op  = B_COPY;
    s.out = to;
    s.x   = from;
    return launch_blas(ctx, s);
}


// ||b - A x||^2 in FP64 (true residual); r receives b - A x.
int true_residual(c2q_ctx* ctx, int op, const c2q_gauge* g, const c2q_spinor_eo* x, const c2q_spinor_eo* b,
                  double kappa, double mubar, int action, c2q_spinor_eo* r, c2q_spinor_eo* t1, c2q_spinor_eo* t2,
                  double* r2, int* sweeps, int gk64 = G64)
{
    int rc = apply_operator(ctx, op, r, g, gk64, x, kappa, mubar, action, t1, t2, DotSpec{}, sweeps);
    if (rc) return rc;
    return saxpy_norm(ctx, r, Cx{1, 0}, r, b, FIN_STORE_RESULT, r2);
}

// |x|^2 (to skip A x when the start vector is zero)
int norm2(c2q_ctx* ctx, const c2q_spinor_eo* x, double* out)
{
    Cx c;
    int rc = dot_read(ctx, x, x, &c);
    *out   = c.re;
    return rc;
}

bool validate(c2q_ctx* ctx, const c2q_spinor_eo* x, const c2q_gauge* g, const c2q_spinor_eo* b,
              const c2q_solver_params* p, int* rc)
{
    if (!x || !g || !b || !p) {
        *rc = C2Q_BAD_ARG;
        return false;
    }
    if (x->prec != 64 || b->prec != 64 || !same_lattice(x->lat, b->lat) || !same_lattice(x->lat, g->lat)) {
        *rc = fail(ctx, C2Q_BAD_ARG, "solver fields must be FP64 fields on the gauge field's lattice");
        return false;
    }
    if (p->iter_refresh <= 0 || p->resid_check_every <= 0 || p->cgmax < 0) {
        *rc = fail(ctx, C2Q_BAD_ARG, "solverRestartEvery and solverResiduumCheckEvery must be positive");
        return false;
    }
    if (p->precision != 64 && p->precision != 32 && p->precision != 16) {
        *rc = fail(ctx, C2Q_BAD_ARG, "precision must be 64, 32 or 16");
        return false;
    }
    return true;
}

double stop_threshold(const c2q_solver_params* p, double b2)
{
    double thr = 0.0;
    if (p->prec > 0) thr = p->prec;
    if (p->rel_tol > 0) thr = std::max(thr, p->rel_tol * p->rel_tol * b2);
    return thr;
}

void finish_report(c2q_solve_report* rep, int status, int iters, int rel, double r2, double true_rel, double secs,
                   int sweeps)
{
    if (!rep) return;
    rep->status              = status;
    rep->iterations          = iters;
    rep->reliable_updates    = rel;
    rep->resid_sq            = r2;
    rep->true_resid_rel      = true_rel;
    rep->seconds             = secs;
    rep->dslash_applications = sweeps;
}

// Ring of pinned slots receiving |r|^2 (SolverScalars::resid) and the
// division flag of each iteration, with one event per slot.
struct ResidRing {
    static constexpr int N = 4;
    c2q_ctx* ctx;
    explicit ResidRing(c2q_ctx* c) : ctx(c) {}
    int push(int k)
    {
        // SolverScalars::resid, aux[2], flag: the first 28 bytes of the slot
        static_assert(offsetof(SolverScalars, flag) == offsetof(SolverScalars, resid) + 3 * sizeof(double),
                      "flag follows resid and aux[2]");
        return ring_push(ctx, k, ctx->host_pinned_dev + 32 + 4 * (k % N), &ctx->scalars->resid, 0,
                         4 * sizeof(double), 1);
    }
    int pop(int k, double* resid, int* flag)
    {
        C2Q_CUDA(ctx, cudaEventSynchronize(ctx->ring_ev[k % N]));
        const double* slot = ctx->host_pinned + 32 + 4 * (k % N);
        *resid             = slot[0];
        int f;
        memcpy(&f, slot + 3, sizeof(int));
        *flag = f;
        return C2Q_OK;
    }
};

// ------------------------------------------------------------------ FP64 CG
// physics/algorithms/solvers/cg.cpp:277-400 with device-resident scalars.
int cg_fp64(c2q_ctx* ctx, c2q_spinor_eo* x, int op, const c2q_gauge* g, const c2q_spinor_eo* b, double kappa,
            double mubar, int action, const c2q_solver_params* P, c2q_solve_report* rep)
{
    Fields F;
    int rc = make_fields(ctx, x->lat, 64, 5, F, 0);
    if (rc) return rc;
    c2q_spinor_eo *p = &F.f[0], *rn = &F.f[1], *v = &F.f[2], *t1 = &F.f[3], *t2 = &F.f[4];
    // 12-real links when asked for and the field is SU(3) to rounding (the final
    // true residual always uses the links as uploaded)
    const int gk = gk64_for(g, P->use_rec12);
    int sweeps   = 0;
    SolveClock clock(ctx);

    double b2 = 0;
    rc        = saxpy_norm(ctx, rn, Cx{0, 0}, b, b, FIN_STORE_RESULT, &b2);
    if (rc) return rc;
    const double thr = stop_threshold(P, b2);
    SolverScalars zero{};
    rc = write_sc(ctx, zero);
    if (rc) return rc;

    int iter = 0, status = C2Q_DID_NOT_SOLVE;
    double resid = std::numeric_limits<double>::quiet_NaN();
    bool force_refresh = false;
    double r2_confirmed = -1.0;  // true residual of the returned solution, when already computed
    if (P->rel_tol > 0) {
        // True-residual target: residual monitored every iteration through the
        // pinned ring (no host round trip per iteration); a converged iterated
        // residual is confirmed by an FP64 true residual, else CG restarts from it.
        ResidRing ring(ctx);
        int skip_upto = -1;
        // With use_graph the iteration body between refreshes (p = rn + beta p,
        // v = A p with (p, v) -> alpha, the x / rn update) replays as one captured
        // CUDA graph: small lattices are bound by launch latency.  It is captured
        // after the first (eager) iteration has sized every launch.
        const bool graphs = P->use_graph && !ctx->profiling;
        struct Exec {
            cudaGraphExec_t e = nullptr;
            ~Exec()
            {
                if (e) cudaGraphExecDestroy(e);
            }
        } gexec;
        long long gkernels = 0;
        int gsweeps        = 0;
        auto apply_update = [&](int* sw) -> int {
            DotSpec d;
            d.mode = DOT_Y;
            d.y    = p;
            d.fin  = FIN_CG_ALPHA;
            int e  = apply_operator(ctx, op, v, g, gk, p, kappa, mubar, action, t1, t2, d, sw);
            return e ? e : launch_cg_update(ctx, x, rn, p, v);
        };
        for (iter = 0; iter < P->cgmax || iter < P->min_iter; iter++) {
            if (iter % P->iter_refresh == 0 || force_refresh) {
                force_refresh = false;
                rc = apply_operator(ctx, op, rn, g, gk, x, kappa, mubar, action, t1, t2, DotSpec{}, &sweeps);
                if (!rc) rc = saxpy_norm(ctx, rn, Cx{1, 0}, rn, b, FIN_CG_OMEGA, nullptr);
                if (!rc) rc = copy_field(ctx, p, rn);
                if (!rc) rc = apply_update(&sweeps);
            } else if (graphs) {
                if (!gexec.e) {
                    cudaGraph_t gr     = nullptr;
                    const long long l0 = ctx->launches;
                    C2Q_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
                    int eb = launch_cg_p(ctx, p, rn);
                    if (!eb) eb = apply_update(&gsweeps);
                    const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &gr);
                    if (eb) {
                        if (gr) cudaGraphDestroy(gr);
                        return eb;
                    }
                    C2Q_CUDA(ctx, ec);
                    const cudaError_t ei = cudaGraphInstantiate(&gexec.e, gr, 0);
                    cudaGraphDestroy(gr);
                    C2Q_CUDA(ctx, ei);
                    gkernels      = ctx->launches - l0;
                    ctx->launches = l0;
                }
                C2Q_CUDA(ctx, cudaGraphLaunch(gexec.e, ctx->stream));
                ctx->launches += gkernels;
                sweeps += gsweeps;
            } else {
                rc = launch_cg_p(ctx, p, rn);  // p = rn + beta p
                if (!rc) rc = apply_update(&sweeps);
            }
            if (!rc) rc = ring.push(iter);
            if (rc) return rc;
            if (iter == 0) continue;
            double rprev = 0.0;
            int bad      = 0;
            rc           = ring.pop(iter - 1, &rprev, &bad);
            if (rc) return rc;
            if (iter - 1 <= skip_upto) continue;
            resid = rprev;
            if (resid != resid) {
                status = C2Q_SOLVER_STUCK;
                break;
            }
            if (resid < thr && iter >= P->min_iter) {
                double r2t = 0;
                rc = true_residual(ctx, op, g, x, b, kappa, mubar, action, t2, t1, v, &r2t, &sweeps);
                if (rc) return rc;
                if (r2t <= P->rel_tol * P->rel_tol * b2 || (P->prec > 0 && r2t < P->prec)) {
                    status       = iter;
                    r2_confirmed = r2t;
                    break;
                }
                force_refresh = true;  // the iterated residual drifted: restart from the true residual
                skip_upto     = iter;
            }
        }
    } else {
        for (iter = 0; iter < P->cgmax || iter < P->min_iter; iter++) {
            if (iter % P->iter_refresh == 0 || force_refresh) {
                force_refresh = false;
                rc = apply_operator(ctx, op, rn, g, gk, x, kappa, mubar, action, t1, t2, DotSpec{}, &sweeps);
                if (!rc) rc = saxpy_norm(ctx, rn, Cx{1, 0}, rn, b, FIN_CG_OMEGA, nullptr);  // rn = b - A x ; omega = (rn,rn)
                if (!rc) rc = copy_field(ctx, p, rn);
                if (rc) return rc;
            }
            DotSpec d;
            d.mode = DOT_Y;
            d.y    = p;
            d.fin  = FIN_CG_ALPHA;  // rho = (p, v) ; alpha = omega / rho
            rc     = apply_operator(ctx, op, v, g, gk, p, kappa, mubar, action, t1, t2, d, &sweeps);
            if (!rc) rc = launch_cg_update(ctx, x, rn, p, v);  // x += alpha p ; rn -= alpha v ; beta, omega
            if (rc) return rc;
            if (iter % P->resid_check_every == 0) {
                SolverScalars h;
                rc = read_sc(ctx, &h);
                if (rc) return rc;
                resid = h.resid;
                if (resid != resid) {
                    status = C2Q_SOLVER_STUCK;
                    break;
                }
                if (resid < thr && iter >= P->min_iter) {
                    if (P->rel_tol > 0) {
                        double r2t = 0;
                        rc = true_residual(ctx, op, g, x, b, kappa, mubar, action, t2, t1, v, &r2t, &sweeps);
                        if (rc) return rc;
                        if (r2t <= P->rel_tol * P->rel_tol * b2 || (P->prec > 0 && r2t < P->prec)) {
                            status       = iter;
                            r2_confirmed = r2t;
                            break;
                        }
                        force_refresh = true;  // iterated residual drifted: restart from the true residual
                        continue;
                    }
                    status = iter;
                    break;
                }
            }
            rc = launch_cg_p(ctx, p, rn);  // p = rn + beta p
            if (rc) return rc;
        }
    }
    double r2t = r2_confirmed;
    if (r2t < 0) {
        rc = true_residual(ctx, op, g, x, b, kappa, mubar, action, rn, t1, t2, &r2t, &sweeps);
        if (rc) return rc;
    }
    finish_report(rep, status, iter, 0, resid, b2 > 0 ? std::sqrt(r2t / b2) : 0.0, clock.seconds(), sweeps);
    if (status == C2Q_DID_NOT_SOLVE) fail(ctx, status, "Solver did not solve in solverMaxIterations iterations");
    if (status == C2Q_SOLVER_STUCK) fail(ctx, status, "NAN occured in the CG residual");
    return status;
}

// ------------------------------------------------------- mixed-precision CG
// CG in reduced precision PB (operator, search direction) / FP32 (residual,
// solution increment), with FP64 reliable updates: whenever the iterated
// residual has dropped by `reliable_delta` since the last update (or reached
// the stopping threshold), the increment is added to the FP64 solution and the
// residual is recomputed from scratch in FP64 with FP64 links.
// Batched mixed-precision vector updates: entry r of each array is one
// right-hand side (FP32 xs, rs; PB p, v; its solver scalars).
struct MixBatch {
    int n = 0;
    c2q_spinor_eo* xs[MAX_BATCH] = {};
    c2q_spinor_eo* rs[MAX_BATCH] = {};
    c2q_spinor_eo* p[MAX_BATCH]  = {};
    const c2q_spinor_eo* v[MAX_BATCH] = {};
    SolverScalars* sc[MAX_BATCH] = {};
};

static MixArgs mix_args(const MixBatch& B)
{
    MixArgs A;
    memset(&A, 0, sizeof A);
    for (int r = 0; r < B.n; ++r) {
        MixFields& F = A.f[r];
        F.x          = B.xs[r] ? B.xs[r]->data : nullptr;
        F.r          = B.rs[r]->data;
        F.p          = B.p[r]->data;
        F.p_norm     = B.p[r]->norm;
        F.v          = B.v[r] ? B.v[r]->data : nullptr;
        F.v_norm     = B.v[r] ? B.v[r]->norm : nullptr;
        F.sc         = B.sc[r];
    }
    A.nrhs = B.n;
    A.H    = B.rs[0]->geom.seo / 2;
    A.ss   = B.rs[0]->geom.stride / 2;
    return A;
}

template <int PB>
int mix_update_batch(c2q_ctx* ctx, const MixBatch& B)
{
    MixArgs A        = mix_args(B);
    const int blocks = (A.H + MIX_THREADS - 1) / MIX_THREADS * B.n;
    int rc           = ensure_partials(ctx, blocks);
    if (rc) return rc;
    A.red.partials = ctx->partials;
    A.red.ticket   = ctx->ticket;
    A.red.result   = ctx->red_result;
    A.red.sc       = ctx->scalars;
    A.red.fin      = FIN_CG_BETA;
    C2Q_CUDA(ctx, launch_dep(ctx->pdl, mix_update_kernel<PB>, dim3(blocks), dim3(MIX_THREADS), 0, ctx->stream, A));
    ctx->launches++;
    return C2Q_OK;
}

template <int PB>
int mix_p_batch(c2q_ctx* ctx, const MixBatch& B)
{
    const MixArgs A  = mix_args(B);
    const int blocks = (A.H + MIX_THREADS - 1) / MIX_THREADS * B.n;
    C2Q_CUDA(ctx, launch_dep(ctx->pdl, mix_p_kernel<PB>, dim3(blocks), dim3(MIX_THREADS), 0, ctx->stream, A));
    ctx->launches++;
    return C2Q_OK;
}

// x += x_s + alpha p (alpha from `sc`; sc null: x += x_s), x_s = 0
template <int PB>
int accumulate(c2q_ctx* ctx, c2q_spinor_eo* x, c2q_spinor_eo* xs, const c2q_spinor_eo* p, const SolverScalars* sc)
{
    const int n = x->geom.seo;
    accumulate_kernel<PB><<<(n + BLAS_THREADS - 1) / BLAS_THREADS, BLAS_THREADS, 0, ctx->stream>>>(
        sptr<64>(x), sptr<32>(xs), sptr<PB>(p), sc, n, x->geom.stride);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

// A reliable update's scalars: beta rescaled to the true residual r2 (the
// search direction is kept), omega = resid = r2, alpha = 0 (the deferred x
// update was accumulated).
__global__ void mixed_rescale_kernel(SolverScalars* s, double r2)
{
    if (threadIdx.x != 0) return;
    s->beta[0] *= r2 / s->resid;
    s->beta[1] *= r2 / s->resid;
    s->omega[0] = r2;
    s->omega[1] = 0.0;
    s->resid    = r2;
    s->alpha[0] = 0.0;
    s->alpha[1] = 0.0;
}

// Mixed-precision CG on a batch of right-hand sides that share the operator:
// the right-hand sides iterate in lockstep (every sweep and vector update is
// one launch over the active ones, so each link is read once per batch), each
// with its own device scalars, its own pipelined residual monitoring and its
// own FP64 reliable updates, and leaves the batch when it converges.  With
// use_graph the iterations run as a captured CUDA graph (recaptured whenever
// the set of active right-hand sides changes).  One right-hand side is the
// plain mixed-precision CG.
struct RhsState {
    double b2 = 0, thr = 0, r2 = 0, resid = 0, maxrr = 0, r2_confirmed = -1;
    int status = C2Q_DID_NOT_SOLVE, iters = 0, reliable = 0, skip_upto = -1, sweeps = 0;
    bool active = false;
};

struct BatchGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<int> set;
    long long kernels = 0;
    ~BatchGraph() { reset(); }
    void reset()
    {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        set.clear();
    }
};

template <int PB>
int cg_mixed_batch(c2q_ctx* ctx, c2q_spinor_eo* const* x, int op, const c2q_gauge* g, const c2q_spinor_eo* const* b,
                   int n, double kappa, double mubar, int action, const c2q_solver_params* P, c2q_solve_report* reps)
{
    if (n < 1 || n > PK_MAX_RHS) return fail(ctx, C2Q_BAD_ARG, "batch size must be 1..16");
    const c2q_lattice& lat = x[0]->lat;
    Fields F;
    int rc = make_fields(ctx, lat, 64, 3, F, 0);                // r64, a64, b64 (reliable updates)
    if (!rc) rc = make_fields(ctx, lat, 32, 2 * n, F, 3);        // rs, xs per right-hand side
    if (!rc) rc = make_fields(ctx, lat, PB, 4 * n, F, 3 + 2 * n);  // p, v, t1, t2 per right-hand side
    if (rc) return rc;
    c2q_spinor_eo *r64 = &F.f[0], *a64 = &F.f[1], *b64 = &F.f[2];
    c2q_spinor_eo *rs[PK_MAX_RHS], *xs[PK_MAX_RHS], *p[PK_MAX_RHS], *v[PK_MAX_RHS], *t1[PK_MAX_RHS],
        *t2[PK_MAX_RHS];
    for (int k = 0; k < n; ++k) {
        rs[k] = &F.f[3 + 2 * k];
        xs[k] = &F.f[4 + 2 * k];
        p[k]  = &F.f[3 + 2 * n + 4 * k];
        v[k]  = &F.f[4 + 2 * n + 4 * k];
        t1[k] = &F.f[5 + 2 * n + 4 * k];
        t2[k] = &F.f[6 + 2 * n + 4 * k];
    }
    // inner sweeps in the temporal gauge (QplusQminus_eo with pure-phase T weights):
    // residuals enter as G r, increments leave as G^dagger x_s
    const bool use_tg = op == C2Q_OP_QPLUSQMINUS_EO && P->use_temporal_gauge && tg_applicable(lat);
    const int gk      = use_tg ? gkind_tg(gkind_for(PB, P->use_rec12)) : gkind_for(PB, P->use_rec12);
    // FP64 residuals of the intermediate reliable updates on 12-real FP64 links
    // when 12-real links were asked for and the uploaded field is SU(3) to
    // rounding (row 2 rebuilt in FP64: the same operator); the residual that
    // decides convergence, and the one reported, always use the links as uploaded
    const int gk64 = gk64_for(g, P->use_rec12);
    rc             = gauge_ensure(const_cast<c2q_gauge*>(g), gk);
    if (!rc) rc = gauge_ensure(const_cast<c2q_gauge*>(g), gk64);
    if (rc) return rc;
    SolverScalars* dsc = nullptr;
    C2Q_CUDA(ctx, cudaMallocAsync(&dsc, n * sizeof(SolverScalars), ctx->stream));
    struct Free {
        c2q_ctx* c;
        void* q;
        ~Free() { cudaFreeAsync(q, c->stream); }
    } free_dsc{ctx, dsc};
    C2Q_CUDA(ctx, cudaMemsetAsync(dsc, 0, n * sizeof(SolverScalars), ctx->stream));
    if (!ctx->batch_ring) {
        C2Q_CUDA(ctx, cudaMallocHost(&ctx->batch_ring, 4 * PK_MAX_RHS * 4 * sizeof(double)));
        C2Q_CUDA(ctx, cudaHostGetDevicePointer((void**)&ctx->batch_ring_dev, ctx->batch_ring, 0));
    }
    const double delta = P->reliable_delta > 0 ? P->reliable_delta : 0.1;
    SolveClock clock(ctx);

    auto write_one = [&](int k, const SolverScalars& h) -> int {
        memcpy(ctx->host_pinned, &h, sizeof(SolverScalars));
        const int rc1 = pinned_copy(ctx, dsc + k, 0, ctx->host_pinned_dev, 0, sizeof(SolverScalars));
        if (rc1) return rc1;
        C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        return C2Q_OK;
    };

    auto to_inner = [&](c2q_spinor_eo* out, const c2q_spinor_eo* in) -> int {
        return use_tg ? tg_to_inner(ctx, g, out, in) : launch_convert(ctx, out, in);
    };
    auto take_out = [&](int k, const SolverScalars* sc) -> int {
        return use_tg ? tg_accumulate(ctx, g, x[k], xs[k], p[k], sc) : accumulate<PB>(ctx, x[k], xs[k], p[k], sc);
    };

    // ---- initial residuals
    RhsState S[PK_MAX_RHS];
    for (int k = 0; k < n; ++k) {
        RhsState& s = S[k];
        rc          = saxpy_norm(ctx, r64, Cx{0, 0}, b[k], b[k], FIN_STORE_RESULT, &s.b2);
        if (rc) return rc;
        s.thr     = stop_threshold(P, s.b2);
        double x2 = 0;
        rc        = norm2(ctx, x[k], &x2);
        if (rc) return rc;
        if (x2 == 0.0) {  // r = b - A 0 = b
            rc   = to_inner(rs[k], b[k]);
            s.r2 = s.b2;
        } else {
            rc = true_residual(ctx, op, g, x[k], b[k], kappa, mubar, action, r64, a64, b64, &s.r2, &s.sweeps, G64);
            if (!rc) rc = to_inner(rs[k], r64);
        }
        if (rc) return rc;
        s.resid = s.r2;
        // r = 0 (a zero source with a zero start): x is exact and alpha would be 0/0
        if (s.r2 < s.thr || s.r2 == 0.0) {
            s.status       = 0;
            s.r2_confirmed = s.r2;
            continue;
        }
        rc = c2q_spinor_eo_zero(xs[k]);
        if (!rc) rc = launch_convert(ctx, p[k], rs[k]);
        SolverScalars h0{};
        h0.omega[0] = s.r2;
        if (!rc) rc = write_one(k, h0);
        if (rc) return rc;
        s.maxrr  = std::sqrt(s.r2);
        s.active = true;
    }

    // ---- iterations
    const int per_apply = op == C2Q_OP_QPLUSQMINUS_EO ? 4 : 2;
    // QplusQminus_eo: the solution update x_s += alpha p rides in the third sweep
    // and the residual update in the last one; otherwise x_s += alpha p is
    // deferred to the next mix_p or to the reliable-update accumulation
    const bool fused    = op == C2Q_OP_QPLUSQMINUS_EO;
    const bool graphs   = P->use_graph && !ctx->profiling;
    BatchGraph graph;
    auto body = [&](const std::vector<int>& A, bool with_p) -> int {
        const int m = (int)A.size();
        MixBatch MB;
        MB.n = m;
        c2q_spinor_eo *outs[PK_MAX_RHS], *T1[PK_MAX_RHS], *T2[PK_MAX_RHS];
        const c2q_spinor_eo* ins[PK_MAX_RHS];
        SolverScalars* scs[PK_MAX_RHS];
        for (int i = 0; i < m; ++i) {
            const int k = A[i];
            MB.xs[i]    = xs[k];
            MB.rs[i]    = rs[k];
            MB.p[i]     = p[k];
            MB.v[i]     = v[k];
            MB.sc[i]    = dsc + k;
            outs[i]     = v[k];
            ins[i]      = p[k];
            scs[i]      = dsc + k;
            T1[i]       = t1[k];
            T2[i]       = t2[k];
        }
        if (fused) {
            // p = r + beta p; then Q+Q- p: (p, Q+Q- p) = |Q- p|^2 -> alpha after the
            // second sweep, the third sweep updates x_s += alpha p and the last one
            // r -= alpha Q+Q- p with |r|^2 -> beta (v is never stored)
            c2q_spinor_eo *R[PK_MAX_RHS], *X[PK_MAX_RHS];
            for (int i = 0; i < m; ++i) {
                R[i]     = rs[A[i]];
                X[i]     = xs[A[i]];
                MB.xs[i] = nullptr;
            }
            int e = with_p ? mix_p_batch<PB>(ctx, MB) : 0;
            if (!e)
                e = apply_operator_batch(ctx, op, m, outs, g, gk, ins, kappa, mubar, action, T1, T2, DOT_Y, ins,
                                         FIN_CG_ALPHA, scs, nullptr, R, X);
            return e;
        }
        int e = with_p ? mix_p_batch<PB>(ctx, MB) : 0;  // x += alpha p (previous), p = r + beta p
        if (!e)  // v = A p with (p, v) -> alpha
            e = apply_operator_batch(ctx, op, m, outs, g, gk, ins, kappa, mubar, action, T1, T2, DOT_Y, ins,
                                     FIN_CG_ALPHA, scs, nullptr);
        if (!e) e = mix_update_batch<PB>(ctx, MB);  // r -= alpha v, |r|^2 -> beta
        return e;
    };
    // Pipelined residual monitoring: every iteration copies |r|^2 and the
    // division flag of all right-hand sides into a pinned ring slot and
    // records an event; the host reads iteration k-1 while iteration k runs
    // and applies its decisions after iteration k.
    std::vector<int> hist[4], act;
    int iter = 0;
    for (iter = 0; iter < P->cgmax; ++iter) {
        act.clear();
        for (int k = 0; k < n; ++k)
            if (S[k].active) act.push_back(k);
        if (act.empty()) break;
        hist[iter % 4] = act;
        if (graphs && iter > 0) {
            if (graph.set != act) {
                graph.reset();
                cudaGraph_t gr     = nullptr;
                const long long l0 = ctx->launches;
                C2Q_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
                const int eb         = body(act, true);
                const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &gr);
                if (eb) {
                    if (gr) cudaGraphDestroy(gr);
                    return eb;
                }
                C2Q_CUDA(ctx, ec);
                const cudaError_t ei = cudaGraphInstantiate(&graph.exec, gr, 0);
                cudaGraphDestroy(gr);
                C2Q_CUDA(ctx, ei);
                graph.set     = act;
                graph.kernels = ctx->launches - l0;
                ctx->launches = l0;
            }
            C2Q_CUDA(ctx, cudaGraphLaunch(graph.exec, ctx->stream));
            ctx->launches += graph.kernels;
        } else {
            rc = body(act, iter > 0);
            if (rc) return rc;
        }
        for (int k : act) S[k].sweeps += per_apply;
        rc = ring_push(ctx, iter, ctx->batch_ring_dev + (size_t)(iter % 4) * PK_MAX_RHS * 4, &dsc[0].resid,
                       sizeof(SolverScalars), 4 * sizeof(double), n);
        if (rc) return rc;
        if (iter == 0) continue;
        C2Q_CUDA(ctx, cudaEventSynchronize(ctx->ring_ev[(iter - 1) % 4]));
        const double* prev = ctx->batch_ring + (size_t)((iter - 1) % 4) * PK_MAX_RHS * 4;
        for (int k : hist[(iter - 1) % 4]) {
            RhsState& s = S[k];
            if (!s.active || iter - 1 <= s.skip_upto) continue;
            const double resid = prev[4 * k];
            int bad            = 0;
            memcpy(&bad, prev + 4 * k + 3, sizeof(int));  // SolverScalars::flag follows resid and aux[2]
            s.resid = resid;
            if (resid != resid || bad) {
                s.status = C2Q_SOLVER_STUCK;
                s.iters  = iter;
                s.active = false;
                rc       = take_out(k, nullptr);  // keep what was gained
                if (rc) return rc;
                continue;
            }
            const double rn = std::sqrt(resid);
            if (rn > s.maxrr) s.maxrr = rn;
            if (rn < delta * s.maxrr || resid < s.thr) {
                // reliable update in FP64 after iteration `iter`
                // (an update expected to be the last one uses the uploaded links;
                // one that converges unexpectedly on 12-real links is confirmed on them)
                rc = take_out(k, fused ? nullptr : dsc + k);
                const int gk_upd = resid < s.thr ? G64 : gk64;
                if (!rc)
                    rc = true_residual(ctx, op, g, x[k], b[k], kappa, mubar, action, r64, a64, b64, &s.r2, &s.sweeps,
                                       gk_upd);
                if (!rc && gk_upd != G64 && s.r2 < s.thr)
                    rc = true_residual(ctx, op, g, x[k], b[k], kappa, mubar, action, r64, a64, b64, &s.r2, &s.sweeps,
                                       G64);
                if (rc) return rc;
                ++s.reliable;
                s.resid = s.r2;
                if (s.r2 < s.thr) {
                    s.status       = iter + 1;
                    s.iters        = iter + 1;
                    s.r2_confirmed = s.r2;
                    s.active       = false;
                    continue;
                }
                rc = to_inner(rs[k], r64);
                if (rc) return rc;
                s.maxrr = std::sqrt(s.r2);
                // keep the search direction; rescale beta to the true residual (on
                // the device: the scalars never cross to the host here)
                mixed_rescale_kernel<<<1, 32, 0, ctx->stream>>>(dsc + k, s.r2);
                ctx->launches++;
                C2Q_CUDA(ctx, cudaGetLastError());
                s.skip_upto = iter;
            }
        }
    }
    graph.reset();
    for (int k = 0; k < n; ++k)
        if (S[k].active) {  // out of iterations: keep what was gained
            S[k].iters  = iter;
            S[k].active = false;
            rc          = take_out(k, fused ? nullptr : dsc + k);
            if (rc) return rc;
        }
    const double secs = clock.seconds();
    int worst         = 0;
    for (int k = 0; k < n; ++k) {
        RhsState& s = S[k];
        double r2t  = s.r2_confirmed;
        if (r2t < 0) {
            rc = true_residual(ctx, op, g, x[k], b[k], kappa, mubar, action, r64, a64, b64, &r2t, &s.sweeps, G64);
            if (rc) return rc;
        }
        finish_report(reps ? &reps[k] : nullptr, s.status, s.iters, s.reliable, s.resid,
                      s.b2 > 0 ? std::sqrt(r2t / s.b2) : 0.0, secs, s.sweeps);
        if (s.status < 0 && (worst == 0 || s.status == C2Q_SOLVER_STUCK)) worst = s.status;
    }
    if (worst == C2Q_DID_NOT_SOLVE) fail(ctx, worst, "Solver did not solve in solverMaxIterations iterations");
    if (worst == C2Q_SOLVER_STUCK) fail(ctx, worst, "NAN occured in the mixed-precision CG residual");
    if (worst < 0) return worst;
    return n == 1 ? S[0].status : C2Q_OK;
}

// ------------------------------------------------- solver vector spaces
// The vector space of a Krylov solve with host-side scalars: one FP64 eo field
// (EoSpace), or a full field held as its two parities (FullSpace: the
// reference's physics::lattices::Spinorfield of useEO=false inversions,
// inversion.cpp:98-122).  Both provide the operator, the BLAS calls and the
// inner products of the solvers; a full field's inner products are the sums of
// its two halves'.
struct EoSpace {
    using V = c2q_spinor_eo*;
    c2q_ctx* ctx;
    const c2q_lattice* lat;
    int op;
    const c2q_gauge* g;
    int gk;
    double kappa, mubar;
    int action;
    Fields F;
    c2q_spinor_eo *t1 = nullptr, *t2 = nullptr;
    int sweeps = 0;
    int prec   = 64;  // storage precision of the work fields (gk must match)
    int alloc(int n, std::vector<V>& out)
    {
        int rc = make_fields(ctx, *lat, prec, n + 2, F, 0);
        if (rc) return rc;
        out.resize(n);
        for (int k = 0; k < n; ++k) out[k] = &F.f[k];
        t1 = &F.f[n];
        t2 = &F.f[n + 1];
        return C2Q_OK;
    }
    int apply(V out, V in)
    {
        return apply_operator(ctx, op, out, g, gk, in, kappa, mubar, action, t1, t2, DotSpec{}, &sweeps);
    }
    // the same with a reduction fused into the last sweep
    int apply_dot(V out, V in, const DotSpec& d)
    {
        return apply_operator(ctx, op, out, g, gk, in, kappa, mubar, action, t1, t2, d, &sweeps);
    }
    int saxpy(V out, Cx a, V x, V y)
    {
        BlasSpec sp;
        sp.op  = B_SAXPY;
        sp.out = out;
        sp.x   = x;
        sp.y   = y;
        sp.a   = coef_host(a.re, a.im);
        return launch_blas(ctx, sp);
    }
    int saxsbypz(V out, Cx a, V x, Cx b, V y, V z)
    {
        BlasSpec sp;
        sp.op  = B_SAXSBYPZ;
        sp.out = out;
        sp.x   = x;
        sp.y   = y;
        sp.z   = z;
        sp.a   = coef_host(a.re, a.im);
        sp.b   = coef_host(b.re, b.im);
        return launch_blas(ctx, sp);
    }
    int zero(V f) { return c2q_spinor_eo_zero(f); }
    int dot(V x, V y, Cx* out) { return dot_read(ctx, x, y, out); }
};

struct FullSpace {
    struct V {
        c2q_spinor_eo *e, *o;  // the sites with x+y+z+t even, odd
    };
    c2q_ctx* ctx;
    const c2q_lattice* lat;
    int op;  // C2Q_FULL_*
    const c2q_gauge* g;
    double kappa, mubar;
    int action;
    Fields F;
    EoSpace half;  // the BLAS of one parity (only its context is used)
    int sweeps = 0;
    int alloc(int n, std::vector<V>& out)
    {
        int rc = make_fields(ctx, *lat, 64, 2 * n, F, 0);
        if (rc) return rc;
        out.resize(n);
        for (int k = 0; k < n; ++k) out[k] = V{&F.f[2 * k], &F.f[2 * k + 1]};
        return C2Q_OK;
    }
    int apply(V out, V in)
    {
        sweeps += op == C2Q_FULL_QPLUSQMINUS ? 4 : 2;
        return c2q_apply_full(op, out.e, out.o, g, in.e, in.o, kappa, mubar, action);
    }
    int saxpy(V out, Cx a, V x, V y)
    {
        int rc = half.saxpy(out.e, a, x.e, y.e);
        return rc ? rc : half.saxpy(out.o, a, x.o, y.o);
    }
    int saxsbypz(V out, Cx a, V x, Cx b, V y, V z)
    {
        int rc = half.saxsbypz(out.e, a, x.e, b, y.e, z.e);
        return rc ? rc : half.saxsbypz(out.o, a, x.o, b, y.o, z.o);
    }
    int copy(V to, V from)
    {
        int rc = copy_field(ctx, to.e, from.e);
        return rc ? rc : copy_field(ctx, to.o, from.o);
    }
    int zero(V f)
    {
        int rc = c2q_spinor_eo_zero(f.e);
        return rc ? rc : c2q_spinor_eo_zero(f.o);
    }
    int dot(V x, V y, Cx* out)
    {
        Cx a{0, 0}, b{0, 0};
        int rc = dot_read(ctx, x.e, y.e, &a);
        if (!rc) rc = dot_read(ctx, x.o, y.o, &b);
        *out = {a.re + b.re, a.im + b.im};
        return rc;
    }
    int dot2(V x, V y, Cx* xy, Cx* xx)
    {
        Cx a{0, 0}, b{0, 0}, c{0, 0}, d{0, 0};
        int rc = dot2_read(ctx, x.e, y.e, &a, &c);
        if (!rc) rc = dot2_read(ctx, x.o, y.o, &b, &d);
        *xy = {a.re + b.re, a.im + b.im};
        *xx = {c.re + d.re, c.im + d.im};
        return rc;
    }
};

// ------------------------------------------------------------- BiCGStab
// physics/algorithms/solvers/bicgstab.cpp:566-733 (fast) and :401-564 (save);
// scalars are read back every iteration as the reference does.
template <class S>
int bicgstab_generic(S& sp, typename S::V x, typename S::V b, const c2q_solver_params* P, c2q_solve_report* rep)
{
    c2q_ctx* ctx = sp.ctx;
    std::vector<typename S::V> w;
    int rc = sp.alloc(7, w);
    if (rc) return rc;
    const auto p = w[0], rn = w[1], rhat = w[2], s = w[3], t = w[4], v = w[5], aux = w[6];
    const bool save = P->solver == C2Q_SOLVER_BICGSTAB_SAVE;
    SolveClock clock(ctx);
    Cx bb{0, 0};
    rc = sp.dot(b, b, &bb);
    if (rc) return rc;
    const double b2  = bb.re;
    const double thr = stop_threshold(P, b2);
    const Cx one{1, 0}, mone{-1, 0};
    Cx alpha{1, 0}, omega{1, 0}, rho{1, 0}, rho_next, beta, tmp1, tmp2;
    double resid = std::numeric_limits<double>::quiet_NaN();
    int iter = 0, status = C2Q_DID_NOT_SOLVE;

    auto sqnorm = [&](typename S::V f, double* out) {
        Cx c{0, 0};
        int r = sp.dot(f, f, &c);
        *out  = c.re;
        return r;
    };
    // true residual |b - A x|^2 into *tr (aux receives b - A x)
    auto true_r2 = [&](double* tr) {
        int r = sp.apply(aux, x);
        if (!r) r = sp.saxpy(aux, one, aux, b);
        if (!r) r = sqnorm(aux, tr);
        return r;
    };
    // true-residual confirmation (used by the save variant and by rel_tol)
    auto confirmed = [&](bool* ok) {
        double tr = 0;
        int r     = true_r2(&tr);
        const double lim = P->rel_tol > 0 ? std::max(thr, 0.0) : P->prec;
        *ok              = tr < (P->rel_tol > 0 ? std::max(P->rel_tol * P->rel_tol * b2, P->prec > 0 ? P->prec : 0.0)
                                                 : lim);
        return r;
    };

    if (!save) {
        for (iter = 0; iter < P->cgmax; iter++) {
            if (iter % P->iter_refresh == 0) {
                rc = sp.apply(rn, x);
                if (!rc) rc = sp.saxpy(p, one, rn, b);
                if (!rc) rc = sp.copy(rhat, p);
                if (!rc) rc = sp.copy(rn, p);
                if (!rc) rc = sp.dot(rhat, rn, &rho);
                if (rc) return rc;
            }
            rc = sqnorm(rn, &resid);
            if (rc) return rc;
            if (resid != resid) {
                status = C2Q_SOLVER_STUCK;
                break;
            }
            if (resid < thr) {
                bool ok = true;
                if (P->rel_tol > 0) {
                    rc = confirmed(&ok);
                    if (rc) return rc;
                }
                if (ok) {
                    status = iter;
                    break;
                }
            }
            rc = sp.apply(v, p);
            if (!rc) rc = sp.dot(rhat, v, &tmp1);
            if (rc) return rc;
            alpha = cdiv(rho, tmp1);
            rc    = sp.saxpy(s, alpha, v, rn);
            if (!rc) rc = sp.apply(t, s);
            if (!rc) rc = sp.dot2(t, s, &tmp1, &tmp2);  // (t, s) and (t, t)
            if (rc) return rc;
            omega = cdiv(tmp1, tmp2);
            rc    = sp.saxsbypz(x, alpha, p, omega, s, x);
            if (!rc) rc = sp.saxpy(rn, omega, t, s);
            if (!rc) rc = sp.dot(rhat, rn, &rho_next);
            if (rc) return rc;
            if (std::fabs(rho_next.re) < 1e-25 && std::fabs(rho_next.im) < 1e-25) {
                status = C2Q_SOLVER_STUCK;
                break;
            }
            tmp1 = cdiv(rho_next, rho);
            tmp2 = cdiv(alpha, omega);
            beta = cmulx(tmp1, tmp2);
            tmp1 = cmulx(beta, omega);
            tmp2 = cmulx(mone, tmp1);
            rc   = sp.saxsbypz(p, beta, p, tmp2, v, rn);
            if (rc) return rc;
            rho = rho_next;
        }
    } else {
        for (iter = 0; iter < P->cgmax; iter++) {
            if (iter % P->iter_refresh == 0) {
                rc = sp.zero(v);
                if (!rc) rc = sp.zero(p);
                if (!rc) rc = sp.apply(rn, x);
                if (!rc) rc = sp.saxpy(rn, one, rn, b);
                if (!rc) rc = sp.copy(rhat, rn);
                if (rc) return rc;
                alpha = one;
                omega = one;
                rho   = one;
            }
            rc = sp.dot(rhat, rn, &rho_next);
            if (rc) return rc;
            if (std::fabs(rho_next.re) < 1e-25 && std::fabs(rho_next.im) < 1e-25) {
                status = C2Q_SOLVER_STUCK;
                break;
            }
            tmp1 = cdiv(rho_next, rho);
            rho  = rho_next;
            tmp2 = cdiv(alpha, omega);
            beta = cmulx(tmp1, tmp2);
            tmp1 = cmulx(beta, omega);
            tmp2 = cmulx(mone, tmp1);
            rc   = sp.saxsbypz(p, beta, p, tmp2, v, rn);
            if (!rc) rc = sp.apply(v, p);
            if (!rc) rc = sp.dot(rhat, v, &tmp1);
            if (rc) return rc;
            alpha = cdiv(rho, tmp1);
            rc    = sp.saxpy(s, alpha, v, rn);
            if (!rc) rc = sp.apply(t, s);
            if (!rc) rc = sp.dot2(t, s, &tmp1, &tmp2);  // (t, s) and (t, t)
            if (rc) return rc;
            omega = cdiv(tmp1, tmp2);
            rc    = sp.saxpy(rn, omega, t, s);
            if (!rc) rc = sp.saxsbypz(x, alpha, p, omega, s, x);
            if (!rc) rc = sqnorm(rn, &resid);
            if (rc) return rc;
            if (resid != resid) {
                status = C2Q_SOLVER_STUCK;
                break;
            }
            if (resid < thr) {
                bool ok = false;
                rc      = confirmed(&ok);
                if (rc) return rc;
                if (ok) {
                    status = iter;
                    break;
                }
            }
        }
    }
    double r2t = 0;
    rc         = true_r2(&r2t);
    if (rc) return rc;
    finish_report(rep, status, iter, 0, resid, b2 > 0 ? std::sqrt(r2t / b2) : 0.0, clock.seconds(), sp.sweeps);
    if (status == C2Q_DID_NOT_SOLVE) fail(ctx, status, "Solver did not solve in solverMaxIterations iterations");
    if (status == C2Q_SOLVER_STUCK) fail(ctx, status, "BiCGStab stuck (NaN residual or vanishing rho)");
    return status;
}

// ----------------------------------------------- BiCGStab, device-driven
// The eo BiCGStab above (fast and save variants; the same operations in the
// same order, the same stopping and stuck tests, the same returned iterate)
// with every scalar kept on the device.  The last block of each reduction
// computes alpha, omega, beta, rho and applies the tests (FIN_BI_* in
// reduce.cuh, rounded as the host's complex arithmetic); the BLAS read their
// coefficients from device memory; at the end of each iteration |r|^2 and the
// halt bits go to a ring slot (ring_push), which the host reads one iteration
// behind the queue.  When a test fires it sets
// SolverScalars::halt, and every later BLAS / dslash launch of the solve finds
// it set and leaves at once (RedArgs::halt), so the iteration already queued
// behind the stopping one changes nothing: the solve stops on exactly the
// iterate the reference's loop returns.  A stop that needs the host (the
// true-residual confirmation of the save variant and of rel_tol) clears the
// halt and re-queues the iteration that was skipped.
__global__ void bicg_end_kernel(SolverScalars* s)
{
    if (threadIdx.x != 0) return;
    s->halt      = s->halt | s->halt_next;  // the next iteration's opening test takes effect
    s->halt_next = 0;
}

struct HaltScope {  // the context's launch predicate for the duration of a solve
    c2q_ctx* ctx;
    HaltScope(c2q_ctx* c, const int* h) : ctx(c) { ctx->halt_dev = h; }
    ~HaltScope() { ctx->halt_dev = nullptr; }
};

// The device-driven iteration on an eo vector space: the field set, the
// enqueueing of one fast or save iteration, and the residual ring.
struct BicgLoop {
    c2q_ctx* ctx;
    EoSpace& sp;
    SolverScalars* sc;
    c2q_spinor_eo *p, *rn, *rhat, *s, *t, *v, *aux;
    int A;  // sweeps of one operator application (Aee-type 2, QplusQminus_eo 4)
    int R;  // refresh interval
    DotSpec alpha_dot;
    const Coef one = coef_host(1.0, 0.0), none = coef_host(0.0, 0.0);

    BicgLoop(EoSpace& space, const std::vector<c2q_spinor_eo*>& w, int refresh)
        : ctx(space.ctx), sp(space), sc(space.ctx->scalars), p(w[0]), rn(w[1]), rhat(w[2]), s(w[3]), t(w[4]),
          v(w[5]), aux(w[6]), A(space.op == C2Q_OP_QPLUSQMINUS_EO ? 4 : 2), R(refresh)
    {
        alpha_dot.mode = DOT_Y;  // (rhat, A p) reduced in the operator's last sweep
        alpha_dot.y    = rhat;
        alpha_dot.fin  = FIN_BI_ALPHA;
    }
    int blas(int op, c2q_spinor_eo* out, Coef a, const c2q_spinor_eo* X, Coef bc, const c2q_spinor_eo* Y,
             const c2q_spinor_eo* Z, int dot = 0, int fin = FIN_STORE_RESULT, int fin_arg = 0)
    {
        BlasSpec q;
        q.op      = op;
        q.out     = out;
        q.a       = a;
        q.x       = X;
        q.b       = bc;
        q.y       = Y;
        q.z       = Z;
        q.dot     = dot;
        q.fin     = fin;
        q.fin_arg = fin_arg;
        return launch_blas(ctx, q);
    }
    // (x, y) reductions into a finisher: dot 1 = <x,y>, dot 3 = <x,y> and <x,x>
    int dot(const c2q_spinor_eo* X, const c2q_spinor_eo* Y, int kind, int fin, int fin_arg = 0)
    {
        return blas(B_SAXPY, nullptr, none, X, none, Y, nullptr, kind, fin, fin_arg);
    }
    // bicgstab.cpp:612-723 (the x update, the rn update and the two reductions
    // that follow them run as one pass, B_BICG_XR).  refresh 2: x is zero, so
    // rn = b without applying the operator.
    int fast_iter(c2q_spinor_eo* x, const c2q_spinor_eo* b, int it, int refresh)
    {
        int e = 0;
        if (refresh == 2) {
            e = copy_field(ctx, p, b);
        } else if (refresh) {
            e = sp.apply(rn, x);
            if (!e) e = blas(B_SAXPY, p, one, rn, none, b, nullptr);  // p = b - rn
        }
        if (refresh) {
            if (!e) e = copy_field(ctx, rhat, p);
            if (!e) e = copy_field(ctx, rn, p);
            if (!e) e = dot(rhat, rn, 3, FIN_BI_REFRESH);  // rho = (rhat, rn); resid = (rn, rn); the test
        }
        if (!e) e = sp.apply_dot(v, p, alpha_dot);  // v = A p; tmp1 = (rhat, v); alpha
        if (!e) e = blas(B_SAXPY, s, coef_dev(sc->alpha), v, none, rn, nullptr);  // s = rn - alpha v
        if (!e) e = sp.apply(t, s);
        if (!e) e = dot(t, s, 3, FIN_BI_OMEGA);
        if (!e) {  // x += alpha p + omega s; rn = s - omega t; |rn|^2, (rhat, rn): beta and the tests
            BlasSpec q;
            q.op      = B_BICG_XR;
            q.out     = x;
            q.a       = coef_dev(sc->alpha);
            q.x       = p;
            q.b       = coef_dev(sc->omega);
            q.y       = s;
            q.z       = t;
            q.w       = rhat;
            q.out2    = rn;
            q.dot     = 4;
            q.fin     = FIN_BI_XR;
            q.fin_arg = (it + 1) % R != 0;
            e         = launch_blas(ctx, q);
        }
        if (!e) e = blas(B_SAXSBYPZ, p, coef_dev(sc->beta), p, coef_dev(sc->tmp2), v, rn);
        return e;
    }
    // bicgstab.cpp:445-505 (x is updated before rn here: the two updates are independent)
    int save_iter(c2q_spinor_eo* x, const c2q_spinor_eo* b, bool refresh)
    {
        int e = 0;
        if (refresh) {
            e = sp.zero(v);
            if (!e) e = sp.zero(p);
            if (!e) e = sp.apply(rn, x);
            if (!e) e = blas(B_SAXPY, rn, one, rn, none, b, nullptr, 2, FIN_BIS_INIT);  // rn = b - rn; 1, 1, 1
            if (!e) e = copy_field(ctx, rhat, rn);
        }
        if (!e) e = dot(rhat, rn, 1, FIN_BIS_RHO);
        if (!e) e = blas(B_SAXSBYPZ, p, coef_dev(sc->beta), p, coef_dev(sc->tmp2), v, rn);
        if (!e) e = sp.apply_dot(v, p, alpha_dot);
        if (!e) e = blas(B_SAXPY, s, coef_dev(sc->alpha), v, none, rn, nullptr);
        if (!e) e = sp.apply(t, s);
        if (!e) e = dot(t, s, 3, FIN_BI_OMEGA);
        if (!e) e = blas(B_SAXSBYPZ, x, coef_dev(sc->alpha), p, coef_dev(sc->omega), s, x);
        if (!e) e = blas(B_SAXPY, rn, coef_dev(sc->omega), t, none, s, nullptr, 2, FIN_BI_RESID, 1);
        return e;
    }
    // ring slot k: resid, aux[2], flag, halt -- the first 32 bytes from SolverScalars::resid
    int push(int k)
    {
        static_assert(offsetof(SolverScalars, halt) ==
                          offsetof(SolverScalars, resid) + 3 * sizeof(double) + sizeof(int),
                      "halt follows resid, aux[2] and flag");
        bicg_end_kernel<<<1, 32, 0, ctx->stream>>>(sc);
        ctx->launches++;
        C2Q_CUDA(ctx, cudaGetLastError());
        return ring_push(ctx, k, ctx->host_pinned_dev + 32 + 4 * (k % 4), &sc->resid, 0, 4 * sizeof(double), 1);
    }
    int pop(int k, double* r, int* h)
    {
        C2Q_CUDA(ctx, cudaEventSynchronize(ctx->ring_ev[k % 4]));
        const double* slot = ctx->host_pinned + 32 + 4 * (k % 4);
        *r                 = slot[0];
        memcpy(h, reinterpret_cast<const char*>(slot + 3) + sizeof(int), sizeof(int));
        return C2Q_OK;
    }
};

int bicgstab_dev(EoSpace& sp, c2q_spinor_eo* x, c2q_spinor_eo* b, const c2q_solver_params* P,
                 c2q_solve_report* rep)
{
    c2q_ctx* ctx = sp.ctx;
    std::vector<c2q_spinor_eo*> w;
    int rc = sp.alloc(7, w);
    if (rc) return rc;
    BicgLoop L(sp, w, P->iter_refresh);
    c2q_spinor_eo* const aux = L.aux;
    const bool save          = P->solver == C2Q_SOLVER_BICGSTAB_SAVE;
    SolveClock clock(ctx);
    Cx bb{0, 0};
    rc = sp.dot(b, b, &bb);
    if (rc) return rc;
    const double b2  = bb.re;
    const double thr = stop_threshold(P, b2);
    SolverScalars* sc = ctx->scalars;
    SolverScalars init{};
    init.thr = thr;
    rc       = write_sc(ctx, init);
    if (rc) return rc;
    const Coef one = L.one, none = L.none;
    const int A    = L.A, R = L.R;
    auto blas      = [&](int op, c2q_spinor_eo* out, Coef a, const c2q_spinor_eo* X, Coef bc,
                    const c2q_spinor_eo* Y, const c2q_spinor_eo* Z, int dot = 0, int fin = FIN_STORE_RESULT) {
        return L.blas(op, out, a, X, bc, Y, Z, dot, fin);
    };
    auto fast_iter = [&](int it, bool refresh) { return L.fast_iter(x, b, it, refresh ? 1 : 0); };
    auto save_iter = [&](int, bool refresh) { return L.save_iter(x, b, refresh); };
    auto push      = [&](int k) { return L.push(k); };
    auto pop       = [&](int k, double* r, int* h) { return L.pop(k, r, h); };
    // the true-residual confirmation (save variant, rel_tol); unpredicated
    auto confirmed = [&](bool* ok) -> int {
        ctx->halt_dev = nullptr;
        int e         = sp.apply(aux, x);
        if (!e) e = blas(B_SAXPY, aux, one, aux, none, b, nullptr, 2, FIN_STORE_RESULT);
        double tr[2] = {0, 0};
        if (!e) e = read_scalars(ctx, ctx->red_result, 2, tr);
        ctx->halt_dev = &sc->halt;
        const double lim = P->rel_tol > 0 ? std::max(P->rel_tol * P->rel_tol * b2, P->prec > 0 ? P->prec : 0.0)
                                          : P->prec;
        *ok = tr[0] < lim;
        return e;
    };

    HaltScope scope(ctx, &sc->halt);
    int status = C2Q_DID_NOT_SOLVE, iters = P->cgmax, executed = 0, resume = -1;
    bool skip_refresh = false;
    bool refreshed[4] = {};
    double resid      = std::numeric_limits<double>::quiet_NaN();
    // What a halted slot q means (bits h): 1 stop, 2 resume at `resume`.
    auto settle = [&](int q, int h) -> int {
        const int sweeps_q = (refreshed[q % 4] ? A : 0) + 2 * A;  // all of iteration q
        if (h & HALT_STUCK) {  // fast: after the x update; save: at the top
            executed += save ? (refreshed[q % 4] ? A : 0) : sweeps_q;
            status = C2Q_SOLVER_STUCK;
            iters  = q;
            return 1;
        }
        if (h & HALT_NAN) {  // fast: the refresh's test; save: the end of q
            executed += save ? sweeps_q : A;
            status = C2Q_SOLVER_STUCK;
            iters  = q;
            return 1;
        }
        int j;
        if (save) {
            executed += sweeps_q;
            j = q;
        } else if (h & HALT_CONV) {  // the test of refresh iteration q
            executed += A;
            j = q;
        } else {  // NAN_NEXT / CONV_NEXT: the test at the top of q + 1
            executed += sweeps_q;
            j = q + 1;
            if (j >= P->cgmax) return 1;  // the reference leaves its loop first
            if (h & HALT_NAN_NEXT) {
                status = C2Q_SOLVER_STUCK;
                iters  = j;
                return 1;
            }
        }
        bool ok = true;
        if (save || P->rel_tol > 0) {
            const int s0 = sp.sweeps;
            rc           = confirmed(&ok);
            executed += sp.sweeps - s0;
            if (rc) return -1;
        }
        if (ok) {
            status = j;
            iters  = j;
            return 1;
        }
        // the iterated residual drifted: clear the halt and carry on where the reference does
        SolverScalars hs;
        rc = read_sc(ctx, &hs);
        if (rc) return -1;
        hs.halt = hs.halt_next = 0;
        rc                     = write_sc(ctx, hs);
        if (rc) return -1;
        if (save) {
            resume = q + 1;
        } else {
            resume       = j;
            skip_refresh = (h & HALT_CONV) != 0;  // its refresh ran; the rest of it did not
        }
        return 2;
    };
    int k = 0, first = 0;
    for (;;) {
        const bool more = k < P->cgmax;
        if (more) {
            const bool refresh = k % R == 0 && !skip_refresh;
            skip_refresh       = false;
            refreshed[k % 4]   = refresh;
            rc                 = save ? save_iter(k, refresh) : fast_iter(k, refresh);
            if (!rc) rc = push(k);
            if (rc) return rc;
        }
        if (k > first) {  // slot k - 1: read one iteration behind the queue
            int h = 0;
            rc    = pop(k - 1, &resid, &h);
            if (rc) return rc;
            if (h) {
                const int r = settle(k - 1, h);
                if (r < 0) return rc;
                if (r == 1) break;
                k = first = resume;
                continue;
            }
            executed += (refreshed[(k - 1) % 4] ? A : 0) + 2 * A;
        }
        if (!more) break;
        ++k;
    }
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->halt_dev = nullptr;
    double r2t    = 0;
    {
        rc = sp.apply(aux, x);
        if (!rc) rc = blas(B_SAXPY, aux, one, aux, none, b, nullptr, 2, FIN_STORE_RESULT);
        double tr[2] = {0, 0};
        if (!rc) rc = read_scalars(ctx, ctx->red_result, 2, tr);
        if (rc) return rc;
        r2t = tr[0];
        executed += A;
    }
    sp.sweeps = executed;
    finish_report(rep, status, iters, 0, resid, b2 > 0 ? std::sqrt(r2t / b2) : 0.0, clock.seconds(), executed);
    if (status == C2Q_DID_NOT_SOLVE) fail(ctx, status, "Solver did not solve in solverMaxIterations iterations");
    if (status == C2Q_SOLVER_STUCK) fail(ctx, status, "BiCGStab stuck (NaN residual or vanishing rho)");
    return status;
}

int bicgstab_impl(c2q_ctx* ctx, c2q_spinor_eo* x, int op, const c2q_gauge* g, const c2q_spinor_eo* b,
                  double kappa, double mubar, int action, const c2q_solver_params* P, c2q_solve_report* rep)
{
    EoSpace sp{ctx, &x->lat, op, g, gk64_for(g, P->use_rec12), kappa, mubar, action};
    return bicgstab_dev(sp, x, const_cast<c2q_spinor_eo*>(b), P, rep);
}

// Mixed-precision BiCGStab (no counterpart in the reference, whose solvers run
// in FP64), with reliable updates: the device-driven BiCGStab iteration above
// (fast variant) runs on FP32 or FP16 fields and links and accumulates its
// solution increment xs there; whenever its iterated residual has dropped by
// reliable_delta since the last update, or below the stopping threshold, x +=
// xs in FP64 and the FP64 true residual r = b - A x replaces the iterated one
// (with rho = (rhat, r)), and the iteration goes on with its search direction,
// shadow residual and scalars kept -- the Krylov space survives the updates
// (Sleijpen and van der Vorst's reliable updates for BiCGStab).  The stopping
// test (prec / rel_tol) is applied to the FP64 true residual, confirmed on the
// links as uploaded.  A vanishing rho restarts the iteration from the true
// residual (twice in a row without progress: SolverStuck); cgmax bounds the
// iterations.  The save variant's defining step, confirming convergence with
// the true residual, is what every update does, so both settings run this.
template <int PB>
int bicgstab_mixed(c2q_ctx* ctx, c2q_spinor_eo* x, int op, const c2q_gauge* g, const c2q_spinor_eo* b,
                   double kappa, double mubar, int action, const c2q_solver_params* P, c2q_solve_report* rep)
{
    const auto t0  = std::chrono::steady_clock::now();
    // 12-real FP64 residuals only where they are the uploaded operator; the
    // residual that stops the solve is confirmed on the links as uploaded
    const int gk64 = gk64_for(g, P->use_rec12);
    const int gk   = gkind_for(PB, P->use_rec12);
    int rc         = gauge_ensure(const_cast<c2q_gauge*>(g), gk);
    if (!rc) rc = gauge_ensure(const_cast<c2q_gauge*>(g), gk64);
    if (rc) return rc;
    Fields F64, FB;
    rc = make_fields(ctx, x->lat, 64, 4, F64, 0);
    if (!rc) rc = make_fields(ctx, x->lat, PB, 2, FB, 0);
    if (rc) return rc;
    c2q_spinor_eo *r64 = &F64.f[0], *a64 = &F64.f[1], *b64 = &F64.f[2], *e64 = &F64.f[3];
    c2q_spinor_eo *rin = &FB.f[0], *xs = &FB.f[1];
    EoSpace sp{ctx, &x->lat, op, g, gk, kappa, mubar, action};
    sp.prec = PB;
    std::vector<c2q_spinor_eo*> w;
    rc = sp.alloc(7, w);
    if (rc) return rc;
    BicgLoop L(sp, w, 1 << 30);  // no periodic refresh: the reliable updates replace it
    double b2 = 0;
    rc        = norm2(ctx, b, &b2);
    if (rc) return rc;
    const double thr   = stop_threshold(P, b2);
    const double delta = P->reliable_delta > 0 && P->reliable_delta < 1 ? P->reliable_delta : 0.003;
    int iters = 0, updates = 0, sweeps = 0, status = C2Q_DID_NOT_SOLVE, stuck_run = 0;
    double r2 = 0, maxr = 0;

    // x += xs in FP64, then r = b - A x; returns 1 when r meets the stopping test
    auto reliable = [&](bool* conv) -> int {
        *conv  = false;
        int e  = launch_convert(ctx, e64, xs);
        BlasSpec up;  // x = x - (-1) e
        up.op  = B_SAXPY;
        up.out = x;
        up.x   = e64;
        up.y   = x;
        up.a   = coef_host(-1.0, 0.0);
        if (!e) e = launch_blas(ctx, up);
        if (!e) e = c2q_spinor_eo_zero(xs);
        if (!e) e = true_residual(ctx, op, g, x, b, kappa, mubar, action, r64, a64, b64, &r2, &sweeps, gk64);
        if (!e && gk64 != G64 && r2 < thr)
            e = true_residual(ctx, op, g, x, b, kappa, mubar, action, r64, a64, b64, &r2, &sweeps, G64);
        if (e) return e;
        *conv = r2 < thr || r2 == 0.0;
        maxr  = std::sqrt(r2);
        return C2Q_OK;
    };
    // a fresh start of the iteration from the FP64 residual: rin = r, xs = 0
    SolverScalars init{};  // thr 0: the iteration never stops itself; the host tests the FP64 residual
    auto restart = [&]() -> int {
        int e = launch_convert(ctx, rin, r64);
        if (!e) e = write_sc(ctx, init);
        return e;
    };

    rc = c2q_spinor_eo_zero(xs);
    if (!rc) rc = true_residual(ctx, op, g, x, b, kappa, mubar, action, r64, a64, b64, &r2, &sweeps, G64);
    if (rc) return rc;
    maxr = std::sqrt(r2);
    if (r2 < thr || r2 == 0.0) {
        status = 0;
    } else if (r2 != r2) {
        status = C2Q_SOLVER_STUCK;
    } else {
        rc = restart();
        if (rc) return rc;
        HaltScope scope(ctx, &ctx->scalars->halt);
        int refresh = 2, skip_upto = -1;
        for (int k = 0;; ++k) {
            const bool more = k < P->cgmax;
            if (more) {
                rc = L.fast_iter(xs, rin, k, refresh);
                if (!rc) rc = L.push(k);
                if (rc) return rc;
                refresh = 0;
            }
            if (k == 0) continue;
            double res = 0;
            int h      = 0;
            rc         = L.pop(k - 1, &res, &h);
            if (rc) return rc;
            if (k - 1 <= skip_upto) {  // queued before the last update, which took in what it did
                if (!h) ++iters;        // (it ran, unless a halt stopped it)
                if (!more) break;
                continue;
            }
            ++iters;
            const bool stuck = (h & HALT_STUCK) != 0;
            if ((h & (HALT_NAN | HALT_NAN_NEXT)) || res != res) {
                status = C2Q_SOLVER_STUCK;
                break;
            }
            if (stuck || res < delta * delta * maxr * maxr || res < thr || !more) {
                // an update after the iteration queued behind this one (or a
                // restart where rho vanished); nothing is predicated meanwhile
                ctx->halt_dev       = nullptr;
                const double before = maxr;
                bool conv           = false;
                rc                  = reliable(&conv);
                if (rc) return rc;
                ++updates;
                if (conv) {
                    status = iters;
                    break;
                }
                if (r2 != r2) {
                    status = C2Q_SOLVER_STUCK;
                    break;
                }
                if (!more) break;
                if (stuck) {
                    stuck_run = maxr < 0.5 * before ? 0 : stuck_run + 1;
                    if (stuck_run >= 2) {
                        status = C2Q_SOLVER_STUCK;
                        break;
                    }
                    rc      = restart();
                    refresh = 2;
                } else {
                    // the true residual replaces the iterated one: rn = r, rho = (rhat, rn)
                    rc = launch_convert(ctx, L.rn, r64);
                    if (!rc) rc = L.dot(L.rhat, L.rn, 1, FIN_BI_RHO);
                }
                if (rc) return rc;
                ctx->halt_dev = &ctx->scalars->halt;
                skip_upto     = k;
            } else if (!more) {
                break;
            }
        }
    }
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    sweeps += sp.sweeps;
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    finish_report(rep, status, iters, updates, r2, b2 > 0 ? std::sqrt(r2 / b2) : 0.0, secs, sweeps);
    if (status == C2Q_DID_NOT_SOLVE) fail(ctx, status, "Solver did not solve in solverMaxIterations iterations");
    if (status == C2Q_SOLVER_STUCK) fail(ctx, status, "mixed-precision BiCGStab stuck (NaN residual or vanishing rho)");
    return status;
}

// CG with host-side scalars, physics/algorithms/solvers/cg.cpp:277-400: the
// residual is refreshed every iter_refresh iterations and checked every
// resid_check_every (|r|^2 < prec; with rel_tol confirmed by the true
// residual).  Used for the full-lattice solves of useEO=false inversions.
template <class S>
int cg_generic(S& sp, typename S::V x, typename S::V b, const c2q_solver_params* P, c2q_solve_report* rep)
{
    c2q_ctx* ctx = sp.ctx;
    std::vector<typename S::V> w;
    int rc = sp.alloc(4, w);
    if (rc) return rc;
    const auto p = w[0], rn = w[1], v = w[2], aux = w[3];
    SolveClock clock(ctx);
    Cx bb{0, 0};
    rc = sp.dot(b, b, &bb);
    if (rc) return rc;
    const double b2  = bb.re;
    const double thr = stop_threshold(P, b2);
    const Cx one{1, 0};
    Cx omega{0, 0}, rho{0, 0}, alpha{0, 0}, beta{0, 0}, omega_next{0, 0};
    double resid = std::numeric_limits<double>::quiet_NaN();
    int iter = 0, status = C2Q_DID_NOT_SOLVE;
    bool force_refresh = false;
    auto true_r2 = [&](double* tr) {
        int r = sp.apply(aux, x);
        if (!r) r = sp.saxpy(aux, one, aux, b);
        Cx c{0, 0};
        if (!r) r = sp.dot(aux, aux, &c);
        *tr = c.re;
        return r;
    };
    for (iter = 0; iter < P->cgmax || iter < P->min_iter; iter++) {
        if (iter % P->iter_refresh == 0 || force_refresh) {
            force_refresh = false;
            rc = sp.apply(rn, x);
            if (!rc) rc = sp.saxpy(rn, one, rn, b);  // rn = b - A x
            if (!rc) rc = sp.copy(p, rn);
            if (!rc) rc = sp.dot(rn, rn, &omega);
            if (rc) return rc;
        }
        rc = sp.apply(v, p);
        if (!rc) rc = sp.dot(p, v, &rho);
        if (rc) return rc;
        alpha = cdiv(omega, rho);
        rc    = sp.saxpy(x, Cx{-alpha.re, -alpha.im}, p, x);  // x += alpha p
        if (!rc) rc = sp.saxpy(rn, alpha, v, rn);           // rn -= alpha v
        if (!rc) rc = sp.dot(rn, rn, &omega_next);
        if (rc) return rc;
        beta  = cdiv(omega_next, omega);
        omega = omega_next;
        if (iter % P->resid_check_every == 0) {
            resid = omega.re;
            if (resid != resid) {
                status = C2Q_SOLVER_STUCK;
                break;
            }
            if (resid < thr && iter >= P->min_iter) {
                if (P->rel_tol > 0) {
                    double r2t = 0;
                    rc         = true_r2(&r2t);
                    if (rc) return rc;
                    if (!(r2t <= P->rel_tol * P->rel_tol * b2 || (P->prec > 0 && r2t < P->prec))) {
                        force_refresh = true;  // the iterated residual drifted: restart from the true residual
                        continue;
                    }
                }
                status = iter;
                break;
            }
        }
        rc = sp.saxpy(p, Cx{-beta.re, -beta.im}, p, rn);  // p = rn + beta p
        if (rc) return rc;
    }
    double r2t = 0;
    rc         = true_r2(&r2t);
    if (rc) return rc;
    finish_report(rep, status, iter, 0, resid, b2 > 0 ? std::sqrt(r2t / b2) : 0.0, clock.seconds(), sp.sweeps);
    if (status == C2Q_DID_NOT_SOLVE) fail(ctx, status, "Solver did not solve in solverMaxIterations iterations");
    if (status == C2Q_SOLVER_STUCK) fail(ctx, status, "NAN occured in the CG residual");
    return status;
}

}  // namespace
}  // namespace c2q

using namespace c2q;

extern "C" {

C2Q_EXPORT void c2q_solver_params_default(c2q_solver_params* p)
{
    if (!p) return;
    p->solver            = C2Q_SOLVER_BICGSTAB;  // meta/parametersSolver.cpp:93
    p->prec              = 1e-23;                // :76-78 (double precision build)
    p->rel_tol           = 0.0;
    p->cgmax             = 1000;                 // :85
    p->iter_refresh      = 100;                  // :84
    p->resid_check_every = 10;                   // :87
    p->min_iter          = 0;
    p->precision         = C2Q_PREC_FP64;
    p->reliable_delta    = 0.003;
    p->use_rec12         = 0;
    p->use_graph         = 0;
    p->use_temporal_gauge = 1;
}

C2Q_EXPORT int c2q_cg(c2q_spinor_eo* x, int op, const c2q_gauge* g, const c2q_spinor_eo* b, double kappa,
                      double mubar, int action, const c2q_solver_params* p, c2q_solve_report* report)
{
    if (!x) return C2Q_BAD_ARG;
    c2q_ctx* ctx = x->ctx;
    int rc       = 0;
    if (!validate(ctx, x, g, b, p, &rc)) return rc;
    if (x == b) return fail(ctx, C2Q_BAD_ARG, "solution and source must be different fields");
    switch (p->precision) {
        case 64: return cg_fp64(ctx, x, op, g, b, kappa, mubar, action, p, report);
        case 32: return cg_mixed_batch<32>(ctx, &x, op, g, &b, 1, kappa, mubar, action, p, report);
        default: return cg_mixed_batch<16>(ctx, &x, op, g, &b, 1, kappa, mubar, action, p, report);
    }
}

C2Q_EXPORT int c2q_bicgstab(c2q_spinor_eo* x, int op, const c2q_gauge* g, const c2q_spinor_eo* b, double kappa,
                            double mubar, int action, const c2q_solver_params* p, c2q_solve_report* report)
{
    if (!x) return C2Q_BAD_ARG;
    c2q_ctx* ctx = x->ctx;
    int rc       = 0;
    if (!validate(ctx, x, g, b, p, &rc)) return rc;
    if (x == b) return fail(ctx, C2Q_BAD_ARG, "solution and source must be different fields");
    switch (p->precision) {
        case 64: return bicgstab_impl(ctx, x, op, g, b, kappa, mubar, action, p, report);
        case 32: return bicgstab_mixed<32>(ctx, x, op, g, b, kappa, mubar, action, p, report);
        default: return bicgstab_mixed<16>(ctx, x, op, g, b, kappa, mubar, action, p, report);
    }
}

C2Q_EXPORT int c2q_cg_multi(c2q_spinor_eo* const* x, int op, const c2q_gauge* g, const c2q_spinor_eo* const* b,
                            int nrhs, double kappa, double mubar, int action, const c2q_solver_params* p,
                            c2q_solve_report* reports)
{
    if (!x || !b || nrhs <= 0 || !x[0]) return C2Q_BAD_ARG;
    c2q_ctx* ctx = x[0]->ctx;
    int rc       = 0;
    for (int k = 0; k < nrhs; ++k) {
        if (!x[k] || !validate(ctx, x[k], g, b[k], p, &rc)) return rc ? rc : C2Q_BAD_ARG;
        if (x[k]->ctx != ctx || !same_lattice(x[k]->lat, x[0]->lat))
            return fail(ctx, C2Q_BAD_ARG, "all right-hand sides must share the context and lattice");
        for (int l = 0; l < nrhs; ++l)
            if (x[k] == b[l] || (l != k && x[k] == x[l]))
                return fail(ctx, C2Q_BAD_ARG, "solutions must be distinct fields, distinct from the sources");
    }
    int worst = 0;
    if (p->precision == 64) {  // the reference's FP64 CG, one right-hand side after the other
        for (int k = 0; k < nrhs; ++k) {
            rc = c2q_cg(x[k], op, g, b[k], kappa, mubar, action, p, reports ? &reports[k] : nullptr);
            if (rc < 0 && (worst == 0 || rc == C2Q_SOLVER_STUCK)) worst = rc;
        }
        return worst;
    }
    // mixed precision: batches of up to 16 right-hand sides share every sweep
    for (int k0 = 0; k0 < nrhs; k0 += PK_MAX_RHS) {
        const int m = std::min(PK_MAX_RHS, nrhs - k0);
        rc          = p->precision == 32
                          ? cg_mixed_batch<32>(ctx, x + k0, op, g, b + k0, m, kappa, mubar, action, p,
                                               reports ? reports + k0 : nullptr)
                          : cg_mixed_batch<16>(ctx, x + k0, op, g, b + k0, m, kappa, mubar, action, p,
                                               reports ? reports + k0 : nullptr);
        if (rc < 0 && rc != C2Q_SOLVER_STUCK && rc != C2Q_DID_NOT_SOLVE) return rc;
        if (rc < 0 && (worst == 0 || rc == C2Q_SOLVER_STUCK)) worst = rc;
    }
    return worst;
}

// Eo branch of invert_M_nf2_upperflavour (physics/algorithms/inversion.cpp:129-236).
// ---- full-lattice solves (useEO=false)
static int full_solve(bool cg, c2q_spinor_eo* x_even, c2q_spinor_eo* x_odd, int op, const c2q_gauge* g,
                      const c2q_spinor_eo* b_even, const c2q_spinor_eo* b_odd, double kappa, double mubar, int action,
                      const c2q_solver_params* p, c2q_solve_report* report)
{
    if (!x_even || !x_odd || !b_even || !b_odd) return C2Q_BAD_ARG;
    c2q_ctx* ctx = x_even->ctx;
    int rc       = 0;
    if (!validate(ctx, x_even, g, b_even, p, &rc) || !validate(ctx, x_odd, g, b_odd, p, &rc)) return rc;
    if (x_even == x_odd || b_even == b_odd || x_even == b_even || x_odd == b_odd || x_even == b_odd ||
        x_odd == b_even)
        return fail(ctx, C2Q_BAD_ARG, "solution and source halves must be four different fields");
    if (op < C2Q_FULL_M_TM_PLUS || op > C2Q_FULL_QPLUSQMINUS)
        return fail(ctx, C2Q_BAD_ARG, "unknown full-lattice fermion matrix");
    if (p->precision != 64) return fail(ctx, C2Q_BAD_ARG, "the full-lattice solvers run in FP64");
    FullSpace sp{ctx, &x_even->lat, op, g, kappa, mubar, action};
    sp.half.ctx = ctx;
    const FullSpace::V x{x_even, x_odd}, b{const_cast<c2q_spinor_eo*>(b_even), const_cast<c2q_spinor_eo*>(b_odd)};
    return cg ? cg_generic(sp, x, b, p, report) : bicgstab_generic(sp, x, b, p, report);
}

C2Q_EXPORT int c2q_cg_full(c2q_spinor_eo* x_even, c2q_spinor_eo* x_odd, int op, const c2q_gauge* g,
                           const c2q_spinor_eo* b_even, const c2q_spinor_eo* b_odd, double kappa, double mubar,
                           int action, const c2q_solver_params* p, c2q_solve_report* report)
{
    return full_solve(true, x_even, x_odd, op, g, b_even, b_odd, kappa, mubar, action, p, report);
}

C2Q_EXPORT int c2q_bicgstab_full(c2q_spinor_eo* x_even, c2q_spinor_eo* x_odd, int op, const c2q_gauge* g,
                                 const c2q_spinor_eo* b_even, const c2q_spinor_eo* b_odd, double kappa, double mubar,
                                 int action, const c2q_solver_params* p, c2q_solve_report* report)
{
    return full_solve(false, x_even, x_odd, op, g, b_even, b_odd, kappa, mubar, action, p, report);
}

// invert_M_nf2_upperflavour, non-eo branch (inversion.cpp:98-122): from a cold
// start, CG on QplusQminus with the source gamma5 b followed by Qminus, or
// BiCGStab on M; result = M^-1 source (host full fields).
C2Q_EXPORT int c2q_perform_inversion_full(c2q_ctx* ctx, double* result, const c2q_gauge* g, const double* source,
                                          double kappa, double mubar, int action, const c2q_solver_params* p,
                                          c2q_solve_report* report)
{
    if (!ctx || !result || !g || !source || !p) return C2Q_BAD_ARG;
    Fields F;
    int rc = make_fields(ctx, g->lat, 64, 6, F, 0);
    if (rc) return rc;
    c2q_spinor_eo *xe = &F.f[0], *xo = &F.f[1], *be = &F.f[2], *bo = &F.f[3], *te = &F.f[4], *to = &F.f[5];
    rc = c2q_convert_to_eoprec(be, bo, source);
    if (!rc) rc = c2q_spinor_eo_cold(xe);
    if (!rc) rc = c2q_spinor_eo_cold(xo);
    if (rc) return rc;
    int conv = 0;
    if (p->solver == C2Q_SOLVER_CG) {
        // tmp = gamma5 b; QplusQminus y = tmp; x = Qminus y
        rc = c2q_gamma5_eo(be);
        if (!rc) rc = c2q_gamma5_eo(bo);
        if (rc) return rc;
        conv = c2q_cg_full(xe, xo, C2Q_FULL_QPLUSQMINUS, g, be, bo, kappa, mubar, action, p, report);
        if (conv < 0) return conv;
        rc = copy_field(ctx, te, xe);
        if (!rc) rc = copy_field(ctx, to, xo);
        if (!rc) rc = c2q_apply_full(C2Q_FULL_QMINUS, xe, xo, g, te, to, kappa, mubar, action);
    } else {
        conv = c2q_bicgstab_full(xe, xo, C2Q_FULL_M_TM_PLUS, g, be, bo, kappa, mubar, action, p, report);
        if (conv < 0) return conv;
    }
    if (!rc) rc = c2q_convert_from_eoprec(result, xe, xo);
    return rc ? rc : conv;
}

C2Q_EXPORT int c2q_perform_inversion_eo(c2q_ctx* ctx, double* result, const c2q_gauge* g, const double* source,
                                        double kappa, double mubar, int action, const c2q_solver_params* p,
                                        c2q_solve_report* report)
{
    if (!ctx || !result || !g || !source || !p) return C2Q_BAD_ARG;
    Fields F;
    int rc = make_fields(ctx, g->lat, 64, 2, F, 0);
    if (rc) return rc;
    const int conv = c2q_perform_inversion_eo_fields(ctx, &F.f[0], &F.f[1], g, source, kappa, mubar, action, p, report);
    if (conv < 0) return conv;
    rc = c2q_convert_from_eoprec(result, &F.f[0], &F.f[1]);
    return rc ? rc : conv;
}

C2Q_EXPORT int c2q_perform_inversion_eo_fields(c2q_ctx* ctx, c2q_spinor_eo* out_even, c2q_spinor_eo* out_odd,
                                               const c2q_gauge* g, const double* source, double kappa, double mubar,
                                               int action, const c2q_solver_params* p, c2q_solve_report* report)
{
    if (!ctx || !out_even || !out_odd || !g || !source || !p) return C2Q_BAD_ARG;
    if (out_even->prec != 64 || out_odd->prec != 64 || !same_lattice(out_even->lat, g->lat) ||
        !same_lattice(out_odd->lat, g->lat))
        return fail(ctx, C2Q_BAD_ARG, "inversion results must be FP64 fields on the gauge field's lattice");
    Fields F;
    int rc = make_fields(ctx, g->lat, 64, 5, F, 0);
    if (rc) return rc;
    c2q_spinor_eo *src_even = &F.f[0], *src_odd = &F.f[1], *tmp1 = &F.f[2], *tmp2 = &F.f[3], *res = &F.f[4];
    const bool tm = action == C2Q_ACTION_TWISTEDMASS;
    // parity-role swap of the reference (issue #387 workaround, inversion.cpp:141-149)
    rc = c2q_convert_to_eoprec(src_odd, src_even, source);
    if (rc) return rc;
    // b_e' = D M^{-1} b_o - b_e  (saxpy(&source_even, one, source_even, tmp), inversion.cpp:159-170)
    if (tm) {
        rc = c2q_tm_sitediagonal(tmp1, src_odd, mubar, C2Q_DIAG_M_TM_INVERSE);
        if (!rc) rc = c2q_dslash_eo(tmp2, g, tmp1, C2Q_EVEN, kappa);
        if (!rc) rc = c2q_saxpy(src_even, 1, 0, src_even, tmp2);
    } else {
        rc = c2q_dslash_eo(tmp1, g, src_odd, C2Q_EVEN, kappa);
        if (!rc) rc = c2q_saxpy(src_even, 1, 0, src_even, tmp1);
    }
    if (!rc) rc = c2q_spinor_eo_cold(res);
    if (rc) return rc;
    c2q_solver_params pb = *p;
    if (p->solver == C2Q_SOLVER_CG) pb.solver = C2Q_SOLVER_BICGSTAB;  // solver=cg tries BiCGStab first (:176-181)
    int conv = c2q_bicgstab(res, C2Q_OP_AEE, g, src_even, kappa, mubar, action, &pb, report);
    if (conv < 0 && conv != C2Q_SOLVER_STUCK && conv != C2Q_DID_NOT_SOLVE) return conv;
    if (conv < 0) {
        if (p->solver != C2Q_SOLVER_CG) return conv;
        // CG fallback on QplusQminus_eo with g5 b, then x = Qminus_eo y (:182-195)
        rc = c2q_gamma5_eo(src_even);
        if (rc) return rc;
        conv = c2q_cg(res, C2Q_OP_QPLUSQMINUS_EO, g, src_even, kappa, mubar, action, p, report);
        if (conv < 0) return conv;
        rc = c2q_apply_eo(C2Q_OP_QMINUS_EO, src_even, g, res, kappa, mubar, action, 0);
        if (!rc) rc = c2q_copyData(res, src_even);
        if (rc) return rc;
    }
    // x_o = -(M^{-1} D x_e + M^{-1} b_o)  (:204-221)
    if (tm) {
        rc = c2q_dslash_eo(tmp2, g, res, C2Q_ODD, kappa);
        if (!rc) rc = c2q_tm_sitediagonal(tmp1, tmp2, mubar, C2Q_DIAG_M_TM_INVERSE);
        if (!rc) rc = c2q_tm_sitediagonal(tmp2, src_odd, mubar, C2Q_DIAG_M_TM_INVERSE);
        if (!rc) rc = c2q_saxpy(tmp1, -1, 0, tmp1, tmp2);
        if (!rc) rc = c2q_sax(tmp1, -1, 0, tmp1);
    } else {
        rc = c2q_dslash_eo(tmp1, g, res, C2Q_ODD, kappa);
        if (!rc) rc = c2q_saxpy(tmp1, -1, 0, tmp1, src_odd);
        if (!rc) rc = c2q_sax(tmp1, -1, 0, tmp1);
    }
    if (rc) return rc;
    // the even sites of the full result are tmp1, the odd ones res (parity roles swapped back)
    rc = c2q_copyData(out_even, tmp1);
    if (!rc) rc = c2q_copyData(out_odd, res);
    return rc ? rc : conv;
}

}  // extern "C"
