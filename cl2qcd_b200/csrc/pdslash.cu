// pdslash.cu -- host side of the paired-site dslash (pdslash.cuh): launches
// for one right-hand side (the FP32 / FP16 branch of launch_dslash) and for
// batches of right-hand sides sharing one gauge field.
#include <cstdio>
#include <cstring>

#include "c2q_host.h"
#include "pdslash.cuh"

namespace c2q {

void pk_dispatch32_c0(const PkParams<32>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s);
void pk_dispatch32_c1(const PkParams<32>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s);
void pk_dispatch16_c0(const PkParams<16>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s);
void pk_dispatch16_c1(const PkParams<16>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s);
bool pk2_dispatch(const PkParams<16>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s);

// Resident blocks per SM of a configuration: its launch bound, or what its
// shared-memory ring leaves room for (228 KB per SM, 1 KB reserved per block).
static int pk_blocks_per_sm(int P, int nl, int cfg)
{
    int minb     = 0;
    size_t bytes = 0;
    if (P == 16 && nl == 6) {
        minb  = cfg ? PkStage<16, 6, 1>::MINB : PkStage<16, 6, 0>::MINB;
        bytes = cfg ? PkStage<16, 6, 1>::BYTES : PkStage<16, 6, 0>::BYTES;
    } else if (P == 16) {
        minb  = cfg ? PkStage<16, 9, 1>::MINB : PkStage<16, 9, 0>::MINB;
        bytes = cfg ? PkStage<16, 9, 1>::BYTES : PkStage<16, 9, 0>::BYTES;
    } else if (nl == 6) {
        minb  = cfg ? PkStage<32, 6, 1>::MINB : PkStage<32, 6, 0>::MINB;
        bytes = cfg ? PkStage<32, 6, 1>::BYTES : PkStage<32, 6, 0>::BYTES;
    } else {
        minb  = cfg ? PkStage<32, 9, 1>::MINB : PkStage<32, 9, 0>::MINB;
        bytes = cfg ? PkStage<32, 9, 1>::BYTES : PkStage<32, 9, 0>::BYTES;
    }
    const int by_smem = (int)((228u * 1024u) / (bytes + 1024u));
    return minb < by_smem ? minb : by_smem;
}

// Grid of a launch: one block per tile, or (grid-stride) as many blocks per
// right-hand side as the GPU holds resident at once.
static int pk_grid(c2q_ctx* ctx, int P, int nl, int cfg, bool persistent, int ntiles, int nrhs)
{
    if (!persistent) return ntiles * nrhs;
    if (ctx->sm_count <= 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, ctx->device);
        ctx->sm_count = n > 0 ? n : 148;
    }
    const int resident = pk_blocks_per_sm(P, nl, cfg) * ctx->sm_count;
    int G              = (resident + nrhs - 1) / nrhs;
    if (G > ntiles) G = ntiles;
    if (G < 1) G = 1;
    return G * nrhs;
}

template <int P>
static void pk_dispatch(const PkParams<P>& prm, int cfg, int nl, int epi, int dot, int blocks, cudaStream_t s)
{
    if constexpr (P == 16) {
        if (cfg)
            pk_dispatch16_c1(prm, nl, epi, dot, blocks, s);
        else
            pk_dispatch16_c0(prm, nl, epi, dot, blocks, s);
    } else {
        if (cfg)
            pk_dispatch32_c1(prm, nl, epi, dot, blocks, s);
        else
            pk_dispatch32_c0(prm, nl, epi, dot, blocks, s);
    }
}

// Autotuner: the first launch of each shape (precision, link format,
// epilogue, reduction, phase pattern, batch size, volume) outside stream
// capture times every configuration -- one warm-up launch, then two timed
// launches each, with the reductions redirected to scratch so the caller's
// solver scalars are untouched -- and keeps the fastest.  The timed launches
// are idempotent (the output depends only on the inputs; the in-place CG
// residual update is timed as the same sweep without it), so tuning does not
// change results.  Shapes first met inside a graph capture use
// configuration 0 and are not recorded.
// A tuning choice c < 4 selects the kernel configuration c & 1 and the grid
// (c >> 1: grid-stride over resident blocks instead of one block per tile).
// Choice 4, for FP16 batches of two or more right-hand sides in the temporal
// gauge (the batched mixed-precision CG), runs two right-hand sides per thread
// (pdslash2.cuh: each link staged and decoded once for both), an odd last one
// with configuration 0.
constexpr int PK_CHOICES    = 2 * PK_CONFIGS;
constexpr int PK_CHOICE_RB2 = PK_CHOICES;

template <int P>
static bool pk_rb2_applies(const PkParams<P>& prm)
{
    return P == 16 && prm.tg && prm.nrhs >= 2;
}

// Launch a sweep with a tuning choice.
template <int P>
static int pk_run(c2q_ctx* ctx, const PkParams<P>& prm, int nl, int epi, int dot, int choice, cudaStream_t s)
{
    if constexpr (P == 16) {
        if (choice == PK_CHOICE_RB2) {
            const int npair = prm.nrhs / 2;
            PkParams<16> a  = prm;
            a.nrhs          = 2 * npair;
            if (!pk2_dispatch(a, nl, epi, dot, prm.ntiles * npair, s))
                return fail(ctx, C2Q_BAD_ARG, "no two-sources-per-thread sweep for this shape");
            if (prm.nrhs & 1) {  // the odd last right-hand side, one per thread
                PkParams<16> b = prm;
                b.r[0]         = prm.r[prm.nrhs - 1];
                b.nrhs         = 1;
                pk_dispatch<16>(b, 0, nl, epi, dot, pk_grid(ctx, 16, nl, 0, false, b.ntiles, 1), s);
            }
            return C2Q_OK;
        }
    }
    const int cfg = choice & 1;
    pk_dispatch<P>(prm, cfg, nl, epi, dot, pk_grid(ctx, P, nl, cfg, choice >> 1, prm.ntiles, prm.nrhs), s);
    return C2Q_OK;
}

template <int P>
static int pk_choose(c2q_ctx* ctx, const PkParams<P>& prm, int nl, int epi, int dot, int* cfg)
{
    *cfg = 0;
    if (ctx->force_choice >= 0) {  // a fixed choice, where it applies to the shape
        const int c = ctx->force_choice;
        *cfg        = (c < PK_CHOICES || (c == PK_CHOICE_RB2 && pk_rb2_applies(prm))) ? c : 0;
        return C2Q_OK;
    }
    // the fused CG updates change their residual or solution in place, so their
    // launches are not repeatable: they take the choice timed on the same sweep
    // without the update
    if (dot == DOT_CGR || dot == DOT_XUPD) dot = DOT_NONE;
    if (!ctx->autotune) return C2Q_OK;
    const unsigned m = prm.c.real_mask;
    const int ph     = prm.tg ? 3 : m == 0xFFu ? 0 : ((m & 0xFCu) == 0xFCu ? 1 : 2);
    std::vector<int> key{P, nl, epi, dot, ph, prm.nrhs, 2 * prm.g.H};
    auto it = ctx->tune.find(key);
    if (it != ctx->tune.end()) {
        *cfg = it->second.cfg;
        return C2Q_OK;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    C2Q_CUDA(ctx, cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return C2Q_OK;
    if (!ctx->tune_scratch)
        C2Q_CUDA(ctx, cudaMalloc(&ctx->tune_scratch, (PK_MAX_RHS + 1) * sizeof(SolverScalars)));
    PkParams<P> t = prm;
    t.red.sc      = ctx->tune_scratch + PK_MAX_RHS;
    t.red.result  = ctx->tune_scratch[PK_MAX_RHS].aux;
    t.red.halt    = nullptr;  // timing launches always run
    for (int r = 0; r < t.nrhs; ++r) {
        t.r[r].sc     = ctx->tune_scratch + r;
        t.r[r].result = nullptr;
    }
    c2q_ctx::TuneEntry e{0, {0, 0, 0, 0, 0}};
    float best       = 0;
    const int nchoice = pk_rb2_applies(prm) ? PK_CHOICES + 1 : PK_CHOICES;
    for (int c = 0; c < nchoice; ++c) {
        int rc = pk_run<P>(ctx, t, nl, epi, dot, c, ctx->stream);
        if (rc) return rc;
        C2Q_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        pk_run<P>(ctx, t, nl, epi, dot, c, ctx->stream);
        pk_run<P>(ctx, t, nl, epi, dot, c, ctx->stream);
        C2Q_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
        C2Q_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
        C2Q_CUDA(ctx, cudaGetLastError());
        float ms = 0;
        C2Q_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        e.us[c] = 500.0f * ms;
        if (c == 0 || e.us[c] < best) {
            best  = e.us[c];
            e.cfg = c;
        }
        ctx->launches += 3 * ((c == PK_CHOICE_RB2 && (t.nrhs & 1)) ? 2 : 1);
    }
    ctx->tune[key] = e;
    *cfg           = e.cfg;
    return C2Q_OK;
}

PkGeom pk_geom(const Geom& g)
{
    PkGeom p;
    p.ns      = g.ns;
    p.nsh     = g.nsh;
    p.nt2     = g.nt / 2;
    p.H       = g.seo / 2;
    p.ss      = g.stride / 2;
    p.vs_h    = g.vs_h;
    p.div_nsh = make_fastdiv((unsigned)g.nsh);
    p.div_ns  = make_fastdiv((unsigned)g.ns);
    return p;
}

static void fill_field(const c2q_spinor_eo* f, const void** d, const float** n)
{
    *d = f ? f->data : nullptr;
    *n = f ? f->norm : nullptr;
}

template <int P>
static int pk_launch(c2q_ctx* ctx, const c2q_gauge* g, int gkind, const PkBatch& B)
{
    PkParams<P> prm;
    memset(&prm, 0, sizeof prm);
    const c2q_spinor_eo* ref = B.out[0];
    for (int r = 0; r < B.n; ++r) {
        PkRhs& R = prm.r[r];
        R.out      = B.out[r]->data;
        R.out_norm = B.out[r]->norm;
        fill_field(B.in[r], &R.in, &R.in_norm);
        fill_field(B.x[r], &R.x, &R.x_norm);
        fill_field(B.y[r], &R.y, &R.y_norm);
        R.sc     = B.sc[r];
        R.result = nullptr;
    }
    prm.nrhs       = B.n;
    prm.pdl        = ctx->pdl;
    prm.gauge      = g->store[gkind].data;
    prm.g          = pk_geom(ref->geom);
    prm.c          = hop_coef(ref->lat, B.kappa);
    if (gkind_is_tg(gkind)) {
        // temporal gauge: the T phases sit in the transformation, the last slice's
        // T hop carries lambda
        prm.tg     = 1;
        prm.lam_re = g->tg_lam_re;
        prm.lam_im = g->tg_lam_im;
        for (int d = 0; d < 2; ++d) {
            prm.c.re[0][d] = 1.0;
            prm.c.im[0][d] = 0.0;
        }
        prm.c.real_mask = 0xFFu;
    }
    // FP16: links in units of 1/32767 and neighbour spinors in units of norm/32767
    if (P == 16) prm.c.scale *= 1.0 / (32767.0 * 32767.0);
    prm.e          = B.e;
    prm.out_parity = B.out_parity;
    prm.ntiles = (prm.g.H + PK_THREADS - 1) / PK_THREADS;
    if (B.dot_mode != DOT_NONE && B.dot_mode != DOT_XUPD) {  // one partial per tile and right-hand side
        int rc0 = ensure_partials(ctx, (size_t)prm.ntiles * B.n);
        if (rc0) return rc0;
    }
    prm.red.partials = ctx->partials;
    prm.red.ticket   = ctx->ticket;
    prm.red.result   = ctx->red_result;
    prm.red.sc       = ctx->scalars;
    prm.red.fin      = B.fin;
    prm.red.halt     = ctx->halt_dev;
    const bool r12   = gkind_is_r12(gkind);  // else 18-real
    const int nl     = r12 ? 6 : 9;
    int choice       = 0;
    int rc           = pk_choose<P>(ctx, prm, nl, B.epi, B.dot_mode, &choice);
    if (rc) return rc;
    c2q_ctx::Timed tm{};
    if (ctx->profiling) {
        tm.a     = profile_event(ctx);
        tm.b     = profile_event(ctx);
        tm.prec  = P;
        tm.sites = (double)ref->geom.seo * B.n;
        // compulsory traffic: every link once per batch, and per right-hand side
        // the input (once through L2), the output and the epilogue operands
        const double sp = P == 32 ? 96.0 : 52.0;
        const double lk = (r12 ? 12.0 : 18.0) * (P == 32 ? 4.0 : 2.0);
        // (the fused residual update stores no output and reads and writes the FP32
        // residual; the fused solution update reads p and reads and writes the FP32 x)
        const double per_rhs = sp * (2.0 + (B.epi == EPI_AXPY ? 1.0 : 0.0) + (B.dot_mode == DOT_Y ? 1.0 : 0.0)) +
                               (B.dot_mode == DOT_CGR ? 192.0 - sp : 0.0) +
                               (B.dot_mode == DOT_XUPD ? 192.0 + sp : 0.0);
        // (temporal gauge: the T links of a site are read only on the two fold slices
        // of the slot layout, 2 of NT/2 each way)
        const double links = gkind_is_tg(gkind) ? 6.0 + 4.0 / ref->lat.nt : 8.0;
        tm.bytes           = (double)ref->geom.seo * (links * lk + B.n * per_rhs);
        cudaEventRecord(tm.a, ctx->stream);
    }
    rc = pk_run<P>(ctx, prm, nl, B.epi, B.dot_mode, choice, ctx->stream);
    if (rc) return rc;
    if (ctx->profiling) {
        cudaEventRecord(tm.b, ctx->stream);
        ctx->timed.push_back(tm);
    }
    ctx->launches += choice == PK_CHOICE_RB2 && (B.n & 1) ? 2 : 1;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

int launch_pdslash(c2q_ctx* ctx, const c2q_gauge* g, int gkind, const PkBatch& B)
{
    if (B.n < 1 || B.n > PK_MAX_RHS) return fail(ctx, C2Q_BAD_ARG, "batch size must be 1..16");
    const c2q_spinor_eo* ref = B.out[0];
    const int P              = ref->prec;
    for (int r = 0; r < B.n; ++r) {
        const bool cgr = B.dot_mode == DOT_CGR, xup = B.dot_mode == DOT_XUPD;
        for (const c2q_spinor_eo* f :
             {(const c2q_spinor_eo*)B.out[r], B.in[r], B.x[r], cgr || xup ? nullptr : B.y[r]}) {
            if (!f) continue;
            if (f->prec != P || !same_lattice(f->lat, ref->lat))
                return fail(ctx, C2Q_BAD_ARG, "fields of a batch differ in precision or lattice");
        }
        if ((cgr || xup) &&
            (!B.y[r] || B.y[r]->prec != 32 || !same_lattice(B.y[r]->lat, ref->lat) || !B.sc[r] || B.y[r] == B.out[r]))
            return fail(ctx, C2Q_BAD_ARG, "a fused CG update needs a separate FP32 field and solver scalars");
        if (cgr && B.epi != EPI_AXPY) return fail(ctx, C2Q_BAD_ARG, "the fused residual update follows EPI_AXPY");
        if (xup && (B.epi == EPI_AXPY || !B.x[r] || B.x[r] == B.out[r]))
            return fail(ctx, C2Q_BAD_ARG, "the fused solution update needs p and EPI_PLAIN or EPI_DIAG");
        if (!B.in[r] || B.out[r] == B.in[r]) return fail(ctx, C2Q_BAD_ARG, "dslash output must not alias its input");
        if (B.epi == EPI_AXPY && !B.x[r]) return fail(ctx, C2Q_BAD_ARG, "missing axpy operand");
        if (B.dot_mode == DOT_Y && !B.y[r]) return fail(ctx, C2Q_BAD_ARG, "missing dot partner");
    }
    const bool links_ok = P == 32 ? (gkind == G32 || gkind == G32R12 || gkind == G32TG || gkind == G32R12TG)
                                  : (gkind == G16 || gkind == G16R12 || gkind == G16TG || gkind == G16R12TG);
    if (!links_ok) return fail(ctx, C2Q_BAD_ARG, "gauge precision mismatch");
    if (gkind_is_tg(gkind)) {  // the instantiations of the mixed-precision CG sweeps
        const int c = B.dot_mode == DOT_CGR ? 9 : B.dot_mode == DOT_XUPD ? 10 + B.epi : B.epi * 3 + B.dot_mode;
        if (!(c == 0 || c == 3 || c == 6 || c == 8 || c == 9 || c == 10 || c == 11))
            return fail(ctx, C2Q_BAD_ARG, "no temporal-gauge sweep with this epilogue and reduction");
    }
    int rc = gauge_ensure(const_cast<c2q_gauge*>(g), gkind);
    if (rc) return rc;
    return P == 32 ? pk_launch<32>(ctx, g, gkind, B) : pk_launch<16>(ctx, g, gkind, B);
}

// Fermion matrices on a batch of reduced-precision right-hand sides (the
// batched form of apply_operator in fields.cu): every sweep is one launch
// over all right-hand sides.
static int aee_sweeps_batch(c2q_ctx* ctx, int n, c2q_spinor_eo* const* out, const c2q_gauge* g, int gkind,
                            const c2q_spinor_eo* const* in, double kappa, double mubar, int action, int minus, int g5,
                            c2q_spinor_eo* const* tmp, int dot_mode, const c2q_spinor_eo* const* y, int fin,
                            SolverScalars* const* sc, const c2q_spinor_eo* const* xu_p = nullptr,
                            c2q_spinor_eo* const* xu_x = nullptr)
{
    const bool tm = action == C2Q_ACTION_TWISTEDMASS;
    PkBatch B;
    B.n          = n;
    B.kappa      = kappa;
    B.out_parity = 0;  // ODD: the even sites
    B.epi        = tm ? EPI_DIAG : EPI_PLAIN;
    B.e          = tm ? diag_epi(mubar, minus ? C2Q_DIAG_M_TM_INVERSE_MINUS : C2Q_DIAG_M_TM_INVERSE, 0)
                      : EpiArgs{1, 0, 1, 0, 0};
    B.dot_mode   = xu_x ? DOT_XUPD : DOT_NONE;  // the CG solution update xu_x += alpha xu_p rides along
    for (int r = 0; r < n; ++r) {
        B.out[r] = tmp[r];
        B.in[r]  = in[r];
        if (xu_x) {
            B.x[r]  = xu_p[r];
            B.y[r]  = xu_x[r];
            B.sc[r] = sc[r];
        }
    }
    int rc = launch_pdslash(ctx, g, gkind, B);
    if (rc) return rc;
    PkBatch C;
    C.n          = n;
    C.kappa      = kappa;
    C.out_parity = 1;  // EVEN: the odd sites
    C.epi        = EPI_AXPY;
    C.e          = tm ? diag_epi(mubar, minus ? C2Q_DIAG_M_TM_MINUS : C2Q_DIAG_M_TM, g5) : EpiArgs{1, 0, 1, 0, g5};
    C.dot_mode   = dot_mode;
    C.fin        = fin;
    for (int r = 0; r < n; ++r) {
        C.out[r] = out[r];
        C.in[r]  = tmp[r];
        C.x[r]   = in[r];
        C.y[r]   = y ? y[r] : nullptr;
        C.sc[r]  = sc ? sc[r] : nullptr;
    }
    return launch_pdslash(ctx, g, gkind, C);
}

int apply_operator_batch(c2q_ctx* ctx, int op, int n, c2q_spinor_eo* const* out, const c2q_gauge* g, int gkind,
                         const c2q_spinor_eo* const* in, double kappa, double mubar, int action,
                         c2q_spinor_eo* const* tmp1, c2q_spinor_eo* const* tmp2, int dot_mode,
                         const c2q_spinor_eo* const* y, int fin, SolverScalars* const* sc, int* sweeps,
                         c2q_spinor_eo* const* r_update, c2q_spinor_eo* const* x_update)
{
    if (action != C2Q_ACTION_WILSON && action != C2Q_ACTION_TWISTEDMASS)
        return fail(ctx, C2Q_BAD_ARG, "unknown fermion action (wilson or twistedmass)");
    int rc = 0;
    switch (op) {
        case C2Q_OP_AEE:
            rc = aee_sweeps_batch(ctx, n, out, g, gkind, in, kappa, mubar, action, 0, 0, tmp1, dot_mode, y, fin, sc);
            break;
        case C2Q_OP_AEE_MINUS:
            rc = aee_sweeps_batch(ctx, n, out, g, gkind, in, kappa, mubar, action, 1, 0, tmp1, dot_mode, y, fin, sc);
            break;
        case C2Q_OP_QPLUS_EO:
        case C2Q_OP_AEE_AND_GAMMA5_EO:
            rc = aee_sweeps_batch(ctx, n, out, g, gkind, in, kappa, mubar, action, 0, 1, tmp1, dot_mode, y, fin, sc);
            break;
        case C2Q_OP_QMINUS_EO:
        case C2Q_OP_AEE_MINUS_AND_GAMMA5_EO:
            rc = aee_sweeps_batch(ctx, n, out, g, gkind, in, kappa, mubar, action, 1, 1, tmp1, dot_mode, y, fin, sc);
            break;
        case C2Q_OP_QPLUSQMINUS_EO: {
            const c2q_spinor_eo* mid[PK_MAX_RHS];
            bool self = dot_mode == DOT_Y;
            for (int r = 0; r < n && self; ++r) self = y && y[r] == in[r];
            for (int r = 0; r < n; ++r) mid[r] = tmp2[r];
            // <in, Q+ Q- in> = |Q- in|^2 (Qplus_eo is the adjoint of Qminus_eo):
            // reduced from the intermediate in registers, with no operand read
            rc = aee_sweeps_batch(ctx, n, tmp2, g, gkind, in, kappa, mubar, action, 1, 1, tmp1,
                                  self ? DOT_SELF : DOT_NONE, nullptr, fin, sc);
            if (!rc && self && r_update) {
                // alpha is known after the second sweep: the last sweep applies r -= alpha A in
                // and reduces |r|^2 (FIN_CG_BETA) instead of storing A in, and with x_update
                // the third sweep applies x += alpha in
                const c2q_spinor_eo* rr[PK_MAX_RHS];
                for (int r = 0; r < n; ++r) rr[r] = r_update[r];
                rc = aee_sweeps_batch(ctx, n, out, g, gkind, mid, kappa, mubar, action, 0, 1, tmp1, DOT_CGR, rr,
                                      FIN_CG_BETA, sc, x_update ? in : nullptr, x_update);
            } else if (!rc) {
                rc = aee_sweeps_batch(ctx, n, out, g, gkind, mid, kappa, mubar, action, 0, 1, tmp1,
                                      self ? DOT_NONE : dot_mode, y, fin, sc);
            }
            if (sweeps) *sweeps += 2;
            break;
        }
        default: return fail(ctx, C2Q_BAD_ARG, "unknown eo fermion matrix");
    }
    if (sweeps) *sweeps += 2;
    return rc;
}

}  // namespace c2q

using namespace c2q;

extern "C" {

C2Q_EXPORT int c2q_ctx_set_autotune(c2q_ctx* ctx, int enable)
{
    if (!ctx) return C2Q_BAD_ARG;
    ctx->autotune = enable != 0;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_ctx_set_sweep_choice(c2q_ctx* ctx, int choice)
{
    if (!ctx || choice < -1 || choice > PK_CHOICE_RB2) return C2Q_BAD_ARG;
    ctx->force_choice = choice;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_ctx_tune_report(const c2q_ctx* ctx, char* buf, int len)
{
    if (!ctx) return C2Q_BAD_ARG;
    std::string out;
    char line[256];
    for (const auto& kv : ctx->tune) {
        const std::vector<int>& k = kv.first;
        snprintf(line, sizeof line,
                 "prec=%d links=%d epi=%d dot=%d phases=%d nrhs=%d sites=%d choice=%d (%s) "
                 "us=[%.1f, %.1f, %.1f, %.1f, %.1f]\n",
                 k[0], k[1] == 6 ? 12 : 18, k[2], k[3], k[4], k[5], k[6], kv.second.cfg,
                 kv.second.cfg == PK_CHOICE_RB2 ? "two right-hand sides per thread"
                 : (kv.second.cfg >> 1)         ? ((kv.second.cfg & 1) ? "config 1, grid-stride grid"
                                                                       : "config 0, grid-stride grid")
                                                : ((kv.second.cfg & 1) ? "config 1, per-tile grid"
                                                                       : "config 0, per-tile grid"),
                 kv.second.us[0], kv.second.us[1], kv.second.us[2], kv.second.us[3], kv.second.us[4]);
        out += line;
    }
    if (buf && len > 0) {
        const size_t n = out.size() < (size_t)len - 1 ? out.size() : (size_t)len - 1;
        memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return (int)out.size() + 1;
}

}  // extern "C"
