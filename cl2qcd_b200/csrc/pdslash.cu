// pdslash.cu -- host side of the paired-site dslash (pdslash.cuh): launches
// for one right-hand side (the FP32 / FP16 branch of launch_dslash) and for
// batches of right-hand sides sharing one gauge field.
#include "c2q_host.h"
#include "pdslash.cuh"

namespace c2q {

void pk_dispatch32(const PkParams<32>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s);
void pk_dispatch16(const PkParams<16>& prm, int epi, int dot, int blocks, cudaStream_t s);

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
    prm.gauge      = g->store[gkind].data;
    prm.g          = pk_geom(ref->geom);
    prm.c          = hop_coef(ref->lat, B.kappa);
    // FP16: links in units of 1/32767 and neighbour spinors in units of norm/32767
    if (P == 16) prm.c.scale *= 1.0 / (32767.0 * 32767.0);
    prm.e          = B.e;
    prm.out_parity = B.out_parity;
    const int nblk   = (prm.g.H + PK_THREADS - 1) / PK_THREADS;
    const int blocks = nblk * B.n;
    if (B.dot_mode) {
        int rc = ensure_partials(ctx, blocks);
        if (rc) return rc;
    }
    prm.red.partials = ctx->partials;
    prm.red.ticket   = ctx->ticket;
    prm.red.result   = ctx->red_result;
    prm.red.sc       = ctx->scalars;
    prm.red.fin      = B.fin;
    const bool r12   = gkind == G32R12 || gkind == G16R12;
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
        tm.bytes = (double)ref->geom.seo *
                   (8.0 * lk + B.n * sp * (2.0 + (B.epi == EPI_AXPY ? 1.0 : 0.0) + (B.dot_mode == DOT_Y ? 1.0 : 0.0)));
        cudaEventRecord(tm.a, ctx->stream);
    }
    if constexpr (P == 16)
        pk_dispatch16(prm, B.epi, B.dot_mode, blocks, ctx->stream);
    else
        pk_dispatch32(prm, r12 ? 6 : 9, B.epi, B.dot_mode, blocks, ctx->stream);
    if (ctx->profiling) {
        cudaEventRecord(tm.b, ctx->stream);
        ctx->timed.push_back(tm);
    }
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

int launch_pdslash(c2q_ctx* ctx, const c2q_gauge* g, int gkind, const PkBatch& B)
{
    if (B.n < 1 || B.n > PK_MAX_RHS) return fail(ctx, C2Q_BAD_ARG, "batch size must be 1..16");
    const c2q_spinor_eo* ref = B.out[0];
    const int P              = ref->prec;
    for (int r = 0; r < B.n; ++r) {
        for (const c2q_spinor_eo* f : {(const c2q_spinor_eo*)B.out[r], B.in[r], B.x[r], B.y[r]}) {
            if (!f) continue;
            if (f->prec != P || !same_lattice(f->lat, ref->lat))
                return fail(ctx, C2Q_BAD_ARG, "fields of a batch differ in precision or lattice");
        }
        if (!B.in[r] || B.out[r] == B.in[r]) return fail(ctx, C2Q_BAD_ARG, "dslash output must not alias its input");
        if (B.epi == EPI_AXPY && !B.x[r]) return fail(ctx, C2Q_BAD_ARG, "missing axpy operand");
        if (B.dot_mode == DOT_Y && !B.y[r]) return fail(ctx, C2Q_BAD_ARG, "missing dot partner");
    }
    int rc = gauge_ensure(const_cast<c2q_gauge*>(g), gkind);
    if (rc) return rc;
    return P == 32 ? pk_launch<32>(ctx, g, gkind, B) : pk_launch<16>(ctx, g, gkind, B);
}

}  // namespace c2q
