// tgauge.cu -- the temporal gauge of the reduced-precision inner solves.
//
// With c the forward T hop weight (a pure phase: the boundary condition in
// time, times an imaginary chemical potential) the site transformation
//     G(x, 0) = 1,   G(x, t + 1) = G(x, t) c U_T(x, t)
// turns every weighted T link c G(x, t) U_T(x, t) G(x, t + 1)^dagger into the
// identity, except the one leaving the last slice:
//     c G(x, NT - 1) U_T(x, NT - 1) G(x, 0)^dagger = lambda W(x),
//     lambda = c^NT,  W(x) = G_3(x, NT - 1) U_T(x, NT - 1) in SU(3)
// (G = c^t G_3).  Spatial links become G(x) U_mu(x) G(x + mu)^dagger, in SU(3)
// since both ends share t.  The operator on the transformed field is
// G M G^dagger (G acts on colour only, so it commutes with the spin structure,
// the twisted-mass factors and gamma5): the mixed-precision CG runs its inner
// iterations on it, with the residual taken in as G r and the solution
// increment taken out as G^dagger x_s.  The true FP64 residuals and the
// solution stay on the original field.
//
// The transformation is stored per site in FP64 as [parity][9 lanes][stride]
// (the gauge store layout without the direction).
#include <cmath>

#include "c2q_host.h"

namespace c2q {

namespace {

using C = Cplx<double>;

__device__ __forceinline__ void load9(const double2* base, int stride, int i, C m[9])
{
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const double2 v = base[(size_t)k * stride + i];
        m[k]            = cmk(v.x, v.y);
    }
}
__device__ __forceinline__ void store9(double2* base, int stride, int i, const C m[9])
{
#pragma unroll
    for (int k = 0; k < 9; ++k) base[(size_t)k * stride + i] = make_double2(m[k].re, m[k].im);
}
// c = a b
__device__ __forceinline__ void mm(const C a[9], const C b[9], C c[9])
{
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            C s = cmk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 3; ++k) cmac(s, a[3 * r + k], b[3 * k + q]);
            c[3 * r + q] = s;
        }
}
// c = a b^dagger
__device__ __forceinline__ void mmd(const C a[9], const C b[9], C c[9])
{
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            C s = cmk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 3; ++k) cmacc(s, b[3 * q + k], a[3 * r + k]);
            c[3 * r + q] = s;
        }
}

// site coordinates of eo index i on parity par (site = x + NS y + NS^2 z + NS^3 t)
__device__ __forceinline__ void eo_coords(int i, int par, int ns, int* x, int* y, int* z, int* t)
{
    const int s0 = 2 * i;
    int r        = s0 / ns;
    const int x0 = s0 - r * ns;
    *y           = r % ns;
    r /= ns;
    *z = r % ns;
    *t = r / ns;
    *x = x0 + (((*y + *z + *t) & 1) != par);
}

// one thread per spatial site walks up the time direction
__global__ void tg_transform_kernel(const double2* __restrict__ U, double2* __restrict__ Gt, Geom g, double cre,
                                    double cim)
{
    const int vs = g.ns * g.ns * g.ns;
    const int s3 = blockIdx.x * blockDim.x + threadIdx.x;
    if (s3 >= vs) return;
    const int x = s3 % g.ns, y = (s3 / g.ns) % g.ns, z = s3 / (g.ns * g.ns);
    C G[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) G[k] = cmk(k % 4 == 0 ? 1.0 : 0.0, 0.0);
    const C c = cmk(cre, cim);
    for (int t = 0; t < g.nt; ++t) {
        const int site = s3 + vs * t;
        const int par  = (x + y + z + t) & 1, i = site >> 1;
        store9(Gt + (size_t)par * 9 * g.stride, g.stride, i, G);
        if (t + 1 < g.nt) {
            C u[9], n[9];
            load9(U + (size_t)(par * 4) * 9 * g.stride, g.stride, i, u);  // U_T(x, t)
#pragma unroll
            for (int k = 0; k < 9; ++k) u[k] = cmul(c, u[k]);
            mm(G, u, n);
#pragma unroll
            for (int k = 0; k < 9; ++k) G[k] = n[k];
        }
    }
}

// the transformed links in the FP64 9-lane store layout; w = c / lambda
__global__ void tg_links_kernel(const double2* __restrict__ U, const double2* __restrict__ Gt, double2* __restrict__ out,
                                Geom g, double wre, double wim)
{
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 8LL * g.seo) return;
    const int blk = (int)(tid / g.seo), i = (int)(tid - (long long)blk * g.seo);
    const int par = blk >> 2, mu = blk & 3;
    int x, y, z, t;
    eo_coords(i, par, g.ns, &x, &y, &z, &t);
    C r[9];
    if (mu == 0 && t + 1 < g.nt) {
#pragma unroll
        for (int k = 0; k < 9; ++k) r[k] = cmk(k % 4 == 0 ? 1.0 : 0.0, 0.0);
    } else {
        C G[9], u[9], a[9];
        load9(Gt + (size_t)par * 9 * g.stride, g.stride, i, G);
        load9(U + (size_t)(par * 4 + mu) * 9 * g.stride, g.stride, i, u);
        mm(G, u, a);
        if (mu == 0) {  // W = G(x, NT - 1) c U_T(x, NT - 1) / lambda (G(x, 0) = 1)
            const C w = cmk(wre, wim);
#pragma unroll
            for (int k = 0; k < 9; ++k) r[k] = cmul(w, a[k]);
        } else {
            const int xn = mu == 1 ? (x + 1) % g.ns : x, yn = mu == 2 ? (y + 1) % g.ns : y,
                      zn = mu == 3 ? (z + 1) % g.ns : z;
            const int sn = xn + g.ns * (yn + g.ns * (zn + g.ns * t));
            C Gn[9];
            load9(Gt + (size_t)(1 - par) * 9 * g.stride, g.stride, sn >> 1, Gn);
            mmd(a, Gn, r);
        }
    }
    store9(out + (size_t)(par * 4 + mu) * 9 * g.stride, g.stride, i, r);
}

// out = G in on the parity-1 sites (the CG vectors), FP64 arithmetic
template <int PO>
__global__ void __launch_bounds__(BLAS_THREADS) tg_to_inner_kernel(SpinorPtr<PO> out, SpinorPtr<64> in,
                                                                   const double2* __restrict__ G1, int n, int stride)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    C G[9], v[12];
    load9(G1, stride, i, G);
    SpinorIO<64>::load(in, stride, i, v);
    Cplx<typename Prec<PO>::R> o[12];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            C acc = cmk(0.0, 0.0);
#pragma unroll
            for (int b = 0; b < 3; ++b) cmac(acc, G[3 * a + b], v[3 * s + b]);
            o[3 * s + a] = {(typename Prec<PO>::R)acc.re, (typename Prec<PO>::R)acc.im};
        }
    SpinorIO<PO>::store(out, stride, i, o);
}

// x += G^dagger (xs + alpha p) on the parity-1 sites, xs = 0
template <int PB>
__global__ void __launch_bounds__(BLAS_THREADS) tg_accumulate_kernel(SpinorPtr<64> x, SpinorPtr<32> xs,
                                                                     SpinorPtr<PB> p, const SolverScalars* sc,
                                                                     const double2* __restrict__ G1, int n, int stride)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Cplx<float> b[12];
    SpinorIO<32>::load(xs, stride, i, b);
    if (sc) {
        Cplx<float> q[12];
        SpinorIO<PB>::load(p, stride, i, q);
        const Cplx<float> al = cmk<float>((float)sc->alpha[0], (float)sc->alpha[1]);
#pragma unroll
        for (int k = 0; k < 12; ++k) b[k] = b[k] + cmul(al, q[k]);
    }
    C G[9], a[12];
    load9(G1, stride, i, G);
    SpinorIO<64>::load(x, stride, i, a);
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r)  // (G^dagger)_{c r} = conj(G_{r c})
                cmacc(a[3 * s + c], G[3 * r + c], cmk((double)b[3 * s + r].re, (double)b[3 * s + r].im));
    SpinorIO<64>::store(x, stride, i, a);
#pragma unroll
    for (int k = 0; k < 12; ++k) b[k] = cmk<float>(0.f, 0.f);
    SpinorIO<32>::store(xs, stride, i, b);
}

}  // namespace

bool tg_applicable(const c2q_lattice& lat)
{
    if (lat.nt % 4 || lat.nt < 4) return false;
    const HopCoef c = hop_coef(lat, 1.0);
    for (int mu = 1; mu < 4; ++mu)
        if (c.im[mu][0] != 0.0 || c.im[mu][1] != 0.0) return false;
    // the T weights must be a pure phase and its conjugate
    const double fr = c.re[0][0], fi = c.im[0][0];
    if (c.re[0][1] != fr || c.im[0][1] != -fi) return false;
    return std::fabs(fr * fr + fi * fi - 1.0) < 1e-12;
}

int tg_ensure(c2q_gauge* g)
{
    c2q_ctx* ctx = g->ctx;
    if (g->tg_transform.data) return C2Q_OK;
    if (!g->store[G64].data) return fail(ctx, C2Q_BAD_ARG, "gauge field not uploaded");
    if (!tg_applicable(g->lat)) return fail(ctx, C2Q_BAD_ARG, "the temporal gauge needs pure-phase T weights");
    const HopCoef c    = hop_coef(g->lat, 1.0);
    const double cre   = c.re[0][0], cim = c.im[0][0];
    double lre = 1.0, lim = 0.0;  // lambda = c^NT
    for (int t = 0; t < g->lat.nt; ++t) {
        const double r = lre * cre - lim * cim, q = lre * cim + lim * cre;
        lre            = r;
        lim            = q;
    }
    const size_t bytes = (size_t)2 * 9 * g->geom.stride * sizeof(double2);
    void* p            = nullptr;
    C2Q_CUDA(ctx, cudaMalloc(&p, bytes));
    C2Q_CUDA(ctx, cudaMemsetAsync(p, 0, bytes, ctx->stream));
    const int vs = g->lat.ns * g->lat.ns * g->lat.ns;
    tg_transform_kernel<<<(vs + 127) / 128, 128, 0, ctx->stream>>>(static_cast<const double2*>(g->store[G64].data),
                                                                  static_cast<double2*>(p), g->geom, cre, cim);
    ctx->launches++;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFree(p);
        return cuda_fail(ctx, e, "tg_transform_kernel");
    }
    g->tg_transform.data  = p;
    g->tg_transform.bytes = bytes;
    g->tg_lam_re          = lre;
    g->tg_lam_im          = lim;
    return C2Q_OK;
}

int tg_links_fp64(c2q_gauge* g, void* out)
{
    c2q_ctx* ctx = g->ctx;
    int rc       = tg_ensure(g);
    if (rc) return rc;
    const HopCoef c = hop_coef(g->lat, 1.0);
    // w = c / lambda (|lambda| = 1)
    const double cre = c.re[0][0], cim = c.im[0][0], lre = g->tg_lam_re, lim = g->tg_lam_im;
    const double n2  = lre * lre + lim * lim;
    const double wre = (cre * lre + cim * lim) / n2, wim = (cim * lre - cre * lim) / n2;
    const long long n = 8LL * g->geom.seo;
    tg_links_kernel<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(
        static_cast<const double2*>(g->store[G64].data), static_cast<const double2*>(g->tg_transform.data),
        static_cast<double2*>(out), g->geom, wre, wim);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

int tg_to_inner(c2q_ctx* ctx, const c2q_gauge* g, c2q_spinor_eo* out, const c2q_spinor_eo* in)
{
    if (!g->tg_transform.data || out->prec != 32 || in->prec != 64)
        return fail(ctx, C2Q_BAD_ARG, "tg_to_inner: FP64 in, FP32 out, transformation built");
    const int n          = in->geom.seo;
    const double2* G1    = static_cast<const double2*>(g->tg_transform.data) + (size_t)9 * g->geom.stride;
    tg_to_inner_kernel<32><<<(n + BLAS_THREADS - 1) / BLAS_THREADS, BLAS_THREADS, 0, ctx->stream>>>(
        sptr<32>(out), sptr<64>(in), G1, n, in->geom.stride);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

int tg_accumulate(c2q_ctx* ctx, const c2q_gauge* g, c2q_spinor_eo* x, c2q_spinor_eo* xs, const c2q_spinor_eo* p,
                  const SolverScalars* sc)
{
    if (!g->tg_transform.data) return fail(ctx, C2Q_BAD_ARG, "tg_accumulate: transformation not built");
    const int n       = x->geom.seo;
    const double2* G1 = static_cast<const double2*>(g->tg_transform.data) + (size_t)9 * g->geom.stride;
    const unsigned blocks = (unsigned)((n + BLAS_THREADS - 1) / BLAS_THREADS);
    if (p->prec == 16)
        tg_accumulate_kernel<16><<<blocks, BLAS_THREADS, 0, ctx->stream>>>(sptr<64>(x), sptr<32>(xs), sptr<16>(p),
                                                                          sc, G1, n, x->geom.stride);
    else
        tg_accumulate_kernel<32><<<blocks, BLAS_THREADS, 0, ctx->stream>>>(sptr<64>(x), sptr<32>(xs), sptr<32>(p),
                                                                          sc, G1, n, x->geom.stride);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

}  // namespace c2q
