// force.cu -- the eo fermion force of the HMC and the gauge momenta it
// accumulates into: physics::algorithms::fermion_force(gm, Y, X, evenodd, gf,
// params) on eo fields (physics/algorithms/fermion_force.cpp:699-730), i.e. the
// kernels fermion_force_eo_0..3 of ocl_kernel/force_fermion_eo.cl driven by
// hardware/code/molecular_dynamics.cpp:543-625, as one FP64 sweep.
//
// At every site x of the parity evenodd selects (ODD: x+y+z+t even) with
// y = g5 Y(x), for each direction mu:
//   forward : phi = (1 - g_mu) y, psi = (1 - g_mu) X(x + mu), each reduced to
//             its upper rows a, b (the projector table of the dslash);
//             v = phi_a psi_a^+ + phi_b psi_b^+ and
//             F(x, mu) += tr_lambda(bc_mu U_mu(x) v^+);
//   backward: with (1 + g_mu) and X(x - mu), v = psi_a phi_a^+ + psi_b phi_b^+
//             and F(x - mu, mu) += tr_lambda(bc_mu U_mu(x - mu) v^+);
// bc_mu = 2 kappa e^{i theta pi / N} for both hops, T links multiplied by
// e^{cp_re} e^{i cp_im} (forward) or e^{-cp_re} e^{i cp_im} (backward), and
// tr_lambda(M)_k = Tr[i T_k (M - M^+)] (T_k = lambda_k / 2, the generator
// basis of ocl_kernel/operations_gaugemomentum.cl:68-88).  A thread owns the
// forward links of its site and the backward links ending there: for one
// parity every link has exactly one writer, so the sweep needs no atomics.
//
// Gauge momenta on the device: 8 reals per link as [parity][mu][8 lanes][stride]
// at the eo index of the link's site; on the host the reference's ae[4V] at
// link mu + 4 site.
#include <cmath>
#include <cstring>

#include "c2q_host.h"
#include "dslash.cuh"

struct c2q_gaugemomenta {
    c2q_ctx* ctx = nullptr;
    c2q_lattice lat{};
    c2q::Geom geom{};
    double* data = nullptr;
    size_t bytes = 0;
};

namespace c2q {

int read_scalars(c2q_ctx* ctx, const double* dev, int n, double* host);

namespace {

using C = Cplx<double>;

struct ForceCoef {
    double bre[4], bim[4];      // 2 kappa e^{i theta pi / N} per direction
    double cpf[2], cpb[2];      // T link factors, forward and backward hop
};

__device__ __forceinline__ size_t gm_at(const Geom& g, int par, int mu, int k, int i)
{
    return ((size_t)((par * 4 + mu) * 8 + k)) * g.stride + i;
}

// site coordinates of eo index i on parity par
__device__ __forceinline__ void coords(const Geom& g, int i, int par, int c[4])
{
    const int s0 = 2 * i;
    int r        = s0 / g.ns;
    const int x0 = s0 - r * g.ns;
    c[2]         = r % g.ns;
    r /= g.ns;
    c[3] = r % g.ns;
    c[0] = r / g.ns;
    c[1] = x0 + (((c[2] + c[3] + c[0]) & 1) != par);
}
__device__ __forceinline__ int site_of(const Geom& g, const int c[4])
{
    return c[1] + g.ns * (c[2] + g.ns * (c[3] + g.ns * c[0]));
}

// h = psi_a + c psi_p for the unit codes of the dslash (0: 1, 1: -1, 2: i, 3: -i)
__device__ __forceinline__ C unit_mul(int code, C v)
{
    return code == 0 ? v : code == 1 ? cmk(-v.re, -v.im) : code == 2 ? cmk(-v.im, v.re) : cmk(v.im, -v.re);
}

template <int MU, bool BACK>
__device__ __forceinline__ void force_hop(const double2* __restrict__ U, const SpinorPtr<64>& X, double* __restrict__ gm,
                                          const Geom& g, const ForceCoef& fc, int par, const int c[4], const C y[12])
{
    using T        = Proj<MU>;
    const int u0   = BACK ? NegUnit<T::c0>::value : T::c0;
    const int u1   = BACK ? NegUnit<T::c1>::value : T::c1;
    int n[4]       = {c[0], c[1], c[2], c[3]};
    const int ext  = MU == 0 ? g.nt : g.ns;
    n[MU]          = BACK ? (c[MU] + ext - 1) % ext : (c[MU] + 1) % ext;
    const int in   = site_of(g, n) >> 1;  // eo index of the neighbour (other parity)
    const int lpar = BACK ? 1 - par : par, li = BACK ? in : site_of(g, c) >> 1;
    C plus[12];
    SpinorIO<64>::load(X, g.stride, in, plus);
    C psi[2][3], phi[2][3];
#pragma unroll
    for (int col = 0; col < 3; ++col) {
        psi[0][col] = plus[col] + unit_mul(u0, plus[3 * T::p0 + col]);
        psi[1][col] = plus[3 + col] + unit_mul(u1, plus[3 * T::p1 + col]);
        phi[0][col] = y[col] + unit_mul(u0, y[3 * T::p0 + col]);
        phi[1][col] = y[3 + col] + unit_mul(u1, y[3 * T::p1 + col]);
    }
    // v = phi psi^+ (forward) or psi phi^+ (backward), summed over the two rows
    C v[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            C s = cmk(0.0, 0.0);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (BACK)
                    cmacc(s, phi[a][q], psi[a][r]);
                else
                    cmacc(s, psi[a][q], phi[a][r]);
            }
            v[3 * r + q] = s;
        }
    // w = bc U v^+ with the T link's chemical-potential factor
    const double2* ul = U + (size_t)((lpar * 4 + MU) * 9) * g.stride + li;
    C u[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const double2 t = ul[(size_t)e * g.stride];
        u[e]            = cmk(t.x, t.y);
        if (MU == 0) u[e] = cmul(u[e], BACK ? cmk(fc.cpb[0], fc.cpb[1]) : cmk(fc.cpf[0], fc.cpf[1]));
    }
    const C bc = cmk(fc.bre[MU], fc.bim[MU]);
    C w[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            C s = cmk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 3; ++k) cmacc(s, v[3 * q + k], u[3 * r + k]);  // U_rk conj(v_qk)
            w[3 * r + q] = cmul(s, bc);
        }
    double ae[8];
    ae[0] = -w[3].im - w[1].im;
    ae[1] = w[3].re - w[1].re;
    ae[2] = -w[0].im + w[4].im;
    ae[3] = -w[6].im - w[2].im;
    ae[4] = w[6].re - w[2].re;
    ae[5] = -w[7].im - w[5].im;
    ae[6] = w[7].re - w[5].re;
    ae[7] = (-w[0].im - w[4].im + 2.0 * w[8].im) * 0.577350269189625;
#pragma unroll
    for (int k = 0; k < 8; ++k) gm[gm_at(g, lpar, MU, k, li)] += ae[k];
}

__global__ void __launch_bounds__(128) fermion_force_eo_kernel(const double2* __restrict__ U, SpinorPtr<64> Y,
                                                               SpinorPtr<64> X, double* __restrict__ gm, Geom g,
                                                               ForceCoef fc, int par)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.seo) return;
    int c[4];
    coords(g, i, par, c);
    C y[12];
    SpinorIO<64>::load(Y, g.stride, i, y);
#pragma unroll
    for (int k = 6; k < 12; ++k) y[k] = cmk(-y[k].re, -y[k].im);  // g5
    force_hop<0, false>(U, X, gm, g, fc, par, c, y);
    force_hop<0, true>(U, X, gm, g, fc, par, c, y);
    force_hop<1, false>(U, X, gm, g, fc, par, c, y);
    force_hop<1, true>(U, X, gm, g, fc, par, c, y);
    force_hop<2, false>(U, X, gm, g, fc, par, c, y);
    force_hop<2, true>(U, X, gm, g, fc, par, c, y);
    force_hop<3, false>(U, X, gm, g, fc, par, c, y);
    force_hop<3, true>(U, X, gm, g, fc, par, c, y);
}

// host ae[4V] (link mu + 4 site) <-> device lanes
__global__ void gm_import_kernel(const double* __restrict__ aos, double* __restrict__ out, Geom g, int vol)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4LL * vol) return;
    const int s = (int)(t >> 2), mu = (int)(t & 3);
    int c[4];
    c[1] = s % g.ns;
    c[2] = (s / g.ns) % g.ns;
    c[3] = (s / (g.ns * g.ns)) % g.ns;
    c[0] = s / (g.ns * g.ns * g.ns);
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
#pragma unroll
    for (int k = 0; k < 8; ++k) out[gm_at(g, par, mu, k, s >> 1)] = aos[8 * t + k];
}
__global__ void gm_export_kernel(double* __restrict__ aos, const double* __restrict__ in, Geom g, int vol)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4LL * vol) return;
    const int s = (int)(t >> 2), mu = (int)(t & 3);
    int c[4];
    c[1] = s % g.ns;
    c[2] = (s / g.ns) % g.ns;
    c[3] = (s / (g.ns * g.ns)) % g.ns;
    c[0] = s / (g.ns * g.ns * g.ns);
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
#pragma unroll
    for (int k = 0; k < 8; ++k) aos[8 * t + k] = in[gm_at(g, par, mu, k, s >> 1)];
}

// sum of e_k^2 over every link (deterministic two-stage reduction)
__global__ void __launch_bounds__(256) gm_squarenorm_kernel(const double* __restrict__ gm, Geom g, RedArgs ra)
{
    __shared__ double smem[2 * 32];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dv[2]      = {0.0, 0.0};
    if (t < 8LL * g.seo) {
        const int blk = (int)(t / g.seo), i = (int)(t - (long long)blk * g.seo);  // blk = parity * 4 + mu
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double e = gm[((size_t)(blk * 8 + k)) * g.stride + i];
            dv[0]          = fma(e, e, dv[0]);
        }
    }
    block_sum<2>(dv, smem);
    finish_reduction<2>(dv, ra, smem);
}

}  // namespace
}  // namespace c2q

using namespace c2q;

extern "C" {

C2Q_EXPORT int c2q_gaugemomenta_create(c2q_ctx* ctx, const c2q_lattice* lat, c2q_gaugemomenta** out)
{
    if (!ctx || !lat || !out) return C2Q_BAD_ARG;
    *out = nullptr;
    Geom g;
    if (!make_geom(*lat, &g)) return fail(ctx, C2Q_BAD_ARG, "lattice extents must be even and positive");
    auto* m  = new c2q_gaugemomenta;
    m->ctx   = ctx;
    m->lat   = *lat;
    m->geom  = g;
    m->bytes = (size_t)2 * 4 * 8 * g.stride * sizeof(double);
    if (cudaMalloc(&m->data, m->bytes) != cudaSuccess) {
        delete m;
        return fail(ctx, C2Q_OOM, "gauge momenta: out of device memory");
    }
    const cudaError_t e = cudaMemsetAsync(m->data, 0, m->bytes, ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(m->data);
        delete m;
        return cuda_fail(ctx, e, "cudaMemsetAsync(gauge momenta)");
    }
    *out = m;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_gaugemomenta_destroy(c2q_gaugemomenta* m)
{
    if (!m) return C2Q_OK;
    cudaStreamSynchronize(m->ctx->stream);
    cudaFree(m->data);
    delete m;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_gaugemomenta_zero(c2q_gaugemomenta* m)
{
    if (!m) return C2Q_BAD_ARG;
    C2Q_CUDA(m->ctx, cudaMemsetAsync(m->data, 0, m->bytes, m->ctx->stream));
    return C2Q_OK;
}

C2Q_EXPORT int c2q_gaugemomenta_upload(c2q_gaugemomenta* m, const double* aos)
{
    if (!m || !aos) return C2Q_BAD_ARG;
    c2q_ctx* ctx       = m->ctx;
    const int vol      = 2 * m->geom.seo;
    const size_t bytes = (size_t)4 * vol * 8 * sizeof(double);
    int rc             = ensure_staging(ctx, bytes);
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaMemcpyAsync(ctx->staging, aos, bytes, cudaMemcpyHostToDevice, ctx->stream));
    const long long n = 4LL * vol;
    gm_import_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>((const double*)ctx->staging, m->data,
                                                                         m->geom, vol);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

C2Q_EXPORT int c2q_gaugemomenta_download(const c2q_gaugemomenta* m, double* aos)
{
    if (!m || !aos) return C2Q_BAD_ARG;
    c2q_ctx* ctx       = m->ctx;
    const int vol      = 2 * m->geom.seo;
    const size_t bytes = (size_t)4 * vol * 8 * sizeof(double);
    int rc             = ensure_staging(ctx, bytes);
    if (rc) return rc;
    const long long n = 4LL * vol;
    gm_export_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>((double*)ctx->staging, m->data, m->geom,
                                                                         vol);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    C2Q_CUDA(ctx, cudaMemcpyAsync(aos, ctx->staging, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

C2Q_EXPORT int c2q_gaugemomenta_squarenorm(const c2q_gaugemomenta* m, double* out)
{
    if (!m || !out) return C2Q_BAD_ARG;
    c2q_ctx* ctx      = m->ctx;
    const long long n = 8LL * m->geom.seo;
    const int blocks  = (int)((n + 255) / 256);
    int rc            = ensure_partials(ctx, (size_t)blocks);
    if (rc) return rc;
    RedArgs ra;
    memset(&ra, 0, sizeof ra);
    ra.partials = ctx->partials;
    ra.ticket   = ctx->ticket;
    ra.result   = ctx->red_result;
    ra.sc       = ctx->scalars;
    ra.fin      = FIN_STORE_RESULT;
    gm_squarenorm_kernel<<<blocks, 256, 0, ctx->stream>>>(m->data, m->geom, ra);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return read_scalars(ctx, ctx->red_result, 1, out);
}

C2Q_EXPORT int c2q_fermion_force_eo(c2q_gaugemomenta* m, const c2q_gauge* g, const c2q_spinor_eo* Y,
                                    const c2q_spinor_eo* X, int evenodd, double kappa)
{
    if (!m || !g || !Y || !X) return C2Q_BAD_ARG;
    c2q_ctx* ctx = m->ctx;
    if (Y->prec != 64 || X->prec != 64) return fail(ctx, C2Q_BAD_ARG, "the fermion force takes FP64 fields");
    if (!same_lattice(m->lat, g->lat) || !same_lattice(Y->lat, g->lat) || !same_lattice(X->lat, g->lat))
        return fail(ctx, C2Q_BAD_ARG, "lattice mismatch between momenta, gauge field and spinor fields");
    if (Y == X) return fail(ctx, C2Q_BAD_ARG, "Y and X live on different parities");
    if (evenodd != C2Q_ODD && evenodd != C2Q_EVEN) return fail(ctx, C2Q_BAD_ARG, "evenodd must be ODD or EVEN");
    if (!g->store[G64].data) return fail(ctx, C2Q_BAD_ARG, "gauge field not uploaded");
    ForceCoef fc;
    // the boundary phases e^{i theta pi / N} with the reference's rounding, without
    // the chemical potential (which multiplies the T link here)
    const c2q_lattice plain{g->lat.ns, g->lat.nt, g->lat.theta_t, g->lat.theta_s, 0, 0, 0.0, 0.0};
    const HopCoef p = hop_coef(plain, 1.0);
    for (int mu = 0; mu < 4; ++mu) {
        fc.bre[mu] = 2.0 * kappa * p.re[mu][0];
        fc.bim[mu] = 2.0 * kappa * p.im[mu][0];
    }
    // T link factors of the chemical potential: e^{cp_re} e^{i cp_im} forward,
    // e^{-cp_re} e^{i cp_im} backward (force_fermion_eo.cl:79-85, 128-135)
    const double er  = g->lat.use_cp_re ? as_build_option(std::exp(g->lat.cp_re)) : 1.0;
    const double emr = g->lat.use_cp_re ? as_build_option(std::exp(-g->lat.cp_re)) : 1.0;
    const double cc  = g->lat.use_cp_im ? as_build_option(std::cos(g->lat.cp_im)) : 1.0;
    const double ss  = g->lat.use_cp_im ? as_build_option(std::sin(g->lat.cp_im)) : 0.0;
    fc.cpf[0] = er * cc;
    fc.cpf[1] = er * ss;
    fc.cpb[0] = emr * cc;
    fc.cpb[1] = emr * ss;
    const int par = evenodd == C2Q_ODD ? 0 : 1;  // ODD: the sites with x+y+z+t even
    const int n   = m->geom.seo;
    fermion_force_eo_kernel<<<(n + 127) / 128, 128, 0, ctx->stream>>>(
        static_cast<const double2*>(g->store[G64].data), sptr<64>(Y), sptr<64>(X), m->data, m->geom, fc, par);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

}  // extern "C"
