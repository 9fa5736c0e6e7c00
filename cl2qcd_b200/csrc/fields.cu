// fields.cu -- context, gauge and spinor objects, layout conversion and the
// kernel launch wrappers (the part of the C ABI that is not a solver).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "blas.cuh"
#include "c2q_host.h"
#include "dslash.cuh"

namespace c2q {

int fail(c2q_ctx* ctx, int code, const std::string& msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(c2q_ctx* ctx, cudaError_t e, const char* where)
{
    const int code = (e == cudaErrorMemoryAllocation) ? C2Q_OOM : C2Q_CUDA_ERROR;
    return fail(ctx, code, std::string(where) + ": " + cudaGetErrorString(e));
}

bool make_geom(const c2q_lattice& lat, Geom* g)
{
    if (lat.ns < 2 || lat.nt < 2 || (lat.ns & 1) || (lat.nt & 1)) return false;
    const long long vol = (long long)lat.ns * lat.ns * lat.ns * lat.nt;
    if (vol / 2 > (1LL << 30)) return false;
    g->ns     = lat.ns;
    g->nt     = lat.nt;
    g->nsh    = lat.ns / 2;
    g->seo    = (int)(vol / 2);
    g->stride = round_up(g->seo, 64);
    g->vs_h   = lat.ns * lat.ns * lat.ns / 2;
    return true;
}

bool same_lattice(const c2q_lattice& a, const c2q_lattice& b)
{
    return a.ns == b.ns && a.nt == b.nt && a.theta_t == b.theta_t && a.theta_s == b.theta_s &&
           a.use_cp_re == b.use_cp_re && a.use_cp_im == b.use_cp_im && a.cp_re == b.cp_re && a.cp_im == b.cp_im;
}

// The reference passes its phases as text build options with 16 significant
// digits and PI = 3.14159265358979 (hardware/code/opencl_module.cpp:190-203,
// common_header_files/globaldefs.hpp); the same values are produced here.
double as_build_option(double v)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%.16g", v);
    return strtod(buf, nullptr);
}

HopCoef hop_coef(const c2q_lattice& lat, double kappa)
{
    const double PI_REF = 3.14159265358979;
    HopCoef c;
    for (int mu = 0; mu < 4; ++mu) {
        const double ang = mu == 0 ? (lat.theta_t * PI_REF) / (double)lat.nt : (lat.theta_s * PI_REF) / (double)lat.ns;
        const double re = as_build_option(std::cos(ang)), im = as_build_option(std::sin(ang));
        double fre = re, fim = im;   // forward  e^{+i phi}
        double bre = re, bim = -im;  // backward e^{-i phi}
        if (mu == 0 && (lat.use_cp_re || lat.use_cp_im)) {
            // chemical potential on T links (ocl_kernel/fermionmatrix_eo.cl:115-121, 222-228):
            // forward U e^{cp_re} e^{i cp_im}, backward (U e^{-cp_re} e^{i cp_im})^dagger
            const double er  = lat.use_cp_re ? as_build_option(std::exp(lat.cp_re)) : 1.0;
            const double emr = lat.use_cp_re ? as_build_option(std::exp(-lat.cp_re)) : 1.0;
            const double cc  = lat.use_cp_im ? as_build_option(std::cos(lat.cp_im)) : 1.0;
            const double ss  = lat.use_cp_im ? as_build_option(std::sin(lat.cp_im)) : 0.0;
            const double f_re = er * cc, f_im = er * ss, b_re = emr * cc, b_im = -emr * ss;
            double r = fre * f_re - fim * f_im, i = fre * f_im + fim * f_re;
            fre = r;
            fim = i;
            r   = bre * b_re - bim * b_im;
            i   = bre * b_im + bim * b_re;
            bre = r;
            bim = i;
        }
        // the phases carry no kappa: -kappa is applied once per site (HopCoef::scale)
        c.re[mu][0] = fre;
        c.im[mu][0] = fim;
        c.re[mu][1] = bre;
        c.im[mu][1] = bim;
    }
    c.scale     = -kappa;
    c.real_mask = 0;
    for (int mu = 0; mu < 4; ++mu)
        for (int d = 0; d < 2; ++d)
            if (c.im[mu][d] == 0.0) c.real_mask |= 1u << (2 * mu + d);
    return c;
}

// Site-diagonal factors (ocl_kernel/fermionmatrix_eo_m.cl:22-109, _m_merged.cl:22-64):
// spins 0,1 get f1, spins 2,3 get f2, the inverse carries 1/(1+mubar^2).
EpiArgs diag_epi(double mubar, int which, int gamma5)
{
    EpiArgs e{1, 0, 1, 0, gamma5};
    const double d = 1. / (1. + mubar * mubar);
    switch (which) {
        case C2Q_DIAG_M_TM: e = {1, mubar, 1, -mubar, gamma5}; break;
        case C2Q_DIAG_M_TM_INVERSE: e = {d, -mubar * d, d, mubar * d, gamma5}; break;
        case C2Q_DIAG_M_TM_MINUS: e = {1, -mubar, 1, mubar, gamma5}; break;
        case C2Q_DIAG_M_TM_INVERSE_MINUS: e = {d, mubar * d, d, -mubar * d, gamma5}; break;
        case C2Q_DIAG_M_TM_AND_GAMMA5: e = {1, mubar, -1, mubar, gamma5}; break;
        case C2Q_DIAG_M_TM_MINUS_AND_GAMMA5: e = {1, -mubar, -1, -mubar, gamma5}; break;
        default: break;
    }
    return e;
}

size_t field_bytes(const Geom& g, int prec)
{
    const size_t lanes = (size_t)g.stride;
    if (prec == 64) return lanes * 12 * 16;
    if (prec == 32) return lanes * 6 * 16;
    return lanes * 3 * 16 + lanes * 4;  // FP16 lanes + float norms
}

int field_alloc(c2q_ctx* ctx, const c2q_lattice& lat, int prec, c2q_spinor_eo* f)
{
    f->ctx  = ctx;
    f->lat  = lat;
    f->prec = prec;
    if (!make_geom(lat, &f->geom)) return fail(ctx, C2Q_BAD_ARG, "lattice extents must be even and >= 2");
    if (prec != 64 && (lat.nt % 4))
        return fail(ctx, C2Q_BAD_ARG, "FP32 / FP16 fields pair the times t and t + NT/2: NT must be a multiple of 4");
    const size_t bytes = field_bytes(f->geom, prec);
    void* p            = nullptr;
    C2Q_CUDA(ctx, cudaMallocAsync(&p, bytes, ctx->stream));
    // zero the padding once so that reductions over whole lanes never see garbage
    C2Q_CUDA(ctx, cudaMemsetAsync(p, 0, bytes, ctx->stream));
    f->data = p;
    f->norm = prec == 16 ? reinterpret_cast<float*>(static_cast<char*>(p) + (size_t)f->geom.stride * 3 * 16) : nullptr;
    f->owned = true;
    return C2Q_OK;
}

void field_free(c2q_spinor_eo* f)
{
    if (f && f->data && f->owned) cudaFreeAsync(f->data, f->ctx->stream);
    if (f) f->data = nullptr;
}

int gkind_for(int prec, int rec12)
{
    if (prec == 64) return rec12 ? G64R12 : G64;
    if (prec == 32) return rec12 ? G32R12 : G32;
    return rec12 ? G16R12 : G16;
}

cudaEvent_t profile_event(c2q_ctx* ctx)
{
    cudaEvent_t e;
    if (!ctx->event_pool.empty()) {
        e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
    } else {
        cudaEventCreate(&e);
    }
    return e;
}

int ensure_staging(c2q_ctx* ctx, size_t bytes)
{
    if (ctx->staging_cap >= bytes) return C2Q_OK;
    if (ctx->staging) {
        C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->staging);
        ctx->staging = nullptr;
    }
    C2Q_CUDA(ctx, cudaMalloc(&ctx->staging, bytes));
    ctx->staging_cap = bytes;
    return C2Q_OK;
}

int ensure_partials(c2q_ctx* ctx, size_t blocks)
{
    const size_t need = blocks * 2;
    if (ctx->partials_cap >= need) return C2Q_OK;
    if (ctx->partials) {
        C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->partials);
        ctx->partials = nullptr;
    }
    const size_t cap = need < 4096 ? 4096 : need;
    C2Q_CUDA(ctx, cudaMalloc(&ctx->partials, cap * sizeof(double)));
    ctx->partials_cap = cap;
    return C2Q_OK;
}

__global__ void pinned_copy_kernel(const unsigned* __restrict__ src, size_t spitch, unsigned* __restrict__ dst,
                                   size_t dpitch, int width, int height)
{
    pdl_enter();
    for (int r = blockIdx.x; r < height; r += gridDim.x)
        for (int c = threadIdx.x; c < width; c += blockDim.x) dst[(size_t)r * dpitch + c] = src[(size_t)r * spitch + c];
}

int pinned_copy(c2q_ctx* ctx, void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, int height,
                cudaStream_t stream)
{
    if (width % 4 || dpitch % 4 || spitch % 4 || height < 1) return fail(ctx, C2Q_BAD_ARG, "pinned_copy: word sizes");
    const int blocks = height < 16 ? height : 16;
    C2Q_CUDA(ctx, launch_dep(ctx->pdl, pinned_copy_kernel, dim3(blocks), dim3(32), 0, stream ? stream : ctx->stream,
                             static_cast<const unsigned*>(src), (size_t)(spitch / 4), static_cast<unsigned*>(dst),
                             (size_t)(dpitch / 4), (int)(width / 4), height));
    ctx->launches++;
    return C2Q_OK;
}

int ring_push(c2q_ctx* ctx, int k, double* dst_host_dev, const void* src, size_t spitch, size_t width, int n)
{
    if (width > 4 * sizeof(double) || n < 1 || n > 16) return fail(ctx, C2Q_BAD_ARG, "ring_push: slot size");
    double* slot = ctx->ring_dev + (size_t)(k % 4) * 16 * 4;
    int rc       = pinned_copy(ctx, slot, 4 * sizeof(double), src, spitch, width, n);
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaEventRecord(ctx->mon_ev[k % 4], ctx->stream));
    C2Q_CUDA(ctx, cudaStreamWaitEvent(ctx->monitor, ctx->mon_ev[k % 4], 0));
    rc = pinned_copy(ctx, dst_host_dev, 4 * sizeof(double), slot, 4 * sizeof(double), width, n, ctx->monitor);
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaEventRecord(ctx->ring_ev[k % 4], ctx->monitor));
    return C2Q_OK;
}

int read_scalars(c2q_ctx* ctx, const double* dev, int n, double* host)
{
    int rc = pinned_copy(ctx, ctx->host_pinned_dev, 0, dev, 0, n * sizeof(double));
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(host, ctx->host_pinned, n * sizeof(double));
    return C2Q_OK;
}

static RedArgs red_args(c2q_ctx* ctx, int fin)
{
    RedArgs r;
    r.partials = ctx->partials;
    r.ticket   = ctx->ticket;
    r.result   = ctx->red_result;
    r.sc       = ctx->scalars;
    r.fin      = fin;
    r.halt     = ctx->halt_dev;
    return r;
}

// ------------------------------------------------------------------ gauge
// AoS Matrixsu3[4V] (link mu + 4*site) -> [parity][mu][9 lanes][stride] FP64.
__global__ void gauge_import_kernel(const double2* __restrict__ aos, double2* __restrict__ out, Geom g, int vol)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4LL * vol) return;
    const int s = (int)(t >> 2), mu = (int)(t & 3);
    int rest = s / g.ns;
    int par  = s - rest * g.ns;
    par += rest % g.ns;
    rest /= g.ns;
    par += rest % g.ns + rest / g.ns;
    par &= 1;
    const int i      = s >> 1;
    const double2* m = aos + (size_t)t * 9;
    double2* dst     = out + (size_t)((par * 4 + mu) * 9) * g.stride + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) dst[(size_t)k * g.stride] = m[k];
}

__global__ void gauge_export_kernel(double2* __restrict__ aos, const double2* __restrict__ in, Geom g, int vol)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4LL * vol) return;
    const int s = (int)(t >> 2), mu = (int)(t & 3);
    int rest = s / g.ns;
    int par  = s - rest * g.ns;
    par += rest % g.ns;
    rest /= g.ns;
    par += rest % g.ns + rest / g.ns;
    par &= 1;
    const int i         = s >> 1;
    double2* m          = aos + (size_t)t * 9;
    const double2* src  = in + (size_t)((par * 4 + mu) * 9) * g.stride + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] = src[(size_t)k * g.stride];
}

// FP64 9-lane store -> FP64 12-real (first NL lanes, same layout).
__global__ void gauge_convert64_kernel(const double2* __restrict__ in, double2* __restrict__ out, Geom g)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8LL * g.stride) return;
    const int blk = (int)(t / g.stride), i = (int)(t - (long long)blk * g.stride);  // blk = parity*4 + mu
    const double2* src = in + (size_t)blk * 9 * g.stride + i;
    double2* dst       = out + (size_t)blk * 6 * g.stride + i;
#pragma unroll
    for (int k = 0; k < 6; ++k) dst[(size_t)k * g.stride] = src[(size_t)k * g.stride];
}

// FP64 9-lane store -> FP32 slot layout (pack.cuh): the links of the sites
// j and j + H of each (parity, mu) group side by side, NL float4 lanes.
template <int NL>
__global__ void gauge_convert32_kernel(const double2* __restrict__ in, float4* __restrict__ out, Geom g)
{
    const int ss = g.stride / 2, H = g.seo / 2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8LL * ss) return;
    const int blk = (int)(t / ss), j = (int)(t - (long long)blk * ss);
    if (j >= H) return;
    const double2* src = in + (size_t)blk * 9 * g.stride;
    float4* dst        = out + (size_t)blk * NL * ss + j;
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const double2 a = src[(size_t)k * g.stride + j], b = src[(size_t)k * g.stride + j + H];
        dst[(size_t)k * ss] = make_float4((float)a.x, (float)b.x, (float)a.y, (float)b.y);
    }
}

// FP64 9-lane store -> FP16 slot layout, biased 16-bit fixed point
// (u = rint(v * 32767) + 32768, v clamped to [-1, 1]).  12-real (NL = 6):
// rows 0 and 1 as three uint4 lanes (entry 2L of both sites, entry 2L+1 of both
// sites); 18-real (NL = 9): entries 0..7 as four uint4 lanes, entry 8 of both
// sites as one uint2 lane after them.
__device__ __forceinline__ unsigned enc16(double2 v)
{
    const double cx = fmin(1.0, fmax(-1.0, v.x)), cy = fmin(1.0, fmax(-1.0, v.y));
    const int lo    = __double2int_rn(cx * 32767.0) + 32768;
    const int hi    = __double2int_rn(cy * 32767.0) + 32768;
    return (unsigned)(lo & 0xffff) | ((unsigned)hi << 16);
}
template <int NL>
__global__ void gauge_convert16_kernel(const double2* __restrict__ in, uint4* __restrict__ out, Geom g)
{
    const int ss = g.stride / 2, H = g.seo / 2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8LL * ss) return;
    const int blk = (int)(t / ss), j = (int)(t - (long long)blk * ss);
    if (j >= H) return;
    const double2* src = in + (size_t)blk * 9 * g.stride;
    // a (parity, mu) group: 48 (12-real) or 72 (18-real) bytes per slot
    char* grp   = reinterpret_cast<char*>(out) + (size_t)blk * (NL == 6 ? 48 : 72) * ss;
    uint4* dst  = reinterpret_cast<uint4*>(grp) + j;
    constexpr int LANES = NL == 6 ? 3 : 4;
#pragma unroll
    for (int L = 0; L < LANES; ++L) {
        const size_t e0 = (size_t)(2 * L) * g.stride, e1 = (size_t)(2 * L + 1) * g.stride;
        dst[(size_t)L * ss] = make_uint4(enc16(src[e0 + j]), enc16(src[e0 + j + H]), enc16(src[e1 + j]),
                                         enc16(src[e1 + j + H]));
    }
    if (NL == 9) {
        uint2* tail = reinterpret_cast<uint2*>(grp + (size_t)64 * ss) + j;
        *tail       = make_uint2(enc16(src[(size_t)8 * g.stride + j]), enc16(src[(size_t)8 * g.stride + j + H]));
    }
}

int gauge_ensure(c2q_gauge* g, int kind)
{
    c2q_ctx* ctx = g->ctx;
    if (kind < 0 || kind >= GAUGE_KINDS) return fail(ctx, C2Q_BAD_ARG, "bad gauge kind");
    if (g->store[kind].data) return C2Q_OK;
    if (!g->store[G64].data) return fail(ctx, C2Q_BAD_ARG, "gauge field not uploaded");
    const size_t lanes = (size_t)8 * g->geom.stride;
    size_t bytes       = 0;
    switch (kind) {
        case G64R12: bytes = lanes * 6 * 16; break;
        case G32: case G32TG: bytes = lanes * 9 * 8; break;
        case G32R12: case G32R12TG: bytes = lanes * 6 * 8; break;
        case G16R12: case G16R12TG: bytes = lanes * 6 * 4; break;
        case G16: case G16TG: bytes = lanes * 9 * 4; break;
        default: return fail(ctx, C2Q_BAD_ARG, "bad gauge kind");
    }
    if (kind != G64R12 && (g->lat.nt % 4))
        return fail(ctx, C2Q_BAD_ARG, "FP32 / FP16 links pair the times t and t + NT/2: NT must be a multiple of 4");
    const double2* src = static_cast<const double2*>(g->store[G64].data);
    void* tmp          = nullptr;  // temporal gauge: the transformed FP64 links
    if (gkind_is_tg(kind)) {
        C2Q_CUDA(ctx, cudaMalloc(&tmp, lanes * 9 * 16));
        const int rc = tg_links_fp64(g, tmp);
        if (rc) {
            cudaFree(tmp);
            return rc;
        }
        src = static_cast<const double2*>(tmp);
    }
    void* p = nullptr;
    const cudaError_t ea = cudaMalloc(&p, bytes);
    if (ea != cudaSuccess) {
        cudaFree(tmp);
        return cuda_fail(ctx, ea, "cudaMalloc(gauge copy)");
    }
    const int threads = 256;
    const unsigned blocks = (unsigned)((lanes + threads - 1) / threads);
    switch (kind) {
        case G64R12: gauge_convert64_kernel<<<blocks, threads, 0, ctx->stream>>>(src, (double2*)p, g->geom); break;
        case G32: gauge_convert32_kernel<9><<<blocks, threads, 0, ctx->stream>>>(src, (float4*)p, g->geom); break;
        case G32R12: gauge_convert32_kernel<6><<<blocks, threads, 0, ctx->stream>>>(src, (float4*)p, g->geom); break;
        case G16R12: gauge_convert16_kernel<6><<<blocks, threads, 0, ctx->stream>>>(src, (uint4*)p, g->geom); break;
        case G16: gauge_convert16_kernel<9><<<blocks, threads, 0, ctx->stream>>>(src, (uint4*)p, g->geom); break;
        case G32TG: gauge_convert32_kernel<9><<<blocks, threads, 0, ctx->stream>>>(src, (float4*)p, g->geom); break;
        case G32R12TG: gauge_convert32_kernel<6><<<blocks, threads, 0, ctx->stream>>>(src, (float4*)p, g->geom); break;
        case G16R12TG: gauge_convert16_kernel<6><<<blocks, threads, 0, ctx->stream>>>(src, (uint4*)p, g->geom); break;
        case G16TG: gauge_convert16_kernel<9><<<blocks, threads, 0, ctx->stream>>>(src, (uint4*)p, g->geom); break;
    }
    ctx->launches++;
    const cudaError_t ek = cudaGetLastError();
    if (tmp) {  // stream-ordered: the conversion finishes before the scratch is released
        cudaStreamSynchronize(ctx->stream);
        cudaFree(tmp);
    }
    if (ek != cudaSuccess) {
        cudaFree(p);
        return cuda_fail(ctx, ek, "gauge conversion");
    }
    g->store[kind].data  = p;
    g->store[kind].bytes = bytes;
    return C2Q_OK;
}

int gauge_drop_derived(c2q_gauge* g)
{
    c2q_ctx* ctx = g->ctx;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int k = 1; k < GAUGE_KINDS; ++k) {
        cudaFree(g->store[k].data);
        g->store[k] = GaugeStore{};
    }
    cudaFree(g->tg_transform.data);
    g->tg_transform = GaugeStore{};
    return C2Q_OK;
}

// ------------------------------------------------------------------ launches
template <int P, int NL, int EPI, int DOT, int PH>
static void dslash_go(const DslashParams<P>& prm, int blocks, cudaStream_t s)
{
    launch_dep(prm.pdl != 0, dslash_kernel<P, NL, EPI, DOT, PH>, dim3(blocks), dim3(128), 0, s, prm);
}

template <int P, int NL, int PH>
static void dslash_dispatch_ph(const DslashParams<P>& prm, int epi, int dot, int blocks, cudaStream_t s)
{
    switch (epi * 3 + dot) {
        case 0: dslash_go<P, NL, EPI_PLAIN, DOT_NONE, PH>(prm, blocks, s); break;
        case 1: dslash_go<P, NL, EPI_PLAIN, DOT_Y, PH>(prm, blocks, s); break;
        case 2: dslash_go<P, NL, EPI_PLAIN, DOT_SELF, PH>(prm, blocks, s); break;
        case 3: dslash_go<P, NL, EPI_DIAG, DOT_NONE, PH>(prm, blocks, s); break;
        case 4: dslash_go<P, NL, EPI_DIAG, DOT_Y, PH>(prm, blocks, s); break;
        case 5: dslash_go<P, NL, EPI_DIAG, DOT_SELF, PH>(prm, blocks, s); break;
        case 6: dslash_go<P, NL, EPI_AXPY, DOT_NONE, PH>(prm, blocks, s); break;
        case 7: dslash_go<P, NL, EPI_AXPY, DOT_Y, PH>(prm, blocks, s); break;
        case 8: dslash_go<P, NL, EPI_AXPY, DOT_SELF, PH>(prm, blocks, s); break;
    }
}

// FP64 (bandwidth-bound) decides the phase pattern per launch.
template <int P, int NL>
static void dslash_dispatch(const DslashParams<P>& prm, int epi, int dot, int blocks, cudaStream_t s)
{
    dslash_dispatch_ph<P, NL, PH_ANY>(prm, epi, dot, blocks, s);
}

template <int P>
static int dslash_typed(c2q_ctx* ctx, const c2q_gauge* g, int gkind, c2q_spinor_eo* out, const c2q_spinor_eo* in,
                        int out_parity, double kappa, int epi, const EpiArgs& e, const c2q_spinor_eo* x,
                        const DotSpec& dot)
{
    DslashParams<P> prm;
    prm.out        = sptr<P>(out);
    prm.in         = sptr<P>(in);
    prm.x          = sptr<P>(x);
    prm.y          = sptr<P>(dot.y);
    prm.gauge      = g->store[gkind].data;
    prm.g          = out->geom;
    prm.c          = hop_coef(out->lat, kappa);
    prm.e          = e;
    prm.out_parity = out_parity;
    const int blocks = (out->geom.seo + 127) / 128;
    if (dot.mode) {
        int rc = ensure_partials(ctx, blocks);
        if (rc) return rc;
    }
    prm.red = red_args(ctx, dot.fin);
    prm.pdl = ctx->pdl;
    const bool r12 = gkind == G64R12 || gkind == G32R12 || gkind == G16R12;  // FP64 here
    c2q_ctx::Timed tm{};
    if (ctx->profiling) {
        tm.a     = profile_event(ctx);
        tm.b     = profile_event(ctx);
        tm.prec  = P;
        tm.sites = (double)out->geom.seo;
        // compulsory traffic per output site: 8 links (each read once per sweep),
        // the input spinor (each read once through L2 reuse), the output, plus
        // the epilogue/reduction operands read at the output site
        const double sp = 192.0;
        const double lk = (r12 ? 12.0 : 18.0) * 8.0;
        tm.bytes = tm.sites * (8.0 * lk + sp * (2.0 + (epi == EPI_AXPY ? 1.0 : 0.0) + (dot.mode == DOT_Y ? 1.0 : 0.0)));
        cudaEventRecord(tm.a, ctx->stream);
    }
    if (r12)
        dslash_dispatch<P, 6>(prm, epi, dot.mode, blocks, ctx->stream);
    else
        dslash_dispatch<P, 9>(prm, epi, dot.mode, blocks, ctx->stream);
    if (ctx->profiling) {
        cudaEventRecord(tm.b, ctx->stream);
        ctx->timed.push_back(tm);
    }
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

static bool gauge_matches(int prec, int gkind)
{
    if (prec == 64) return gkind == G64 || gkind == G64R12;
    if (prec == 32) return gkind == G32 || gkind == G32R12;
    return gkind == G16R12 || gkind == G16;
}

int launch_dslash(c2q_ctx* ctx, const c2q_gauge* g, int gkind, c2q_spinor_eo* out, const c2q_spinor_eo* in,
                  int out_parity, double kappa, int epi, const EpiArgs& e, const c2q_spinor_eo* x,
                  const DotSpec& dot)
{
    if (!out || !in || !g) return fail(ctx, C2Q_BAD_ARG, "null field");
    if (out == in) return fail(ctx, C2Q_BAD_ARG, "dslash output must not alias its input");
    if (in->prec != out->prec || (x && x->prec != out->prec) || (dot.y && dot.y->prec != out->prec))
        return fail(ctx, C2Q_BAD_ARG, "precision mismatch");
    if (!same_lattice(out->lat, in->lat) || !same_lattice(out->lat, g->lat))
        return fail(ctx, C2Q_BAD_ARG, "lattice mismatch between fields and gauge field");
    if (!gauge_matches(out->prec, gkind)) return fail(ctx, C2Q_BAD_ARG, "gauge precision mismatch");
    int rc = gauge_ensure(const_cast<c2q_gauge*>(g), gkind);
    if (rc) return rc;
    if (out->prec == 64) return dslash_typed<64>(ctx, g, gkind, out, in, out_parity, kappa, epi, e, x, dot);
    PkBatch B;
    B.n          = 1;
    B.out[0]     = out;
    B.in[0]      = in;
    B.x[0]       = x;
    B.y[0]       = dot.y;
    B.out_parity = out_parity;
    B.kappa      = kappa;
    B.epi        = epi;
    B.e          = e;
    B.dot_mode   = dot.mode;
    B.fin        = dot.fin;
    return launch_pdslash(ctx, g, gkind, B);
}

template <int P>
static int blas_typed(c2q_ctx* ctx, const BlasSpec& s, const c2q_spinor_eo* ref)
{
    BlasArgs<P> A;
    A.out    = sptr<P>(s.out);
    A.x      = sptr<P>(s.x);
    A.y      = sptr<P>(s.y);
    A.z      = sptr<P>(s.z);
    A.w      = sptr<P>(s.w);
    A.out2   = sptr<P>(s.out2);
    A.a      = s.a;
    A.b      = s.b;
    A.n      = ref->geom.seo;
    A.stride = ref->geom.stride;
    A.op     = s.op;
    A.dot    = s.dot;
    const int blocks = (A.n + BLAS_THREADS - 1) / BLAS_THREADS;
    if (s.dot) {  // dot 3 and 4 reduce four doubles per block
        int rc = ensure_partials(ctx, s.dot >= 3 ? 2 * (size_t)blocks : (size_t)blocks);
        if (rc) return rc;
    }
    A.red         = red_args(ctx, s.fin);
    A.red.fin_arg = s.fin_arg;
    C2Q_CUDA(ctx, launch_dep(ctx->pdl, blas_kernel<P>, dim3(blocks), dim3(BLAS_THREADS), 0, ctx->stream, A));
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

int launch_blas(c2q_ctx* ctx, const BlasSpec& s)
{
    const c2q_spinor_eo* ref = s.out ? s.out : s.x;
    if (!ref || !s.x) return fail(ctx, C2Q_BAD_ARG, "null field");
    if (s.op == B_BICG_XR && (!s.out || !s.y || !s.z || !s.w || !s.out2 || s.dot != 4))
        return fail(ctx, C2Q_BAD_ARG, "B_BICG_XR needs out, x, y, z, w, out2 and dot 4");
    for (const c2q_spinor_eo* f : {(const c2q_spinor_eo*)s.out, s.x, s.y, s.z, s.w, (const c2q_spinor_eo*)s.out2})
        if (f && (f->prec != ref->prec || !same_lattice(f->lat, ref->lat)))
            return fail(ctx, C2Q_BAD_ARG, "fields differ in precision or lattice");
    switch (ref->prec) {
        case 64: return blas_typed<64>(ctx, s, ref);
        case 32: return blas_typed<32>(ctx, s, ref);
        default: return blas_typed<16>(ctx, s, ref);
    }
}

template <int P>
static int cg_update_typed(c2q_ctx* ctx, c2q_spinor_eo* x, c2q_spinor_eo* r, const c2q_spinor_eo* p,
                           const c2q_spinor_eo* v)
{
    CgUpdateArgs<P> A;
    A.x = sptr<P>(x);
    A.r = sptr<P>(r);
    A.p = sptr<P>(p);
    A.v = sptr<P>(v);
    A.sc = ctx->scalars;
    A.n = x->geom.seo;
    A.stride = x->geom.stride;
    const int blocks = (A.n + BLAS_THREADS - 1) / BLAS_THREADS;
    int rc = ensure_partials(ctx, blocks);
    if (rc) return rc;
    A.red = red_args(ctx, FIN_CG_BETA);
    C2Q_CUDA(ctx, launch_dep(ctx->pdl, cg_update_kernel<P>, dim3(blocks), dim3(BLAS_THREADS), 0, ctx->stream, A));
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

int launch_cg_update(c2q_ctx* ctx, c2q_spinor_eo* x, c2q_spinor_eo* r, const c2q_spinor_eo* p,
                     const c2q_spinor_eo* v)
{
    switch (x->prec) {
        case 64: return cg_update_typed<64>(ctx, x, r, p, v);
        case 32: return cg_update_typed<32>(ctx, x, r, p, v);
        default: return cg_update_typed<16>(ctx, x, r, p, v);
    }
}

template <int P>
static int cg_p_typed(c2q_ctx* ctx, c2q_spinor_eo* p, const c2q_spinor_eo* r)
{
    CgPArgs<P> A;
    A.p = sptr<P>(p);
    A.r = sptr<P>(r);
    A.sc = ctx->scalars;
    A.n = p->geom.seo;
    A.stride = p->geom.stride;
    const int blocks = (A.n + BLAS_THREADS - 1) / BLAS_THREADS;
    C2Q_CUDA(ctx, launch_dep(ctx->pdl, cg_p_kernel<P>, dim3(blocks), dim3(BLAS_THREADS), 0, ctx->stream, A));
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

int launch_cg_p(c2q_ctx* ctx, c2q_spinor_eo* p, const c2q_spinor_eo* r)
{
    switch (p->prec) {
        case 64: return cg_p_typed<64>(ctx, p, r);
        case 32: return cg_p_typed<32>(ctx, p, r);
        default: return cg_p_typed<16>(ctx, p, r);
    }
}

template <int PO, int PI>
static void convert_go(c2q_ctx* ctx, c2q_spinor_eo* out, const c2q_spinor_eo* in)
{
    const int n = out->geom.seo;
    convert_kernel<PO, PI><<<(n + BLAS_THREADS - 1) / BLAS_THREADS, BLAS_THREADS, 0, ctx->stream>>>(
        sptr<PO>(out), sptr<PI>(in), n, out->geom.stride);
}

int launch_convert(c2q_ctx* ctx, c2q_spinor_eo* out, const c2q_spinor_eo* in)
{
    const int key = out->prec * 1000 + in->prec;
    switch (key) {
        case 64064: convert_go<64, 64>(ctx, out, in); break;
        case 64032: convert_go<64, 32>(ctx, out, in); break;
        case 64016: convert_go<64, 16>(ctx, out, in); break;
        case 32064: convert_go<32, 64>(ctx, out, in); break;
        case 32032: convert_go<32, 32>(ctx, out, in); break;
        case 32016: convert_go<32, 16>(ctx, out, in); break;
        case 16064: convert_go<16, 64>(ctx, out, in); break;
        case 16032: convert_go<16, 32>(ctx, out, in); break;
        case 16016: convert_go<16, 16>(ctx, out, in); break;
        default: return fail(ctx, C2Q_BAD_ARG, "bad precision pair");
    }
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    return C2Q_OK;
}

// Fermion matrices (physics/fermionmatrix/fermionmatrix.cpp:224-664), each
// Aee-type application fused into two sweeps:
//   sweep 1: tmp = R_o^{-1} D_oe in           (dslash(ODD) + M_tm_inverse_sitediagonal[_minus])
//   sweep 2: out = [g5](R_e in - D_eo tmp)     (dslash(EVEN) + M_tm_sitediagonal[_minus] + saxpy[_AND_gamma5])
// For the Wilson action R = 1.  QplusQminus_eo = Qplus_eo(Qminus_eo(in)).
static int aee_sweeps(c2q_ctx* ctx, c2q_spinor_eo* out, const c2q_gauge* g, int gkind, const c2q_spinor_eo* in,
                      double kappa, double mubar, int action, int minus, int g5, c2q_spinor_eo* tmp,
                      const DotSpec& dot)
{
    const bool tm = action == C2Q_ACTION_TWISTEDMASS;
    EpiArgs e1    = tm ? diag_epi(mubar, minus ? C2Q_DIAG_M_TM_INVERSE_MINUS : C2Q_DIAG_M_TM_INVERSE, 0)
                       : EpiArgs{1, 0, 1, 0, 0};
    int rc = launch_dslash(ctx, g, gkind, tmp, in, /*ODD -> even sites*/ 0, kappa, tm ? EPI_DIAG : EPI_PLAIN, e1,
                           nullptr, DotSpec{});
    if (rc) return rc;
    EpiArgs e2 = tm ? diag_epi(mubar, minus ? C2Q_DIAG_M_TM_MINUS : C2Q_DIAG_M_TM, g5) : EpiArgs{1, 0, 1, 0, g5};
    return launch_dslash(ctx, g, gkind, out, tmp, /*EVEN -> odd sites*/ 1, kappa, EPI_AXPY, e2, in, dot);
}

int apply_operator(c2q_ctx* ctx, int op, c2q_spinor_eo* out, const c2q_gauge* g, int gkind,
                   const c2q_spinor_eo* in, double kappa, double mubar, int action, c2q_spinor_eo* tmp1,
                   c2q_spinor_eo* tmp2, const DotSpec& dot, int* sweeps)
{
    if (action != C2Q_ACTION_WILSON && action != C2Q_ACTION_TWISTEDMASS)
        return fail(ctx, C2Q_BAD_ARG, "unknown fermion action (wilson or twistedmass)");
    if (out == in) return fail(ctx, C2Q_BAD_ARG, "operator output must not alias its input");
    int rc = 0;
    switch (op) {
        case C2Q_OP_AEE: rc = aee_sweeps(ctx, out, g, gkind, in, kappa, mubar, action, 0, 0, tmp1, dot); break;
        case C2Q_OP_AEE_MINUS: rc = aee_sweeps(ctx, out, g, gkind, in, kappa, mubar, action, 1, 0, tmp1, dot); break;
        case C2Q_OP_QPLUS_EO:
        case C2Q_OP_AEE_AND_GAMMA5_EO:
            rc = aee_sweeps(ctx, out, g, gkind, in, kappa, mubar, action, 0, 1, tmp1, dot);
            break;
        case C2Q_OP_QMINUS_EO:
        case C2Q_OP_AEE_MINUS_AND_GAMMA5_EO:
            rc = aee_sweeps(ctx, out, g, gkind, in, kappa, mubar, action, 1, 1, tmp1, dot);
            break;
        case C2Q_OP_QPLUSQMINUS_EO:
            rc = aee_sweeps(ctx, tmp2, g, gkind, in, kappa, mubar, action, 1, 1, tmp1, DotSpec{});
            if (!rc) rc = aee_sweeps(ctx, out, g, gkind, tmp2, kappa, mubar, action, 0, 1, tmp1, dot);
            if (sweeps) *sweeps += 2;
            break;
        default: return fail(ctx, C2Q_BAD_ARG, "unknown eo fermion matrix");
    }
    if (sweeps) *sweeps += 2;
    return rc;
}

}  // namespace c2q

using namespace c2q;

// ==================================================================== C ABI
extern "C" {

static void profile_recycle(c2q_ctx* ctx);

C2Q_EXPORT const char* c2q_version(void) { return "cl2qcd-b200 0.1 (sm_100a)"; }

C2Q_EXPORT int c2q_ctx_create(c2q_ctx** out, int device, void* cuda_stream)
{
    if (!out) return C2Q_BAD_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return C2Q_NO_DEVICE;
    if (device < 0 || device >= n) return C2Q_BAD_ARG;
    c2q_ctx* ctx = new c2q_ctx();
    ctx->device  = device;
    if (const char* at = getenv("C2Q_AUTOTUNE")) ctx->autotune = at[0] != '0';
    if (const char* pd = getenv("C2Q_DEPENDENT_LAUNCH")) ctx->pdl = pd[0] != '0';
    int rc       = C2Q_OK;
    auto chk     = [&](cudaError_t e, const char* w) {
        if (e != cudaSuccess && rc == C2Q_OK) rc = cuda_fail(ctx, e, w);
    };
    chk(cudaSetDevice(device), "cudaSetDevice");
    if (cuda_stream) {
        ctx->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        chk(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ctx->own_stream = true;
    }
    chk(cudaMalloc(&ctx->ticket, 64 * sizeof(unsigned)), "cudaMalloc(ticket)");
    chk(cudaMalloc(&ctx->red_result, 8 * sizeof(double)), "cudaMalloc(result)");
    chk(cudaMalloc(&ctx->scalars, sizeof(SolverScalars)), "cudaMalloc(scalars)");
    chk(cudaMallocHost(&ctx->host_pinned, 64 * sizeof(double)), "cudaMallocHost");
    if (rc == C2Q_OK) chk(cudaHostGetDevicePointer((void**)&ctx->host_pinned_dev, ctx->host_pinned, 0),
                          "cudaHostGetDevicePointer");
    chk(cudaEventCreate(&ctx->ev0), "cudaEventCreate");
    chk(cudaEventCreate(&ctx->ev1), "cudaEventCreate");
    for (auto& e : ctx->ring_ev) chk(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    for (auto& e : ctx->mon_ev) chk(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    chk(cudaStreamCreateWithFlags(&ctx->monitor, cudaStreamNonBlocking), "cudaStreamCreate(monitor)");
    chk(cudaMalloc(&ctx->ring_dev, 4 * 16 * 4 * sizeof(double)), "cudaMalloc(ring)");
    if (rc == C2Q_OK) {
        chk(cudaMemsetAsync(ctx->ticket, 0, 64 * sizeof(unsigned), ctx->stream), "memset");
        chk(cudaMemsetAsync(ctx->scalars, 0, sizeof(SolverScalars), ctx->stream), "memset");
        rc = rc ? rc : ensure_partials(ctx, 4096);
        // keep freed stream-ordered allocations cached for the next solve
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t thr = ~0ULL;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        chk(cudaStreamSynchronize(ctx->stream), "sync");
    }
    if (rc != C2Q_OK) {
        c2q_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_ctx_destroy(c2q_ctx* ctx)
{
    if (!ctx) return C2Q_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->monitor) cudaStreamSynchronize(ctx->monitor);
    cudaFree(ctx->partials);
    cudaFree(ctx->ring_dev);
    cudaFree(ctx->ticket);
    if (ctx->tune_scratch) cudaFree(ctx->tune_scratch);
    if (ctx->batch_ring) cudaFreeHost(ctx->batch_ring);
    cudaFree(ctx->red_result);
    cudaFree(ctx->scalars);
    cudaFree(ctx->staging);
    if (ctx->host_pinned) cudaFreeHost(ctx->host_pinned);
    profile_recycle(ctx);
    for (auto e : ctx->event_pool) cudaEventDestroy(e);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (auto e : ctx->ring_ev)
        if (e) cudaEventDestroy(e);
    for (auto e : ctx->mon_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->monitor) cudaStreamDestroy(ctx->monitor);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return C2Q_OK;
}

C2Q_EXPORT const char* c2q_last_error(const c2q_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

C2Q_EXPORT int c2q_ctx_synchronize(c2q_ctx* ctx)
{
    if (!ctx) return C2Q_BAD_ARG;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

C2Q_EXPORT long long c2q_ctx_launch_count(const c2q_ctx* ctx) { return ctx ? ctx->launches : 0; }

static void profile_recycle(c2q_ctx* ctx)
{
    for (auto& t : ctx->timed) {
        ctx->event_pool.push_back(t.a);
        ctx->event_pool.push_back(t.b);
    }
    ctx->timed.clear();
}

C2Q_EXPORT int c2q_ctx_profile(c2q_ctx* ctx, int enable)
{
    if (!ctx) return C2Q_BAD_ARG;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    profile_recycle(ctx);
    ctx->profiling = enable != 0;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_ctx_profile_read(c2q_ctx* ctx, int prec, long long* launches, double* total_ms, double* bytes)
{
    if (!ctx || !launches || !total_ms || !bytes) return C2Q_BAD_ARG;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *launches = 0;
    *total_ms = 0.0;
    *bytes    = 0.0;
    for (auto& t : ctx->timed) {
        if (t.prec != prec) continue;
        float ms = 0.f;
        C2Q_CUDA(ctx, cudaEventElapsedTime(&ms, t.a, t.b));
        *launches += 1;
        *total_ms += ms;
        *bytes += t.bytes;
    }
    return C2Q_OK;
}

// ---------------------------------------------------------------- gauge
C2Q_EXPORT int c2q_gauge_create(c2q_ctx* ctx, const c2q_lattice* lat, c2q_gauge** out)
{
    if (!ctx || !lat || !out) return C2Q_BAD_ARG;
    c2q_gauge* g = new c2q_gauge();
    g->ctx       = ctx;
    g->lat       = *lat;
    if (!make_geom(*lat, &g->geom)) {
        delete g;
        return fail(ctx, C2Q_BAD_ARG, "lattice extents must be even and >= 2");
    }
    const size_t bytes = (size_t)8 * 9 * g->geom.stride * 16;
    cudaError_t e      = cudaMalloc(&g->store[G64].data, bytes);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(ctx, e, "cudaMalloc(gauge)");
    }
    g->store[G64].bytes = bytes;
    cudaMemsetAsync(g->store[G64].data, 0, bytes, ctx->stream);
    *out = g;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_gauge_destroy(c2q_gauge* g)
{
    if (!g) return C2Q_OK;
    cudaStreamSynchronize(g->ctx->stream);
    for (auto& s : g->store) cudaFree(s.data);
    cudaFree(g->tg_transform.data);
    delete g;
    return C2Q_OK;
}

C2Q_EXPORT size_t c2q_gauge_device_bytes(const c2q_gauge* g)
{
    size_t b = 0;
    if (g) {
        for (auto& s : g->store) b += s.bytes;
        b += g->tg_transform.bytes;
    }
    return b;
}

C2Q_EXPORT int c2q_gauge_upload(c2q_gauge* g, const double* aos)
{
    if (!g || !aos) return C2Q_BAD_ARG;
    c2q_ctx* ctx     = g->ctx;
    const int vol    = 2 * g->geom.seo;
    const size_t bytes = (size_t)4 * vol * 18 * sizeof(double);
    int rc           = ensure_staging(ctx, bytes);
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaMemcpyAsync(ctx->staging, aos, bytes, cudaMemcpyHostToDevice, ctx->stream));
    const long long n = 4LL * vol;
    gauge_import_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        (const double2*)ctx->staging, (double2*)g->store[G64].data, g->geom, vol);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    // lower-precision copies (and the temporal gauge) are rebuilt from the new
    // links on next use
    rc = gauge_drop_derived(g);
    if (rc) return rc;
    g->rec12_dev = -1.0;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

C2Q_EXPORT int c2q_gauge_download(const c2q_gauge* g, double* aos)
{
    if (!g || !aos) return C2Q_BAD_ARG;
    c2q_ctx* ctx       = g->ctx;
    const int vol      = 2 * g->geom.seo;
    const size_t bytes = (size_t)4 * vol * 18 * sizeof(double);
    int rc             = ensure_staging(ctx, bytes);
    if (rc) return rc;
    const long long n = 4LL * vol;
    gauge_export_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        (double2*)ctx->staging, (const double2*)g->store[G64].data, g->geom, vol);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    C2Q_CUDA(ctx, cudaMemcpyAsync(aos, ctx->staging, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

// ---------------------------------------------------------------- spinors
C2Q_EXPORT int c2q_spinor_eo_create(c2q_ctx* ctx, const c2q_lattice* lat, c2q_spinor_eo** out)
{
    return c2q_spinor_eo_create_precision(ctx, lat, C2Q_PREC_FP64, out);
}

C2Q_EXPORT int c2q_spinor_eo_create_precision(c2q_ctx* ctx, const c2q_lattice* lat, int precision,
                                              c2q_spinor_eo** out)
{
    if (!ctx || !lat || !out) return C2Q_BAD_ARG;
    if (precision != 64 && precision != 32 && precision != 16)
        return fail(ctx, C2Q_BAD_ARG, "precision must be 64, 32 or 16");
    c2q_spinor_eo* f = new c2q_spinor_eo();
    int rc           = field_alloc(ctx, *lat, precision, f);
    if (rc) {
        delete f;
        return rc;
    }
    *out = f;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_spinor_eo_destroy(c2q_spinor_eo* f)
{
    if (!f) return C2Q_OK;
    field_free(f);
    delete f;
    return C2Q_OK;
}

static int aos_transfer(c2q_spinor_eo* f, double* host_dst, const double* host_src, int mode, int par,
                        const double* dev_src_full, cudaStream_t stream = nullptr)
{
    c2q_ctx* ctx       = f->ctx;
    cudaStream_t st    = stream ? stream : ctx->stream;
    const size_t sites = mode == 0 ? (size_t)f->geom.seo : (size_t)f->geom.seo * 2;
    const size_t bytes = sites * 24 * sizeof(double);
    AosArgs A;
    A.soa    = static_cast<double2*>(f->data);
    A.n      = f->geom.seo;
    A.stride = f->geom.stride;
    A.mode   = mode;
    A.par    = par;
    A.ns     = f->geom.ns;
    A.nsh    = f->geom.nsh;
    const int blocks = (A.n + 255) / 256;
    if (host_src || dev_src_full) {
        if (host_src) {
            int rc = ensure_staging(ctx, bytes);
            if (rc) return rc;
            C2Q_CUDA(ctx, cudaMemcpyAsync(ctx->staging, host_src, bytes, cudaMemcpyHostToDevice, st));
            A.aos = static_cast<double*>(ctx->staging);
        } else {
            A.aos = const_cast<double*>(dev_src_full);
        }
        aos_to_soa_kernel<<<blocks, 256, 0, st>>>(A);
        ctx->launches++;
        C2Q_CUDA(ctx, cudaGetLastError());
    } else {
        A.aos = static_cast<double*>(ctx->staging);
        soa_to_aos_kernel<<<blocks, 256, 0, st>>>(A);
        ctx->launches++;
        C2Q_CUDA(ctx, cudaGetLastError());
        if (host_dst) {
            C2Q_CUDA(ctx, cudaMemcpyAsync(host_dst, ctx->staging, bytes, cudaMemcpyDeviceToHost, st));
        }
    }
    return C2Q_OK;
}

C2Q_EXPORT int c2q_spinor_eo_upload(c2q_spinor_eo* f, const double* aos)
{
    if (!f || !aos) return C2Q_BAD_ARG;
    int rc = 0;
    if (f->prec == 64) {
        rc = aos_transfer(f, nullptr, aos, 0, 0, nullptr);
    } else {  // through an FP64 field, rounded on the device
        c2q_spinor_eo t;
        rc = field_alloc(f->ctx, f->lat, 64, &t);
        if (rc) return rc;
        rc = aos_transfer(&t, nullptr, aos, 0, 0, nullptr);
        if (!rc) rc = launch_convert(f->ctx, f, &t);
        field_free(&t);
    }
    if (rc) return rc;
    C2Q_CUDA(f->ctx, cudaStreamSynchronize(f->ctx->stream));
    return C2Q_OK;
}

C2Q_EXPORT int c2q_spinor_eo_download(const c2q_spinor_eo* f, double* aos)
{
    if (!f || !aos) return C2Q_BAD_ARG;
    c2q_spinor_eo* ff = const_cast<c2q_spinor_eo*>(f);
    int rc            = ensure_staging(ff->ctx, (size_t)f->geom.seo * 24 * sizeof(double));
    if (rc) return rc;
    if (f->prec == 64) {
        rc = aos_transfer(ff, aos, nullptr, 0, 0, nullptr);
    } else {
        c2q_spinor_eo t;
        rc = field_alloc(f->ctx, f->lat, 64, &t);
        if (rc) return rc;
        rc = launch_convert(f->ctx, &t, f);
        if (!rc) rc = aos_transfer(&t, aos, nullptr, 0, 0, nullptr);
        if (!rc) C2Q_CUDA(f->ctx, cudaStreamSynchronize(f->ctx->stream));
        field_free(&t);
    }
    if (rc) return rc;
    C2Q_CUDA(f->ctx, cudaStreamSynchronize(f->ctx->stream));
    return C2Q_OK;
}

// The same transfers, enqueued without waiting (FP64 fields) on the context's
// stream or on a stream of the caller's: with a copy stream the transfers of
// one solve's source and solution overlap another solve of the same context.
// The context's staging buffer is shared: its transfers must be ordered (one
// stream, or events).
C2Q_EXPORT int c2q_spinor_eo_upload_async(c2q_spinor_eo* f, const double* aos, void* stream)
{
    if (!f || !aos) return C2Q_BAD_ARG;
    if (f->prec != 64) return fail(f->ctx, C2Q_BAD_ARG, "asynchronous transfers take FP64 fields");
    const int rc = ensure_staging(f->ctx, (size_t)f->geom.seo * 24 * sizeof(double));
    return rc ? rc : aos_transfer(f, nullptr, aos, 0, 0, nullptr, static_cast<cudaStream_t>(stream));
}

C2Q_EXPORT int c2q_spinor_eo_download_async(const c2q_spinor_eo* f, double* aos, void* stream)
{
    if (!f || !aos) return C2Q_BAD_ARG;
    c2q_spinor_eo* ff = const_cast<c2q_spinor_eo*>(f);
    if (f->prec != 64) return fail(f->ctx, C2Q_BAD_ARG, "asynchronous transfers take FP64 fields");
    const int rc = ensure_staging(ff->ctx, (size_t)f->geom.seo * 24 * sizeof(double));
    return rc ? rc : aos_transfer(ff, aos, nullptr, 0, 0, nullptr, static_cast<cudaStream_t>(stream));
}

C2Q_EXPORT int c2q_spinor_eo_precision(const c2q_spinor_eo* f) { return f ? f->prec : C2Q_BAD_ARG; }

C2Q_EXPORT int c2q_spinor_eo_convert(c2q_spinor_eo* out, const c2q_spinor_eo* in)
{
    if (!out || !in) return C2Q_BAD_ARG;
    if (!same_lattice(out->lat, in->lat)) return fail(out->ctx, C2Q_BAD_ARG, "lattice mismatch");
    if (out == in) return C2Q_OK;
    return launch_convert(out->ctx, out, in);
}

C2Q_EXPORT int c2q_ctx_set_link_format(c2q_ctx* ctx, int rec12)
{
    if (!ctx || (rec12 != 0 && rec12 != 1)) return C2Q_BAD_ARG;
    ctx->rec12 = rec12;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_spinor_eo_zero(c2q_spinor_eo* f)
{
    if (!f) return C2Q_BAD_ARG;
    C2Q_CUDA(f->ctx, cudaMemsetAsync(f->data, 0, field_bytes(f->geom, f->prec), f->ctx->stream));
    return C2Q_OK;
}

// Seeded sources generated in place, site by site with the counter-based
// SplitMix64 streams of c2q_source_generate (inputs.cpp): Z2 sources are
// bit-identical to the host generator, Gaussian ones agree to the rounding of
// the device's log / sqrt / sincos.
__device__ __forceinline__ uint64_t smix_next(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z          = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__global__ void source_kernel(double2* f, int n, int stride, int kind, unsigned long long seed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t s = (seed ^ 0x5350494E4F52ULL) ^ ((uint64_t)i * 0x9E3779B97F4A7C15ULL + 0xD1B54A32D192ED03ULL);
    smix_next(s);
    if (kind == 0) {
        const double h      = 1.0 / sqrt(2.0);  // as the host generator computes it
        const uint64_t bits = smix_next(s);
#pragma unroll
        for (int k = 0; k < 12; ++k)
            f[(size_t)k * stride + i] = make_double2(((bits >> (2 * k)) & 1) ? -h : h, ((bits >> (2 * k + 1)) & 1) ? -h : h);
    } else {
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const double u1 = ((smix_next(s) >> 11) + 1) * (1.0 / 9007199254740992.0);
            const double u2 = ((smix_next(s) >> 11) + 1) * (1.0 / 9007199254740992.0);
            const double r  = sqrt(-2.0 * log(u1));
            double sn, cs;
            sincos(6.283185307179586 * u2, &sn, &cs);
            f[(size_t)k * stride + i] = make_double2(r * cs, r * sn);
        }
    }
}

C2Q_EXPORT int c2q_spinor_eo_source(c2q_spinor_eo* f, int kind, unsigned long long seed)
{
    if (!f || (kind != 0 && kind != 1)) return C2Q_BAD_ARG;
    if (f->prec != 64) return fail(f->ctx, C2Q_BAD_ARG, "sources are generated into FP64 fields");
    source_kernel<<<(f->geom.seo + 255) / 256, 256, 0, f->ctx->stream>>>((double2*)f->data, f->geom.seo,
                                                                          f->geom.stride, kind, seed);
    f->ctx->launches++;
    C2Q_CUDA(f->ctx, cudaGetLastError());
    return C2Q_OK;
}

// Pseudoscalar correlator from point sources
// (ocl_kernel/fermionobservables/correlator_ps_point.cl: correlator_ps_t,
// correlator_ps_z): along t, C(t) = (2 kappa)^2 / NS^3 * sum over the solutions
// and the sites of time slice t of |phi|^2; along z, C(z) = (2 kappa)^2 /
// (NS^2 NT) * the same sum over the sites with that z.  The eo index runs with
// t slowest and x fastest, so in each parity the sites of time slice t are the
// range [t NS^3/2, (t+1) NS^3/2) and those of a z slice are, for every t, the
// range of NS^2/2 indices starting at (NS^2 z + NS^3 t)/2.  One block per
// slice sums in a fixed order: deterministic.
constexpr int CORR_THREADS = 256;
__global__ void correlator_ps_kernel(const double2* const* fields, int nfields, int dir, Geom g, double factor,
                                     double* out)
{
    const int s      = blockIdx.x;  // slice coordinate
    const int plane  = g.ns * g.ns / 2;
    const int nsites = dir == 0 ? g.vs_h : plane * g.nt;
    double acc[1]    = {0.0};
    for (int f = 0; f < nfields; ++f) {
        const double2* p = fields[f];
        for (int i = threadIdx.x; i < nsites; i += blockDim.x) {
            const int site = dir == 0 ? s * g.vs_h + i : (i / plane) * g.vs_h + s * plane + (i % plane);
#pragma unroll
            for (int k = 0; k < 12; ++k) {
                const double2 v = p[(size_t)k * g.stride + site];
                acc[0] += v.x * v.x + v.y * v.y;
            }
        }
    }
    __shared__ double smem[32];
    block_sum<1>(acc, smem);
    if (threadIdx.x == 0) out[s] = factor * acc[0];
}

C2Q_EXPORT int c2q_correlator_ps(const c2q_spinor_eo* const* even, const c2q_spinor_eo* const* odd, int n,
                                 double kappa, int direction, double* out)
{
    if (!even || !odd || n < 1 || !out || !even[0] || (direction != 0 && direction != 3)) return C2Q_BAD_ARG;
    c2q_ctx* ctx  = even[0]->ctx;
    const Geom& g = even[0]->geom;
    std::vector<const double2*> ptrs;
    for (int k = 0; k < n; ++k) {
        for (const c2q_spinor_eo* f : {even[k], odd[k]}) {
            if (!f || f->prec != 64 || f->ctx != ctx || !same_lattice(f->lat, even[0]->lat))
                return fail(ctx, C2Q_BAD_ARG, "correlator fields must be FP64 fields of one context and lattice");
            ptrs.push_back(static_cast<const double2*>(f->data));
        }
    }
    const int nslices   = direction == 0 ? g.nt : g.ns;
    const size_t pbytes = ptrs.size() * sizeof(void*);
    const size_t obytes = (size_t)nslices * sizeof(double);
    int rc              = ensure_staging(ctx, ((pbytes + 15) / 16) * 16 + obytes);
    if (rc) return rc;
    char* stage = static_cast<char*>(ctx->staging);
    C2Q_CUDA(ctx, cudaMemcpyAsync(stage, ptrs.data(), pbytes, cudaMemcpyHostToDevice, ctx->stream));
    const double k2     = 2.0 * kappa * 2.0 * kappa;
    const double factor = direction == 0 ? k2 / ((double)g.ns * g.ns * g.ns) : k2 / ((double)g.ns * g.ns * g.nt);
    double* dout        = reinterpret_cast<double*>(stage + ((pbytes + 15) / 16) * 16);
    correlator_ps_kernel<<<nslices, CORR_THREADS, 0, ctx->stream>>>(reinterpret_cast<const double2* const*>(stage),
                                                                    (int)ptrs.size(), direction, g, factor, dout);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    C2Q_CUDA(ctx, cudaMemcpyAsync(out, dout, obytes, cudaMemcpyDeviceToHost, ctx->stream));
    // the pointer array (host vector) must stay alive until the copy has been consumed
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

// every component 1/sqrt(12 V) real (ocl_kernel/spinorfield_eo_cold.cl:22-33)
__global__ void cold_kernel(double2* f, int n, int stride, double v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int k = 0; k < 12; ++k) f[(size_t)k * stride + i] = make_double2(v, 0.0);
}

C2Q_EXPORT int c2q_spinor_eo_cold(c2q_spinor_eo* f)
{
    if (!f || f->prec != 64) return C2Q_BAD_ARG;
    const double v = 1. / std::sqrt(12. * (double)(2 * (size_t)f->geom.seo));
    cold_kernel<<<(f->geom.seo + 255) / 256, 256, 0, f->ctx->stream>>>((double2*)f->data, f->geom.seo,
                                                                        f->geom.stride, v);
    f->ctx->launches++;
    C2Q_CUDA(f->ctx, cudaGetLastError());
    return C2Q_OK;
}

C2Q_EXPORT int c2q_convert_to_eoprec(c2q_spinor_eo* even, c2q_spinor_eo* odd, const double* full)
{
    if (!even || !odd || !full || even->prec != 64 || odd->prec != 64) return C2Q_BAD_ARG;
    c2q_ctx* ctx       = even->ctx;
    const size_t bytes = (size_t)even->geom.seo * 2 * 24 * sizeof(double);
    int rc             = ensure_staging(ctx, bytes);
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaMemcpyAsync(ctx->staging, full, bytes, cudaMemcpyHostToDevice, ctx->stream));
    rc = aos_transfer(even, nullptr, nullptr, 1, 0, (const double*)ctx->staging);
    if (!rc) rc = aos_transfer(odd, nullptr, nullptr, 1, 1, (const double*)ctx->staging);
    if (rc) return rc;
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

C2Q_EXPORT int c2q_convert_from_eoprec(double* full, const c2q_spinor_eo* even, const c2q_spinor_eo* odd)
{
    if (!even || !odd || !full || even->prec != 64 || odd->prec != 64) return C2Q_BAD_ARG;
    c2q_ctx* ctx       = even->ctx;
    const size_t bytes = (size_t)even->geom.seo * 2 * 24 * sizeof(double);
    int rc             = ensure_staging(ctx, bytes);
    if (rc) return rc;
    for (int par = 0; par < 2; ++par) {
        const c2q_spinor_eo* f = par == 0 ? even : odd;
        AosArgs A;
        A.aos    = static_cast<double*>(ctx->staging);
        A.soa    = static_cast<double2*>(f->data);
        A.n      = f->geom.seo;
        A.stride = f->geom.stride;
        A.mode   = 1;
        A.par    = par;
        A.ns     = f->geom.ns;
        A.nsh    = f->geom.nsh;
        soa_to_aos_kernel<<<(A.n + 255) / 256, 256, 0, ctx->stream>>>(A);
        ctx->launches++;
        C2Q_CUDA(ctx, cudaGetLastError());
    }
    C2Q_CUDA(ctx, cudaMemcpyAsync(full, ctx->staging, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    C2Q_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return C2Q_OK;
}

// ---------------------------------------------------------------- explicit ops
C2Q_EXPORT int c2q_dslash_eo(c2q_spinor_eo* out, const c2q_gauge* g, const c2q_spinor_eo* in, int evenodd,
                             double kappa)
{
    if (!out || !g || !in) return C2Q_BAD_ARG;
    if (evenodd != C2Q_EVEN && evenodd != C2Q_ODD) return fail(out->ctx, C2Q_BAD_ARG, "evenodd must be EVEN or ODD");
    return launch_dslash(out->ctx, g, gkind_for(out->prec, out->ctx->rec12), out, in, evenodd == C2Q_ODD ? 0 : 1,
                         kappa, EPI_PLAIN,
                         EpiArgs{1, 0, 1, 0, 0}, nullptr, DotSpec{});
}

C2Q_EXPORT int c2q_dslash_AND_M_tm_inverse_sitediagonal_eo(c2q_spinor_eo* out, const c2q_gauge* g,
                                                           const c2q_spinor_eo* in, int evenodd, double kappa,
                                                           double mubar, int minus)
{
    if (!out || !g || !in) return C2Q_BAD_ARG;
    if (evenodd != C2Q_EVEN && evenodd != C2Q_ODD) return fail(out->ctx, C2Q_BAD_ARG, "evenodd must be EVEN or ODD");
    return launch_dslash(out->ctx, g, gkind_for(out->prec, out->ctx->rec12), out, in, evenodd == C2Q_ODD ? 0 : 1,
                         kappa, EPI_DIAG,
                         diag_epi(mubar, minus ? C2Q_DIAG_M_TM_INVERSE_MINUS : C2Q_DIAG_M_TM_INVERSE, 0), nullptr,
                         DotSpec{});
}

C2Q_EXPORT int c2q_tm_sitediagonal(c2q_spinor_eo* out, const c2q_spinor_eo* in, double mubar, int which)
{
    if (!out || !in || which < 0 || which > 5) return C2Q_BAD_ARG;
    const EpiArgs e = diag_epi(mubar, which, 0);
    BlasSpec s;
    s.op  = B_DIAG;
    s.out = out;
    s.x   = in;
    s.a   = coef_host(e.f1re, e.f1im);
    s.b   = coef_host(e.f2re, e.f2im);
    return launch_blas(out->ctx, s);
}

C2Q_EXPORT int c2q_gamma5_eo(c2q_spinor_eo* inout)
{
    if (!inout) return C2Q_BAD_ARG;
    BlasSpec s;
    s.op  = B_GAMMA5;
    s.out = inout;
    s.x   = inout;
    return launch_blas(inout->ctx, s);
}

C2Q_EXPORT int c2q_apply_eo(int op, c2q_spinor_eo* out, const c2q_gauge* g, const c2q_spinor_eo* in, double kappa,
                            double mubar, int action, int merged)
{
    (void)merged;  // the fused sweeps give identical results with and without kernel merging
    if (!out || !g || !in) return C2Q_BAD_ARG;
    c2q_ctx* ctx = out->ctx;
    c2q_spinor_eo t1, t2;
    int rc = field_alloc(ctx, out->lat, out->prec, &t1);
    if (rc) return rc;
    rc = field_alloc(ctx, out->lat, out->prec, &t2);
    if (!rc)
        rc = apply_operator(ctx, op, out, g, gkind_for(out->prec, ctx->rec12), in, kappa, mubar, action, &t1, &t2,
                            DotSpec{}, nullptr);
    field_free(&t1);
    field_free(&t2);
    return rc;
}

// Full-lattice (non-eo) operators on a field held as its two parities
// (physics/fermionmatrix/fermionmatrix.cpp:41-222, explicit.cpp:36-87;
// ocl_kernel/fermionmatrix_m_tm_plus.cl): M_tm_plus / minus = (1 +/- i mubar g5)
// - kappa D (for the Wilson action 1 - kappa D), Qplus / Qminus = g5 M_tm_plus /
// minus, QplusQminus = Qplus Qminus.  Each parity of the output is one fused
// sweep: the EPI_AXPY epilogue forms f x - h, so the sweep runs with -kappa to
// give f x - kappa D x.
static int full_sweeps(c2q_spinor_eo* oe, c2q_spinor_eo* oo, const c2q_gauge* g, const c2q_spinor_eo* ie,
                       const c2q_spinor_eo* io, double kappa, double mubar, int action, int minus, int g5)
{
    c2q_ctx* ctx  = oe->ctx;
    const int gk  = gkind_for(oe->prec, ctx->rec12);
    EpiArgs e     = action == C2Q_ACTION_TWISTEDMASS ? diag_epi(mubar, minus ? C2Q_DIAG_M_TM_MINUS : C2Q_DIAG_M_TM, g5)
                                                      : EpiArgs{1, 0, 1, 0, g5};
    int rc = launch_dslash(ctx, g, gk, oe, io, /*even sites*/ 0, -kappa, EPI_AXPY, e, ie, DotSpec{});
    if (!rc) rc = launch_dslash(ctx, g, gk, oo, ie, /*odd sites*/ 1, -kappa, EPI_AXPY, e, io, DotSpec{});
    return rc;
}

C2Q_EXPORT int c2q_apply_full(int op, c2q_spinor_eo* out_even, c2q_spinor_eo* out_odd, const c2q_gauge* g,
                              const c2q_spinor_eo* in_even, const c2q_spinor_eo* in_odd, double kappa, double mubar,
                              int action)
{
    if (!out_even || !out_odd || !g || !in_even || !in_odd) return C2Q_BAD_ARG;
    c2q_ctx* ctx = out_even->ctx;
    if (action != C2Q_ACTION_WILSON && action != C2Q_ACTION_TWISTEDMASS)
        return fail(ctx, C2Q_BAD_ARG, "unknown fermion action (wilson or twistedmass)");
    for (const c2q_spinor_eo* o : {(const c2q_spinor_eo*)out_even, (const c2q_spinor_eo*)out_odd})
        if (o == in_even || o == in_odd) return fail(ctx, C2Q_BAD_ARG, "operator output must not alias its input");
    switch (op) {
        case C2Q_FULL_M_TM_PLUS: return full_sweeps(out_even, out_odd, g, in_even, in_odd, kappa, mubar, action, 0, 0);
        case C2Q_FULL_M_TM_MINUS: return full_sweeps(out_even, out_odd, g, in_even, in_odd, kappa, mubar, action, 1, 0);
        case C2Q_FULL_QPLUS: return full_sweeps(out_even, out_odd, g, in_even, in_odd, kappa, mubar, action, 0, 1);
        case C2Q_FULL_QMINUS: return full_sweeps(out_even, out_odd, g, in_even, in_odd, kappa, mubar, action, 1, 1);
        case C2Q_FULL_QPLUSQMINUS: {
            c2q_spinor_eo te, to;
            int rc = field_alloc(ctx, out_even->lat, out_even->prec, &te);
            if (rc) return rc;
            rc = field_alloc(ctx, out_even->lat, out_even->prec, &to);
            if (!rc) rc = full_sweeps(&te, &to, g, in_even, in_odd, kappa, mubar, action, 1, 1);
            if (!rc) rc = full_sweeps(out_even, out_odd, g, &te, &to, kappa, mubar, action, 0, 1);
            field_free(&te);
            field_free(&to);
            return rc;
        }
        default: return fail(ctx, C2Q_BAD_ARG, "unknown full-lattice fermion matrix");
    }
}

// ---------------------------------------------------------------- BLAS
static int blas_simple(int op, c2q_spinor_eo* out, double are, double aim, const c2q_spinor_eo* x,
                       double bre, double bim, const c2q_spinor_eo* y, const c2q_spinor_eo* z)
{
    if (!out || !x) return C2Q_BAD_ARG;
    BlasSpec s;
    s.op  = op;
    s.out = out;
    s.x   = x;
    s.y   = y;
    s.z   = z;
    s.a   = coef_host(are, aim);
    s.b   = coef_host(bre, bim);
    return launch_blas(out->ctx, s);
}

C2Q_EXPORT int c2q_saxpy(c2q_spinor_eo* out, double are, double aim, const c2q_spinor_eo* x, const c2q_spinor_eo* y)
{
    if (!y) return C2Q_BAD_ARG;
    return blas_simple(B_SAXPY, out, are, aim, x, 0, 0, y, nullptr);
}
C2Q_EXPORT int c2q_saxpy_AND_gamma5_eo(c2q_spinor_eo* out, double are, double aim, const c2q_spinor_eo* x,
                                       const c2q_spinor_eo* y)
{
    if (!y) return C2Q_BAD_ARG;
    return blas_simple(B_SAXPY_G5, out, are, aim, x, 0, 0, y, nullptr);
}
C2Q_EXPORT int c2q_sax(c2q_spinor_eo* out, double are, double aim, const c2q_spinor_eo* x)
{
    return blas_simple(B_SAX, out, are, aim, x, 0, 0, nullptr, nullptr);
}
C2Q_EXPORT int c2q_saxsbypz(c2q_spinor_eo* out, double are, double aim, const c2q_spinor_eo* x, double bre,
                            double bim, const c2q_spinor_eo* y, const c2q_spinor_eo* z)
{
    if (!y || !z) return C2Q_BAD_ARG;
    return blas_simple(B_SAXSBYPZ, out, are, aim, x, bre, bim, y, z);
}
C2Q_EXPORT int c2q_copyData(c2q_spinor_eo* to, const c2q_spinor_eo* from)
{
    return blas_simple(B_COPY, to, 0, 0, from, 0, 0, nullptr, nullptr);
}

C2Q_EXPORT int c2q_scalar_product(const c2q_spinor_eo* x, const c2q_spinor_eo* y, double* re, double* im)
{
    if (!x || !y || !re || !im) return C2Q_BAD_ARG;
    c2q_ctx* ctx = x->ctx;
    BlasSpec s;
    s.x   = x;
    s.y   = y;
    s.dot = 1;
    int rc = launch_blas(ctx, s);
    if (rc) return rc;
    double h[2];
    rc = read_scalars(ctx, ctx->red_result, 2, h);
    *re = h[0];
    *im = h[1];
    return rc;
}

C2Q_EXPORT int c2q_squarenorm(const c2q_spinor_eo* x, double* result)
{
    if (!x || !result) return C2Q_BAD_ARG;
    c2q_ctx* ctx = x->ctx;
    BlasSpec s;
    s.x   = x;
    s.y   = x;
    s.dot = 1;
    int rc = launch_blas(ctx, s);
    if (rc) return rc;
    double h[2];
    rc      = read_scalars(ctx, ctx->red_result, 2, h);
    *result = h[0];
    return rc;
}

C2Q_EXPORT int c2q_saxpy_AND_squarenorm(c2q_spinor_eo* out, double are, double aim, const c2q_spinor_eo* x,
                                        const c2q_spinor_eo* y, double* squarenorm)
{
    if (!out || !x || !y || !squarenorm) return C2Q_BAD_ARG;
    c2q_ctx* ctx = out->ctx;
    BlasSpec s;
    s.op  = B_SAXPY;
    s.out = out;
    s.x   = x;
    s.y   = y;
    s.a   = coef_host(are, aim);
    s.dot = 2;
    int rc = launch_blas(ctx, s);
    if (rc) return rc;
    double h[2];
    rc          = read_scalars(ctx, ctx->red_result, 2, h);
    *squarenorm = h[0];
    return rc;
}

}  // extern "C"
