// unitarity.cu -- FP64 unitarity measures of an uploaded gauge field and its
// projection onto SU(3), on the device.
//
// The 12-real link storage (FP64, FP32 and FP16) keeps rows 0 and 1 and
// rebuilds row 2 = conj(row0 x row1), which is the field's own row 2 only for
// an SU(3) matrix.  The solvers therefore ask `rec12_exact` before they use
// 12-real FP64 links for a residual: a field whose row 2 differs from the
// rebuilt one by more than 1e-13 (for example links stored in 32-bit ILDG
// precision, unitary to about 1e-7) keeps every FP64 residual on the links as
// uploaded.  c2q_gauge_reunitarize projects such a field onto SU(3) with the
// reference's project_su3 (ocl_kernel/operations_gaugefield.cl:135-240).
#include <cmath>

#include "c2q_host.h"

namespace c2q {

namespace {

constexpr int UNIT_THREADS = 256;

__device__ __forceinline__ Cplx<double> ld(const double2* p, size_t k, size_t stride)
{
    const double2 v = p[k * stride];
    return {v.x, v.y};
}

__device__ __forceinline__ double cabs2(Cplx<double> a) { return a.re * a.re + a.im * a.im; }

// conj(a x b) component-wise: c0 = conj(a1 b2 - a2 b1), c1 = conj(a2 b0 - a0 b2), c2 = conj(a0 b1 - a1 b0)
__device__ __forceinline__ void cross_conj(const Cplx<double> a[3], const Cplx<double> b[3], Cplx<double> c[3])
{
    for (int k = 0; k < 3; ++k) {
        const int i = (k + 1) % 3, j = (k + 2) % 3;
        const Cplx<double> v = cmul(a[i], b[j]) - cmul(a[j], b[i]);
        c[k]                 = {v.re, -v.im};
    }
}

// Non-negative doubles order like their bit patterns: a max over blocks by
// integer atomics (order-independent, so the result is exact and repeatable).
__device__ __forceinline__ unsigned long long max_bits(double v)
{
    if (!(v == v)) v = INFINITY;  // a NaN link reports as infinitely far from SU(3)
    return (unsigned long long)__double_as_longlong(v);
}

// out[0] = max_ij |(U U^dagger - 1)_ij|, out[1] = max |det U - 1|,
// out[2] = max_j |U_2j - conj(row0 x row1)_j|, over the links of the FP64
// 18-real store ([parity][mu][9 lanes][stride]).
__global__ void __launch_bounds__(UNIT_THREADS) unitarity_kernel(const double2* __restrict__ links, Geom g,
                                                                 unsigned long long* __restrict__ out)
{
    double m0 = 0, m1 = 0, m2 = 0;
    const long long n = 8LL * g.seo;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int blk = (int)(t / g.seo), i = (int)(t - (long long)blk * g.seo);
        const double2* p = links + (size_t)blk * 9 * g.stride + i;
        Cplx<double> u[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) u[k] = ld(p, k, g.stride);
        // U U^dagger: (r, s) entry = sum_c u[r][c] conj(u[s][c])
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int s = r; s < 3; ++s) {
                Cplx<double> acc{r == s ? -1.0 : 0.0, 0.0};
#pragma unroll
                for (int c = 0; c < 3; ++c) cmacc(acc, u[3 * s + c], u[3 * r + c]);
                m0 = fmax(m0, sqrt(cabs2(acc)));
            }
        Cplx<double> c2[3];
        cross_conj(u, u + 3, c2);
        // det U = row2 . (row0 x row1) = sum_j u[2][j] conj(c2[j])
        Cplx<double> det{-1.0, 0.0};
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            cmacc(det, c2[j], u[6 + j]);
            m2 = fmax(m2, sqrt(cabs2(u[6 + j] - c2[j])));
        }
        m1 = fmax(m1, sqrt(cabs2(det)));
    }
    // (fmax ignores a NaN operand: nan_scan_kernel reports non-finite links)
    __shared__ double sm[3][UNIT_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    const int w = threadIdx.x / 32;
    if ((threadIdx.x & 31) == 0) {
        sm[0][w] = m0;
        sm[1][w] = m1;
        sm[2][w] = m2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double m = 0;
        for (int k = 0; k < UNIT_THREADS / 32; ++k) m = fmax(m, sm[threadIdx.x][k]);
        atomicMax(out + threadIdx.x, max_bits(m));
    }
}

// Non-finite entries (which fmax would skip) set all three deviations to infinity.
__global__ void __launch_bounds__(UNIT_THREADS) nan_scan_kernel(const double2* __restrict__ links, Geom g,
                                                                unsigned long long* __restrict__ out)
{
    const long long n = 8LL * g.seo;
    bool bad          = false;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int blk = (int)(t / g.seo), i = (int)(t - (long long)blk * g.seo);
        const double2* p = links + (size_t)blk * 9 * g.stride + i;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const double2 v = p[(size_t)k * g.stride];
            bad |= !isfinite(v.x) || !isfinite(v.y);
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0)
        for (int k = 0; k < 3; ++k) atomicMax(out + k, max_bits(INFINITY));
}

// project_su3 (ocl_kernel/operations_gaugefield.cl:135-240) in place: column 0
// normalised, column 1 orthogonalised against it and normalised, column 2 =
// conj(col0 x col1).
__global__ void __launch_bounds__(UNIT_THREADS) project_su3_kernel(double2* __restrict__ links, Geom g)
{
    const long long n = 8LL * g.seo;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int blk = (int)(t / g.seo), i = (int)(t - (long long)blk * g.seo);
        double2* p = links + (size_t)blk * 9 * g.stride + i;
        Cplx<double> a[3], b[3], c[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            a[r] = ld(p, 3 * r, g.stride);
            b[r] = ld(p, 3 * r + 1, g.stride);
        }
        double na = 0;
#pragma unroll
        for (int r = 0; r < 3; ++r) na += cabs2(a[r]);
        na = 1.0 / sqrt(na);
#pragma unroll
        for (int r = 0; r < 3; ++r) a[r] = {a[r].re * na, a[r].im * na};
        Cplx<double> f{0.0, 0.0};  // <a, b> = sum conj(a) b
#pragma unroll
        for (int r = 0; r < 3; ++r) cmacc(f, a[r], b[r]);
#pragma unroll
        for (int r = 0; r < 3; ++r) b[r] = b[r] - cmul(f, a[r]);
        double nb = 0;
#pragma unroll
        for (int r = 0; r < 3; ++r) nb += cabs2(b[r]);
        nb = 1.0 / sqrt(nb);
#pragma unroll
        for (int r = 0; r < 3; ++r) b[r] = {b[r].re * nb, b[r].im * nb};
        cross_conj(a, b, c);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            p[(size_t)(3 * r) * g.stride]     = make_double2(a[r].re, a[r].im);
            p[(size_t)(3 * r + 1) * g.stride] = make_double2(b[r].re, b[r].im);
            p[(size_t)(3 * r + 2) * g.stride] = make_double2(c[r].re, c[r].im);
        }
    }
}

int grid_for(c2q_ctx* ctx, long long n)
{
    const long long want = (n + UNIT_THREADS - 1) / UNIT_THREADS;
    const long long cap  = (long long)(ctx->sm_count > 0 ? ctx->sm_count : 148) * 8;
    return (int)(want < cap ? want : cap);
}

// the three deviations of the FP64 18-real store into host memory
int measure(c2q_gauge* g, double dev[3])
{
    c2q_ctx* ctx = g->ctx;
    if (!g->store[G64].data) return fail(ctx, C2Q_BAD_ARG, "gauge field not uploaded");
    // the context's reduction result slots (stream-ordered, free between reductions)
    unsigned long long* out = reinterpret_cast<unsigned long long*>(ctx->red_result);
    C2Q_CUDA(ctx, cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), ctx->stream));
    const long long n = 8LL * g->geom.seo;
    const double2* links = static_cast<const double2*>(g->store[G64].data);
    unitarity_kernel<<<grid_for(ctx, n), UNIT_THREADS, 0, ctx->stream>>>(links, g->geom, out);
    nan_scan_kernel<<<grid_for(ctx, n), UNIT_THREADS, 0, ctx->stream>>>(links, g->geom, out);
    ctx->launches += 2;
    C2Q_CUDA(ctx, cudaGetLastError());
    int rc = read_scalars(ctx, ctx->red_result, 3, dev);  // the bit patterns are the doubles
    if (rc) return rc;
    g->rec12_dev = dev[2];
    return C2Q_OK;
}

}  // namespace

bool rec12_exact(c2q_gauge* g)
{
    if (g->rec12_dev < 0) {
        double dev[3];
        if (measure(g, dev)) return false;
    }
    return g->rec12_dev <= REC12_EXACT_TOL;
}

}  // namespace c2q

using namespace c2q;

extern "C" {

C2Q_EXPORT int c2q_gauge_unitarity(const c2q_gauge* g, double* dev)
{
    if (!g || !dev) return C2Q_BAD_ARG;
    return measure(const_cast<c2q_gauge*>(g), dev);
}

C2Q_EXPORT int c2q_gauge_reunitarize(c2q_gauge* g, double* dev_before)
{
    if (!g) return C2Q_BAD_ARG;
    c2q_ctx* ctx = g->ctx;
    double dev[3];
    int rc = measure(g, dev);
    if (rc) return rc;
    if (dev_before) *dev_before = dev[0];
    if (!std::isfinite(dev[0])) return fail(ctx, C2Q_BAD_ARG, "gauge field holds non-finite links");
    const long long n = 8LL * g->geom.seo;
    project_su3_kernel<<<grid_for(ctx, n), UNIT_THREADS, 0, ctx->stream>>>(static_cast<double2*>(g->store[G64].data),
                                                                          g->geom);
    ctx->launches++;
    C2Q_CUDA(ctx, cudaGetLastError());
    // every derived copy (lower precisions, 12-real, temporal gauge) is rebuilt on next use
    rc = gauge_drop_derived(g);
    if (rc) return rc;
    g->rec12_dev = -1.0;
    return C2Q_OK;
}

}  // extern "C"
