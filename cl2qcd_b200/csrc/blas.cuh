// blas.cuh -- eo spinor-field level-1 BLAS, fused CG updates, reductions and
// layout conversions, one thread per eo site, any storage precision.
//
// Semantics follow the reference's eo BLAS (physics/lattices/spinorfield_eo.cpp
// and ocl_kernel/spinorfield_eo_*.cl), including its sign convention
//   saxpy(out, a, x, y) = y - a x         (spinorfield_eo_saxpy.cl:20-37)
//   saxsbypz(out, a, x, b, y, z) = a x + b y + z (spinorfield_eo_saxsbypz.cl:22-43)
//   scalar_product(x, y) = sum conj(x) y  (operations_su3vec.cl:40-48)
// Coefficients come either from the host or from device scalars, so solver
// iterations never wait on the host.
#pragma once

#include "c2q_internal.cuh"
#include "reduce.cuh"

namespace c2q {

constexpr int BLAS_THREADS = 256;

// A complex coefficient: sgn * (dev ? (dev[0], dev[1]) : (re, im)).
struct Coef {
    double re, im;
    const double* dev;
    double sgn;
};
__host__ __device__ inline Coef coef_host(double re, double im) { return Coef{re, im, nullptr, 1.0}; }
__host__ __device__ inline Coef coef_dev(const double* p, double sgn = 1.0) { return Coef{0.0, 0.0, p, sgn}; }
__device__ __forceinline__ Cplx<double> coef_value(const Coef& c)
{
    if (c.dev) return cmk(c.sgn * c.dev[0], c.sgn * c.dev[1]);
    return cmk(c.sgn * c.re, c.sgn * c.im);
}

enum BlasOp : int {
    B_SAXPY = 0,        // out = y - a x
    B_SAXPY_G5,         // out = g5 (y - a x)
    B_SAX,              // out = a x
    B_SAXSBYPZ,         // out = a x + b y + z
    B_COPY,             // out = x
    B_GAMMA5,           // out = g5 x
    B_DIAG,             // out = diag(f1, f2) x   (a = f1, b = f2)
    B_BICG_XR,          // BiCGStab: out = a x + b y + out, out2 = y - b z, with |out2|^2 and
                        // <w, out2> (dot 4)
};

// Field arguments of one BLAS launch; any may be unused.
template <int P>
struct BlasArgs {
    SpinorPtr<P> out, x, y, z;
    SpinorPtr<P> w, out2;  // B_BICG_XR only
    Coef a, b;
    int n, stride;
    int op;
    int dot;          // 0 none, 1 <x,y> (conj(x) y, no output write), 2 |out|^2,
                      // 3 <x,y> and <x,x> in one pass (no output write),
                      // 4 (B_BICG_XR) |out2|^2 and <w, out2>
    RedArgs red;
};

template <int P>
__global__ void __launch_bounds__(BLAS_THREADS) blas_kernel(const BlasArgs<P> A)
{
    pdl_enter();
    if (halted(A.red)) return;  // a stopped device-driven solve: every block leaves
    using R      = typename Prec<P>::R;
    const int i  = blockIdx.x * blockDim.x + threadIdx.x;
    double dv[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < A.n && A.op == B_BICG_XR) {
        // bicgstab.cpp:694-702: x = alpha p + omega s + x; rn = s - omega t;
        // then |rn|^2 and (rhat, rn)
        const Cplx<double> a = coef_value(A.a), b = coef_value(A.b);
        const Cplx<R> ar = cmk<R>((R)a.re, (R)a.im), br = cmk<R>((R)b.re, (R)b.im);
        Cplx<R> xv[12], yv[12], r[12];
        SpinorIO<P>::load(A.x, A.stride, i, xv);
        SpinorIO<P>::load(A.y, A.stride, i, yv);
        SpinorIO<P>::load(A.out, A.stride, i, r);
#pragma unroll
        for (int k = 0; k < 12; ++k) r[k] = (cmul(yv[k], br) + cmul(xv[k], ar)) + r[k];
        SpinorIO<P>::store(A.out, A.stride, i, r);
        SpinorIO<P>::load(A.z, A.stride, i, xv);
#pragma unroll
        for (int k = 0; k < 12; ++k) r[k] = yv[k] - cmul(xv[k], br);
        SpinorIO<P>::store(A.out2, A.stride, i, r);
        // (the reductions use the values computed here: a load of what this kernel
        // just stored could come through the non-coherent read-only path stale)
        SpinorIO<P>::load(A.w, A.stride, i, yv);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            dv[0] += (double)r[k].re * r[k].re + (double)r[k].im * r[k].im;
            const Cplx<R> p = cmulc(yv[k], r[k]);
            dv[2] += (double)p.re;
            dv[3] += (double)p.im;
        }
    } else if (i < A.n) {
        Cplx<R> xv[12], r[12];
        if (A.dot == 1 || A.dot == 3) {
            Cplx<R> yv[12];
            SpinorIO<P>::load(A.x, A.stride, i, xv);
            SpinorIO<P>::load(A.y, A.stride, i, yv);
#pragma unroll
            for (int k = 0; k < 12; ++k) {
                Cplx<R> p = cmulc(xv[k], yv[k]);
                dv[0] += (double)p.re;
                dv[1] += (double)p.im;
                if (A.dot == 3) {  // <x,x>: its imaginary part is rounding only
                    Cplx<R> q = cmulc(xv[k], xv[k]);
                    dv[2] += (double)q.re;
                    dv[3] += (double)q.im;
                }
            }
        } else {
            const Cplx<double> a = coef_value(A.a), b = coef_value(A.b);
            const Cplx<R> ar = cmk<R>((R)a.re, (R)a.im), br = cmk<R>((R)b.re, (R)b.im);
            SpinorIO<P>::load(A.x, A.stride, i, xv);
            switch (A.op) {
                case B_SAXPY:
                case B_SAXPY_G5: {
                    Cplx<R> yv[12];
                    SpinorIO<P>::load(A.y, A.stride, i, yv);
#pragma unroll
                    for (int k = 0; k < 12; ++k) {
                        r[k] = yv[k] - cmul(xv[k], ar);
                        if (A.op == B_SAXPY_G5 && k >= 6) r[k] = cmk<R>(-r[k].re, -r[k].im);
                    }
                    break;
                }
                case B_SAX:
#pragma unroll
                    for (int k = 0; k < 12; ++k) r[k] = cmul(xv[k], ar);
                    break;
                case B_SAXSBYPZ: {
                    Cplx<R> yv[12], zv[12];
                    SpinorIO<P>::load(A.y, A.stride, i, yv);
                    SpinorIO<P>::load(A.z, A.stride, i, zv);
#pragma unroll
                    for (int k = 0; k < 12; ++k) r[k] = (cmul(yv[k], br) + cmul(xv[k], ar)) + zv[k];
                    break;
                }
                case B_COPY:
#pragma unroll
                    for (int k = 0; k < 12; ++k) r[k] = xv[k];
                    break;
                case B_GAMMA5:
#pragma unroll
                    for (int k = 0; k < 12; ++k) r[k] = k >= 6 ? cmk<R>(-xv[k].re, -xv[k].im) : xv[k];
                    break;
                case B_DIAG:
#pragma unroll
                    for (int k = 0; k < 12; ++k) r[k] = cmul(k < 6 ? ar : br, xv[k]);
                    break;
            }
            SpinorIO<P>::store(A.out, A.stride, i, r);
            if (A.dot == 2)
#pragma unroll
                for (int k = 0; k < 12; ++k) dv[0] += (double)r[k].re * r[k].re + (double)r[k].im * r[k].im;
        }
    }
    if (A.dot == 3 || A.dot == 4) {
        __shared__ double smem4[128];
        block_sum<4>(dv, smem4);
        finish_reduction<4>(dv, A.red, smem4);
    } else if (A.dot) {
        __shared__ double smem[64];
        block_sum<2>(dv, smem);
        finish_reduction<2>(dv, A.red, smem);
    }
}

// CG update (cg.cpp:335-347): x = x - tmp1 p with tmp1 = -alpha, r = r - alpha v,
// and |r|^2 reduced into the solver scalars (FIN_CG_BETA).
template <int P>
struct CgUpdateArgs {
    SpinorPtr<P> x, r, p, v;
    const SolverScalars* sc;
    int n, stride;
    RedArgs red;
};

template <int P>
__global__ void __launch_bounds__(BLAS_THREADS) cg_update_kernel(const CgUpdateArgs<P> A)
{
    pdl_enter();
    using R      = typename Prec<P>::R;
    const int i  = blockIdx.x * blockDim.x + threadIdx.x;
    double dv[2] = {0.0, 0.0};
    if (i < A.n) {
        const Cplx<R> al = cmk<R>((R)A.sc->alpha[0], (R)A.sc->alpha[1]);
        const Cplx<R> ma = cmk<R>(-al.re, -al.im);
        Cplx<R> a[12], b[12];
        SpinorIO<P>::load(A.x, A.stride, i, a);
        SpinorIO<P>::load(A.p, A.stride, i, b);
#pragma unroll
        for (int k = 0; k < 12; ++k) a[k] = a[k] - cmul(b[k], ma);
        SpinorIO<P>::store(A.x, A.stride, i, a);
        SpinorIO<P>::load(A.r, A.stride, i, a);
        SpinorIO<P>::load(A.v, A.stride, i, b);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            a[k] = a[k] - cmul(b[k], al);
            dv[0] += (double)a[k].re * a[k].re + (double)a[k].im * a[k].im;
        }
        SpinorIO<P>::store(A.r, A.stride, i, a);
    }
    __shared__ double smem[64];
    block_sum<2>(dv, smem);
    finish_reduction<2>(dv, A.red, smem);
}

// p = r - tmp2 p with tmp2 = -beta (cg.cpp:393-395)
template <int P>
struct CgPArgs {
    SpinorPtr<P> p, r;
    const SolverScalars* sc;
    int n, stride;
};
template <int P>
__global__ void __launch_bounds__(BLAS_THREADS) cg_p_kernel(const CgPArgs<P> A)
{
    pdl_enter();
    using R     = typename Prec<P>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const Cplx<R> mb = cmk<R>((R)-A.sc->beta[0], (R)-A.sc->beta[1]);
    Cplx<R> p[12], r[12];
    SpinorIO<P>::load(A.p, A.stride, i, p);
    SpinorIO<P>::load(A.r, A.stride, i, r);
#pragma unroll
    for (int k = 0; k < 12; ++k) p[k] = r[k] - cmul(p[k], mb);
    SpinorIO<P>::store(A.p, A.stride, i, p);
}

// Precision conversion of a whole eo field (same site order and stride).
template <int PO, int PI>
__global__ void __launch_bounds__(BLAS_THREADS) convert_kernel(SpinorPtr<PO> out, SpinorPtr<PI> in, int n, int stride)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Cplx<typename Prec<PI>::R> a[12];
    Cplx<typename Prec<PO>::R> b[12];
    SpinorIO<PI>::load(in, stride, i, a);
#pragma unroll
    for (int k = 0; k < 12; ++k) b[k] = {(typename Prec<PO>::R)a[k].re, (typename Prec<PO>::R)a[k].im};
    SpinorIO<PO>::store(out, stride, i, b);
}

// ---- layout conversion between the reference's AoS host formats and SoA ----
// mode 0: eo AoS array (spinor[Seo]) <-> eo SoA field
// mode 1: full AoS array (spinor[V], site order) <-> the parity-`par` eo SoA field
struct AosArgs {
    double* aos;      // device staging copy of the host array
    double2* soa;     // FP64 SoA field
    int n, stride, mode, par;
    int ns, nsh;
};

__device__ __forceinline__ size_t aos_site(const AosArgs& A, int i)
{
    if (A.mode == 0) return (size_t)i;
    // the parity-par site with eo index i: 2i or 2i+1 (they differ only in x)
    const int s0   = 2 * i;
    int rest       = s0 / A.ns;
    const int x0   = s0 - rest * A.ns;
    int par0       = x0;
    par0 += rest % A.ns;
    rest /= A.ns;
    par0 += rest % A.ns;
    par0 += rest / A.ns;
    return (size_t)(s0 + (((par0 & 1) == A.par) ? 0 : 1));
}

static __global__ void aos_to_soa_kernel(const AosArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const double* src = A.aos + 24 * aos_site(A, i);
#pragma unroll
    for (int k = 0; k < 12; ++k) A.soa[(size_t)k * A.stride + i] = make_double2(src[2 * k], src[2 * k + 1]);
}

static __global__ void soa_to_aos_kernel(const AosArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    double* dst = A.aos + 24 * aos_site(A, i);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        const double2 v = A.soa[(size_t)k * A.stride + i];
        dst[2 * k]      = v.x;
        dst[2 * k + 1]  = v.y;
    }
}

}  // namespace c2q
