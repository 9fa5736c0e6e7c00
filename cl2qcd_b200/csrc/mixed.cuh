// mixed.cuh -- vector updates of the mixed-precision CG, where the residual
// and the solution increment (precision PA) and the search direction and
// operator output (precision PB) are stored in different precisions.
#pragma once

#include "blas.cuh"

namespace c2q {

// x_s = x_s + alpha p ; r_s = r_s - alpha v ; |r_s|^2 -> FIN_CG_BETA
template <int PA, int PB>
struct MixUpdateArgs {
    SpinorPtr<PA> x, r;
    SpinorPtr<PB> p, v;
    const SolverScalars* sc;
    int n, stride;
    RedArgs red;
};

template <int PA, int PB>
__global__ void __launch_bounds__(BLAS_THREADS) mix_update_kernel(const MixUpdateArgs<PA, PB> A)
{
    const int i  = blockIdx.x * blockDim.x + threadIdx.x;
    double dv[2] = {0.0, 0.0};
    if (i < A.n) {
        const Cplx<float> al = cmk<float>((float)A.sc->alpha[0], (float)A.sc->alpha[1]);
        Cplx<float> a[12], b[12];
        SpinorIO<PA>::load(A.x, A.stride, i, a);
        SpinorIO<PB>::load(A.p, A.stride, i, b);
#pragma unroll
        for (int k = 0; k < 12; ++k) a[k] = a[k] + cmul(b[k], al);
        SpinorIO<PA>::store(A.x, A.stride, i, a);
        SpinorIO<PA>::load(A.r, A.stride, i, a);
        SpinorIO<PB>::load(A.v, A.stride, i, b);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            a[k] = a[k] - cmul(b[k], al);
            dv[0] += (double)a[k].re * a[k].re + (double)a[k].im * a[k].im;
        }
        SpinorIO<PA>::store(A.r, A.stride, i, a);
    }
    __shared__ double smem[64];
    block_sum<2>(dv, smem);
    finish_reduction<2>(dv, A.red, smem);
}

// p = r_s + beta p
template <int PA, int PB>
struct MixPArgs {
    SpinorPtr<PB> p;
    SpinorPtr<PA> r;
    const SolverScalars* sc;
    int n, stride;
};
template <int PA, int PB>
__global__ void __launch_bounds__(BLAS_THREADS) mix_p_kernel(const MixPArgs<PA, PB> A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const Cplx<float> be = cmk<float>((float)A.sc->beta[0], (float)A.sc->beta[1]);
    Cplx<float> p[12], r[12];
    SpinorIO<PB>::load(A.p, A.stride, i, p);
    SpinorIO<PA>::load(A.r, A.stride, i, r);
#pragma unroll
    for (int k = 0; k < 12; ++k) p[k] = r[k] + cmul(p[k], be);
    SpinorIO<PB>::store(A.p, A.stride, i, p);
}

// x64 = x64 + (double) x_s ; x_s = 0   (reliable update accumulation in FP64)
template <int PA>
__global__ void __launch_bounds__(BLAS_THREADS) accumulate_kernel(SpinorPtr<64> x, SpinorPtr<PA> xs, int n, int stride)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Cplx<double> a[12];
    Cplx<float> b[12];
    SpinorIO<64>::load(x, stride, i, a);
    SpinorIO<PA>::load(xs, stride, i, b);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        a[k] = a[k] + cmk<double>((double)b[k].re, (double)b[k].im);
        b[k] = cmk<float>(0.f, 0.f);
    }
    SpinorIO<64>::store(x, stride, i, a);
    SpinorIO<PA>::store(xs, stride, i, b);
}

}  // namespace c2q
