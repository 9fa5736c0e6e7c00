// mixed.cuh -- vector updates of the mixed-precision CG on the paired-site
// slots of pack.cuh: the residual and the solution increment are FP32 fields,
// the search direction and the operator output are FP16 or FP32 (PB).  One
// thread per slot (two sites), packed FP32 arithmetic; a launch covers a batch
// of right-hand sides (block b: right-hand side b % nrhs), each with its own
// solver scalars and its own reduction.
#pragma once

#include "blas.cuh"
#include "pack.cuh"

namespace c2q {

constexpr int MIX_THREADS = 128;

struct MixFields {
    void* x;            // FP32 solution increment
    void* r;            // FP32 residual
    void* p;            // PB search direction
    float* p_norm;
    const void* v;      // PB operator output A p
    const float* v_norm;
    SolverScalars* sc;
};

struct MixArgs {
    MixFields f[PK_MAX_RHS];
    int nrhs;
    int H, ss;
    RedArgs red;
};

// values of a PB field as s = scale * q (FP16: exact integers q and the
// per-site scale; FP32: the values and scale 1)
template <int PB>
__device__ __forceinline__ void mix_load(const void* d, const float* n, int ss, int j, C2 s[12], float2* scale)
{
    if constexpr (PB == 16) {
        SlotF16::load_q(d, n, ss, j, s, scale);
    } else {
        SlotF32::load(d, ss, j, s);
        *scale = bc2(1.0f);
    }
}
template <int PB>
__device__ __forceinline__ void mix_store(void* d, float* n, int ss, int j, const C2 s[12])
{
    if constexpr (PB == 16)
        SlotF16::store(d, n, ss, j, s);
    else
        SlotF32::store(d, ss, j, s);
}

// a += c b for a complex coefficient c (broadcast pairs cre, cim, -cim)
__device__ __forceinline__ C2 caxpy2(C2 a, float2 cre, float2 cim, float2 ncim, C2 b)
{
    return C2{fma2(b.re, cre, fma2(b.im, ncim, a.re)), fma2(b.im, cre, fma2(b.re, cim, a.im))};
}

// r -= alpha v ; |r|^2 -> FIN_CG_BETA of the right-hand side.  The matching
// solution update x += alpha p is deferred to the next mix_p (which reads p
// anyway) or to the reliable-update accumulation.
template <int PB>
__global__ void __launch_bounds__(MIX_THREADS) mix_update_kernel(const MixArgs A)
{
    pdl_enter();
    const int nrhs     = A.nrhs;
    const int rhs      = nrhs == 1 ? 0 : (int)(blockIdx.x % (unsigned)nrhs);
    const int blk      = nrhs == 1 ? (int)blockIdx.x : (int)(blockIdx.x / (unsigned)nrhs);
    const int j        = blk * MIX_THREADS + threadIdx.x;
    const MixFields& F = A.f[rhs];
    float2 n2          = bc2(0.f);
    if (j < A.H) {
        const float ar = (float)F.sc->alpha[0], ai = (float)F.sc->alpha[1];
        C2 a[12], b[12];
        float2 bs;
        SlotF32::load(F.r, A.ss, j, a);
        mix_load<PB>(F.v, F.v_norm, A.ss, j, b, &bs);
        const float2 cr = mul2(bc2(-ar), bs), ci = mul2(bc2(-ai), bs), nci = mul2(bc2(ai), bs);
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            a[c] = caxpy2(a[c], cr, ci, nci, b[c]);
            n2   = fma2(a[c].re, a[c].re, fma2(a[c].im, a[c].im, n2));
        }
        SlotF32::store(F.r, A.ss, j, a);
    }
    double dv[2] = {(double)n2.x + (double)n2.y, 0.0};
    __shared__ double smem[64];
    block_sum<2>(dv, smem);
    RedArgs ra = A.red;
    ra.sc      = F.sc;
    finish_reduction<2>(dv, ra, smem, rhs, nrhs);
}

// x += alpha p (the previous iteration's deferred update; skipped when x is
// null because a sweep applied it), then p = r + beta p
template <int PB>
__global__ void __launch_bounds__(MIX_THREADS) mix_p_kernel(const MixArgs A)
{
    pdl_enter();
    const int nrhs     = A.nrhs;
    const int rhs      = nrhs == 1 ? 0 : (int)(blockIdx.x % (unsigned)nrhs);
    const int blk      = nrhs == 1 ? (int)blockIdx.x : (int)(blockIdx.x / (unsigned)nrhs);
    const int j        = blk * MIX_THREADS + threadIdx.x;
    const MixFields& F = A.f[rhs];
    if (j >= A.H) return;
    const float ar = (float)F.sc->alpha[0], ai = (float)F.sc->alpha[1];
    const float br = (float)F.sc->beta[0], bi = (float)F.sc->beta[1];
    C2 p[12], r[12];
    float2 ps;
    mix_load<PB>(F.p, F.p_norm, A.ss, j, p, &ps);
    if (F.x) {
        SlotF32::load(F.x, A.ss, j, r);
        const float2 cr = mul2(bc2(ar), ps), ci = mul2(bc2(ai), ps), nci = mul2(bc2(-ai), ps);
#pragma unroll
        for (int c = 0; c < 12; ++c) r[c] = caxpy2(r[c], cr, ci, nci, p[c]);
        SlotF32::store(F.x, A.ss, j, r);
    }
    SlotF32::load(F.r, A.ss, j, r);
    const float2 cr = mul2(bc2(br), ps), ci = mul2(bc2(bi), ps), nci = mul2(bc2(-bi), ps);
#pragma unroll
    for (int c = 0; c < 12; ++c) p[c] = caxpy2(r[c], cr, ci, nci, p[c]);
    mix_store<PB>(F.p, F.p_norm, A.ss, j, p);
}

// x64 = x64 + (double) (x_s + alpha p) ; x_s = 0   (reliable update
// accumulation in FP64, including the deferred update of the last iteration;
// `sc` null: x_s only)
template <int PB>
__global__ void __launch_bounds__(BLAS_THREADS) accumulate_kernel(SpinorPtr<64> x, SpinorPtr<32> xs, SpinorPtr<PB> p,
                                                                  const SolverScalars* sc, int n, int stride)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Cplx<double> a[12];
    Cplx<float> b[12];
    SpinorIO<64>::load(x, stride, i, a);
    SpinorIO<32>::load(xs, stride, i, b);
    if (sc) {
        Cplx<float> q[12];
        SpinorIO<PB>::load(p, stride, i, q);
        const Cplx<float> al = cmk<float>((float)sc->alpha[0], (float)sc->alpha[1]);
#pragma unroll
        for (int k = 0; k < 12; ++k) b[k] = b[k] + cmul(al, q[k]);
    }
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        a[k] = a[k] + cmk<double>((double)b[k].re, (double)b[k].im);
        b[k] = cmk<float>(0.f, 0.f);
    }
    SpinorIO<64>::store(x, stride, i, a);
    SpinorIO<32>::store(xs, stride, i, b);
}

}  // namespace c2q
