// dslash.cuh -- the even-odd Wilson hopping term with fused twisted-mass
// epilogues, for one output parity, one thread per output site.
//
// Computes, at every site x of the output parity,
//   h(x) = sum_mu [ c_mu^+ (1 - g_mu) U_mu(x) psi(x+mu)
//                  + c_mu^- (1 + g_mu) U_mu(x-mu)^dagger psi(x-mu) ]
// with c^{+/-} = -kappa e^{+/- i theta pi / N} (times the chemical-potential
// factors on T links), which is the reference's dslash_eo
// (ocl_kernel/fermionmatrix_eo.cl:30-253, fermionmatrix_eo_dslash.cl:28-58),
// then applies one of the epilogues of c2q_internal.cuh:
//   EPI_PLAIN  dslash_eo
//   EPI_DIAG   dslash_AND_M_tm_inverse_sitediagonal(_minus)_eo
//              (fermionmatrix_eo_dslash_AND_M_tm_inverse_sitediagonal.cl:30-62)
//   EPI_AXPY   the tail of Aee / Aee_AND_gamma5_eo: [g5](M_diag(x) - h)
//              (physics/fermionmatrix/fermionmatrix.cpp:250-258, :330-338)
// and optionally reduces <y, out> (DOT_Y) or |out|^2 (DOT_SELF) across the
// grid with the deterministic last-block scheme of reduce.cuh.
//
// Spin projection: each 1 -/+ g_mu has rank two.  For upper spin rows a = 0, 1
// the half spinor is h_a = psi_a + c psi_p, c -> -c for 1 + g_mu; the lower
// row p receives conj(c) * (U h_a).  Forward (p, c) pairs, read off
// fermionmatrix_eo.cl:56-136:  T (2,1)(3,1)  X (3,i)(2,i)  Y (3,1)(2,-1)
// Z (2,i)(3,-i).  Multiplications by +-1, +-i are exact sign/swap operations.
#pragma once

#include "c2q_internal.cuh"
#include "reduce.cuh"

namespace c2q {

template <int P>
struct DslashParams {
    SpinorPtr<P> out;
    SpinorPtr<P> in;   // opposite-parity input field
    SpinorPtr<P> x;    // EPI_AXPY: same-parity field multiplied by M_diag
    SpinorPtr<P> y;    // DOT_Y partner (same parity as out)
    const void* gauge; // [parity][mu][lane][stride]
    Geom g;
    HopCoef c;
    EpiArgs e;
    int out_parity;    // parity of the output sites: 0 = (x+y+z+t) even
    RedArgs red;
};

// multiply by c in {1, -1, i, -i}, encoded as K = 0, 1, 2, 3
template <int K, typename R>
__device__ __forceinline__ Cplx<R> mul_unit(Cplx<R> v)
{
    if (K == 0) return v;
    if (K == 1) return {-v.re, -v.im};
    if (K == 2) return {-v.im, v.re};
    return {v.im, -v.re};
}
// conj of the unit K
template <int K>
struct ConjUnit {
    static constexpr int value = K == 2 ? 3 : (K == 3 ? 2 : K);
};
template <int K>
struct NegUnit {
    static constexpr int value = K == 0 ? 1 : K == 1 ? 0 : K == 2 ? 3 : 2;
};

// forward projector table
template <int MU>
struct Proj;
template <>
struct Proj<0> {  // T
    static constexpr int p0 = 2, c0 = 0, p1 = 3, c1 = 0;
};
template <>
struct Proj<1> {  // X
    static constexpr int p0 = 3, c0 = 2, p1 = 2, c1 = 2;
};
template <>
struct Proj<2> {  // Y
    static constexpr int p0 = 3, c0 = 0, p1 = 2, c1 = 1;
};
template <>
struct Proj<3> {  // Z
    static constexpr int p0 = 2, c0 = 2, p1 = 3, c1 = 3;
};

// One half-spinor channel: acc_a += k U h, acc_p += conj(c) k U h, h = psi_a + c psi_p.
template <typename R, int A, int PP, int CK, bool DAG>
__device__ __forceinline__ void hop_channel(Cplx<R> acc[12], const Cplx<R> psi[12], const Cplx<R> u[9], Cplx<R> k)
{
    Cplx<R> h[3];
#pragma unroll
    for (int col = 0; col < 3; ++col) h[col] = psi[3 * A + col] + mul_unit<CK>(psi[3 * PP + col]);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        Cplx<R> s;
        if (!DAG) {
            s = cmul(u[3 * r + 0], h[0]);
            s = s + cmul(u[3 * r + 1], h[1]);
            s = s + cmul(u[3 * r + 2], h[2]);
        } else {
            s = cmulc(u[0 * 3 + r], h[0]);
            s = s + cmulc(u[1 * 3 + r], h[1]);
            s = s + cmulc(u[2 * 3 + r], h[2]);
        }
        const Cplx<R> w = cmul(s, k);
        acc[3 * A + r]  = acc[3 * A + r] + w;
        acc[3 * PP + r] = acc[3 * PP + r] + mul_unit<ConjUnit<CK>::value>(w);
    }
}

template <typename R, int MU, bool BACK>
__device__ __forceinline__ void hop(Cplx<R> acc[12], const Cplx<R> psi[12], const Cplx<R> u[9], Cplx<R> k)
{
    using T         = Proj<MU>;
    constexpr int c0 = BACK ? NegUnit<T::c0>::value : T::c0;
    constexpr int c1 = BACK ? NegUnit<T::c1>::value : T::c1;
    hop_channel<R, 0, T::p0, c0, BACK>(acc, psi, u, k);
    hop_channel<R, 1, T::p1, c1, BACK>(acc, psi, u, k);
}

template <int P, int NL, int MU>
__device__ __forceinline__ void do_direction(Cplx<typename Prec<P>::R> acc[12], const DslashParams<P>& prm,
                                             int i_fwd, int i_bwd, int i_site)
{
    using R                 = typename Prec<P>::R;
    const Geom& g           = prm.g;
    const size_t ls         = (size_t)g.stride;
    const int po            = prm.out_parity;
    // element size of one complex lane entry in this precision
    constexpr size_t esz    = P == 64 ? 16 : (P == 32 ? 8 : 4);
    const char* gbase       = static_cast<const char*>(prm.gauge);
    const char* fwd_links   = gbase + (size_t)((po * 4 + MU) * NL) * ls * esz;
    const char* bwd_links   = gbase + (size_t)(((1 - po) * 4 + MU) * NL) * ls * esz;

    Cplx<R> psi[12], u[9];
    // forward: U_mu(x) psi(x+mu)
    SpinorIO<P>::load(prm.in, g.stride, i_fwd, psi);
    LinkIO<P, NL>::load(fwd_links, ls, (size_t)i_site, u);
    if (NL == 6) reconstruct_row2(u);
    hop<R, MU, false>(acc, psi, u, cmk<R>((R)prm.c.re[MU][0], (R)prm.c.im[MU][0]));
    // backward: U_mu(x-mu)^dagger psi(x-mu)
    SpinorIO<P>::load(prm.in, g.stride, i_bwd, psi);
    LinkIO<P, NL>::load(bwd_links, ls, (size_t)i_bwd, u);
    if (NL == 6) reconstruct_row2(u);
    hop<R, MU, true>(acc, psi, u, cmk<R>((R)prm.c.re[MU][1], (R)prm.c.im[MU][1]));
}

template <int P, int NL, int EPI, int DOT>
__global__ void __launch_bounds__(128) dslash_kernel(const DslashParams<P> prm)
{
    using R       = typename Prec<P>::R;
    const Geom& g = prm.g;
    const int i   = blockIdx.x * blockDim.x + threadIdx.x;
    double dv[2]  = {0.0, 0.0};

    if (i < g.seo) {
        // coordinates of the output site carrying eo index i
        int rest     = i / g.nsh;
        const int xh = i - rest * g.nsh;
        const int y  = rest % g.ns;
        rest /= g.ns;
        const int z  = rest % g.ns;
        const int t  = rest / g.ns;
        const int x  = 2 * xh + ((prm.out_parity + y + z + t) & 1);
        const int yzt = g.nsh * (y + g.ns * (z + g.ns * t));

        Cplx<R> acc[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) acc[k] = cmk<R>(0, 0);

        {  // T
            const int tp = t + 1 == g.nt ? 0 : t + 1, tm = t == 0 ? g.nt - 1 : t - 1;
            const int base = xh + g.nsh * (y + g.ns * z);
            do_direction<P, NL, 0>(acc, prm, base + g.vs_h * tp, base + g.vs_h * tm, i);
        }
        {  // X
            const int xp = x + 1 == g.ns ? 0 : x + 1, xm = x == 0 ? g.ns - 1 : x - 1;
            do_direction<P, NL, 1>(acc, prm, (xp >> 1) + yzt, (xm >> 1) + yzt, i);
        }
        {  // Y
            const int yp = y + 1 == g.ns ? 0 : y + 1, ym = y == 0 ? g.ns - 1 : y - 1;
            const int zt = g.ns * (z + g.ns * t);
            do_direction<P, NL, 2>(acc, prm, xh + g.nsh * (yp + zt), xh + g.nsh * (ym + zt), i);
        }
        {  // Z
            const int zp = z + 1 == g.ns ? 0 : z + 1, zm = z == 0 ? g.ns - 1 : z - 1;
            do_direction<P, NL, 3>(acc, prm, xh + g.nsh * (y + g.ns * (zp + g.ns * t)),
                                   xh + g.nsh * (y + g.ns * (zm + g.ns * t)), i);
        }

        if (EPI == EPI_DIAG) {
            const Cplx<R> f1 = cmk<R>((R)prm.e.f1re, (R)prm.e.f1im), f2 = cmk<R>((R)prm.e.f2re, (R)prm.e.f2im);
#pragma unroll
            for (int k = 0; k < 12; ++k) acc[k] = cmul(k < 6 ? f1 : f2, acc[k]);
        } else if (EPI == EPI_AXPY) {
            Cplx<R> xv[12];
            SpinorIO<P>::load(prm.x, g.stride, i, xv);
            const Cplx<R> f1 = cmk<R>((R)prm.e.f1re, (R)prm.e.f1im), f2 = cmk<R>((R)prm.e.f2re, (R)prm.e.f2im);
#pragma unroll
            for (int k = 0; k < 12; ++k) {
                Cplx<R> r = cmul(k < 6 ? f1 : f2, xv[k]) - acc[k];
                if (prm.e.gamma5 && k >= 6) r = cmk<R>(-r.re, -r.im);
                acc[k] = r;
            }
        }
        SpinorIO<P>::store(prm.out, g.stride, i, acc);

        if (DOT == DOT_Y) {
            Cplx<R> yv[12];
            SpinorIO<P>::load(prm.y, g.stride, i, yv);
#pragma unroll
            for (int k = 0; k < 12; ++k) {
                const Cplx<R> p = cmulc(yv[k], acc[k]);
                dv[0] += (double)p.re;
                dv[1] += (double)p.im;
            }
        } else if (DOT == DOT_SELF) {
#pragma unroll
            for (int k = 0; k < 12; ++k) dv[0] += (double)acc[k].re * acc[k].re + (double)acc[k].im * acc[k].im;
        }
    }
    if (DOT != DOT_NONE) {
        __shared__ double smem[2 * 32];
        block_sum<2>(dv, smem);
        finish_reduction<2>(dv, prm.red, smem);
    }
}

}  // namespace c2q
