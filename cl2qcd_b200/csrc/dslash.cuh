// dslash.cuh -- the even-odd Wilson hopping term with fused twisted-mass
// epilogues, for one output parity, one thread per output site, on the FP64
// fields (the FP32 / FP16 fields use the paired-site kernel of pdslash.cuh).
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
    int pdl;           // launched as a dependent launch (launch_dep)
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
// KREAL: k is real (k.im ignored).  Everything is written as FMA chains.
template <typename R, int A, int PP, int CK, bool DAG, bool KREAL>
__device__ __forceinline__ void hop_channel(Cplx<R> acc[12], const Cplx<R> h[3], const Cplx<R> u[9], Cplx<R> k)
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        Cplx<R> s;
        if (!DAG) {
            s = cmul(u[3 * r + 0], h[0]);
            cmac(s, u[3 * r + 1], h[1]);
            cmac(s, u[3 * r + 2], h[2]);
        } else {
            s = cmulc(u[0 * 3 + r], h[0]);
            cmacc(s, u[1 * 3 + r], h[1]);
            cmacc(s, u[2 * 3 + r], h[2]);
        }
        // lower row: acc_p += conj(c) * (k s); conj(c) * s is an exact sign/swap
        const Cplx<R> sp = mul_unit<ConjUnit<CK>::value>(s);
        if (KREAL) {
            acc[3 * A + r].re  = fmad(s.re, k.re, acc[3 * A + r].re);
            acc[3 * A + r].im  = fmad(s.im, k.re, acc[3 * A + r].im);
            acc[3 * PP + r].re = fmad(sp.re, k.re, acc[3 * PP + r].re);
            acc[3 * PP + r].im = fmad(sp.im, k.re, acc[3 * PP + r].im);
        } else {
            cmac(acc[3 * A + r], s, k);
            cmac(acc[3 * PP + r], sp, k);
        }
    }
}

// Projected half spinors of a (decoded) spinor for channel A with partner PP and unit CK.
template <typename R, int A, int PP, int CK>
__device__ __forceinline__ void project(Cplx<R> h[3], const Cplx<R> psi[12])
{
#pragma unroll
    for (int col = 0; col < 3; ++col) h[col] = psi[3 * A + col] + mul_unit<CK>(psi[3 * PP + col]);
}
template <typename R, int MU, bool BACK, bool KREAL>
__device__ __forceinline__ void hop_decoded(Cplx<R> acc[12], const Cplx<R> psi[12], const Cplx<R> u[9], Cplx<R> k)
{
    using T          = Proj<MU>;
    constexpr int c0 = BACK ? NegUnit<T::c0>::value : T::c0;
    constexpr int c1 = BACK ? NegUnit<T::c1>::value : T::c1;
    Cplx<R> h[3];
    project<R, 0, T::p0, c0>(h, psi);
    hop_channel<R, 0, T::p0, c0, BACK, KREAL>(acc, h, u, k);
    project<R, 1, T::p1, c1>(h, psi);
    hop_channel<R, 1, T::p1, c1, BACK, KREAL>(acc, h, u, k);
}

// Phase patterns known at compile time (the common boundary conditions): PH_REAL
// all hop phases real, PH_TCPLX only the T phases complex (antiperiodic time,
// periodic space), PH_ANY decided per launch from HopCoef::real_mask.
// PH_TG (paired-site sweeps only): the field is in the temporal gauge (every T
// link is the identity except the one leaving the last time slice, and the T
// phase sits in the transformation), all hop coefficients are real.
enum PhasePattern : int { PH_REAL = 0, PH_TCPLX = 1, PH_ANY = 2, PH_TG = 3 };

// One hop: load the neighbour spinor and the link, weight by the hop phase.
template <int P, int NL, int MU, bool BACK, int PH>
__device__ __forceinline__ void do_hop(Cplx<typename Prec<P>::R> acc[12], const DslashParams<P>& prm,
                                       const char* links, size_t link_idx, int i_nb)
{
    using R          = typename Prec<P>::R;
    const Geom& g    = prm.g;
    const size_t ls  = (size_t)g.stride;
    const int d      = BACK ? 1 : 0;
    const bool kreal = PH == PH_REAL ? true
                       : PH == PH_TCPLX ? (MU != 0)
                                        : (bool)((prm.c.real_mask >> (2 * MU + d)) & 1u);
    Cplx<R> u[9];
    Cplx<R> psi[12];
    SpinorIO<P>::load(prm.in, g.stride, i_nb, psi);
    LinkIO<P, NL>::load(links, ls, link_idx, u);
    if (NL == 6) reconstruct_row2(u);
    const Cplx<R> k = cmk<R>((R)prm.c.re[MU][d], (R)prm.c.im[MU][d]);
    if (kreal)
        hop_decoded<R, MU, BACK, true>(acc, psi, u, k);
    else
        hop_decoded<R, MU, BACK, false>(acc, psi, u, k);
}

template <int P, int NL, int MU, int PH>
__device__ __forceinline__ void do_direction(Cplx<typename Prec<P>::R> acc[12], const DslashParams<P>& prm,
                                             int i_fwd, int i_bwd, int i_site)
{
    const size_t ls       = (size_t)prm.g.stride;
    const int po          = prm.out_parity;
    constexpr size_t esz  = 16;  // one double2 per complex lane entry
    const char* gbase     = static_cast<const char*>(prm.gauge);
    const char* fwd_links = gbase + (size_t)((po * 4 + MU) * NL) * ls * esz;
    const char* bwd_links = gbase + (size_t)(((1 - po) * 4 + MU) * NL) * ls * esz;
    do_hop<P, NL, MU, false, PH>(acc, prm, fwd_links, (size_t)i_site, i_fwd);  // U_mu(x) psi(x+mu)
    do_hop<P, NL, MU, true, PH>(acc, prm, bwd_links, (size_t)i_bwd, i_bwd);    // U_mu(x-mu)^dagger psi(x-mu)
}

template <int P, int NL, int EPI, int DOT, int PH>
__global__ void __launch_bounds__(128) dslash_kernel(const DslashParams<P> prm)
{
    pdl_enter();
    if (halted(prm.red)) return;  // a stopped device-driven solve: every block leaves
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
            do_direction<P, NL, 0, PH>(acc, prm, base + g.vs_h * tp, base + g.vs_h * tm, i);
        }
        {  // X
            const int xp = x + 1 == g.ns ? 0 : x + 1, xm = x == 0 ? g.ns - 1 : x - 1;
            do_direction<P, NL, 1, PH>(acc, prm, (xp >> 1) + yzt, (xm >> 1) + yzt, i);
        }
        {  // Y
            const int yp = y + 1 == g.ns ? 0 : y + 1, ym = y == 0 ? g.ns - 1 : y - 1;
            const int zt = g.ns * (z + g.ns * t);
            do_direction<P, NL, 2, PH>(acc, prm, xh + g.nsh * (yp + zt), xh + g.nsh * (ym + zt), i);
        }
        {  // Z
            const int zp = z + 1 == g.ns ? 0 : z + 1, zm = z == 0 ? g.ns - 1 : z - 1;
            do_direction<P, NL, 3, PH>(acc, prm, xh + g.nsh * (y + g.ns * (zp + g.ns * t)),
                                   xh + g.nsh * (y + g.ns * (zm + g.ns * t)), i);
        }

        // the hopping sum is h = scale * acc (scale = -kappa, times the link dequantisation scale)
        const R sc = (R)prm.c.scale;
        if (EPI == EPI_PLAIN) {
#pragma unroll
            for (int k = 0; k < 12; ++k) acc[k] = cmk<R>(sc * acc[k].re, sc * acc[k].im);
        } else if (EPI == EPI_DIAG) {
            const Cplx<R> f1 = cmk<R>((R)prm.e.f1re * sc, (R)prm.e.f1im * sc);
            const Cplx<R> f2 = cmk<R>((R)prm.e.f2re * sc, (R)prm.e.f2im * sc);
#pragma unroll
            for (int k = 0; k < 12; ++k) acc[k] = cmul(k < 6 ? f1 : f2, acc[k]);
        } else if (EPI == EPI_AXPY) {
            Cplx<R> xv[12];
            SpinorIO<P>::load(prm.x, g.stride, i, xv);
            const Cplx<R> f1 = cmk<R>((R)prm.e.f1re, (R)prm.e.f1im), f2 = cmk<R>((R)prm.e.f2re, (R)prm.e.f2im);
#pragma unroll
            for (int k = 0; k < 12; ++k) {
                const Cplx<R> m = cmul(k < 6 ? f1 : f2, xv[k]);
                Cplx<R> r       = cmk<R>(m.re - sc * acc[k].re, m.im - sc * acc[k].im);
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
