// pdslash2.cuh -- the FP16 paired-site sweep of pdslash.cuh with two
// right-hand sides per thread, for batches of the mixed-precision CG's inner
// solves (fields in the temporal gauge, phase pattern PH_TG).
//
// A batch of right-hand sides shares every link.  The one-source-per-thread
// kernel reads each link from HBM once per batch (the blocks of one slot tile
// run side by side and share it through L2), but every source's thread still
// stages the link and decodes it (FP16 dequantisation and, for 12-real links,
// the row-2 reconstruction: about a quarter of the instructions of a hop).
// Here one thread computes one slot of two sources: per hop it stages the two
// neighbour spinors and the link once, decodes the link once into registers and
// applies it to both spinors, accumulating into two sets of accumulators.
//
// Each source's arithmetic is the same instruction sequence as in the
// one-source kernel (same staged values, same decoded link, same epilogue and
// per-tile reduction tree over the same 128 slots), so a source gives bitwise
// the same result here, in the one-source kernel, and alone.
//
// The ring holds per stage the two neighbour spinors (7 chunks each) and the
// link; the epilogue operands (the EPI_AXPY operand, the DOT_Y partner, the
// search direction of DOT_XUPD) of both sources are staged as the two last hops
// run; the FP32 residual / solution increment of DOT_CGR / DOT_XUPD is
// prefetched into L2 instead and read directly.
#pragma once

#include "pdslash.cuh"

namespace c2q {

template <int NL>
struct Pk2Stage {
    static constexpr int SPC      = PkChunks<16, NL>::SPC;  // 7: six word chunks and the norm pair
    static constexpr int LKC      = PkChunks<16, NL>::LKC;
    static constexpr int CH       = 2 * SPC + LKC;
    static constexpr int STAGES   = NL == 6 ? 3 : 2;        // two blocks of 128 threads per SM either way
    static constexpr int MINB     = 2;
    static constexpr size_t BYTES = (size_t)STAGES * CH * 16 * PK_THREADS;
};

__device__ __forceinline__ void prefetch_l2(const void* p)
{
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

// The epilogue of one source (the code of pdslash_kernel's epilogue, with the
// source's staged operands at s8 / s9 and its FP32 update field read directly).
template <int EPI, int DOT>
__device__ __forceinline__ void pk2_epilogue(C2 acc[12], const PkParams<16>& prm, const PkRhs& rr, const uint4* s8,
                                             const uint4* s9, int ss, int j, float2& dre, float2& dim, float2& dq)
{
    const float sc = (float)prm.c.scale;
    if (EPI == EPI_PLAIN) {
#pragma unroll
        for (int c = 0; c < 12; ++c) acc[c] = C2{mul2(acc[c].re, bc2(sc)), mul2(acc[c].im, bc2(sc))};
    } else if (EPI == EPI_DIAG) {
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const float fr = (float)(c < 6 ? prm.e.f1re : prm.e.f2re) * sc;
            const float fi = (float)(c < 6 ? prm.e.f1im : prm.e.f2im) * sc;
            const C2 a     = acc[c];
            acc[c]         = C2{fma2(a.re, bc2(fr), mul2(a.im, bc2(-fi))), fma2(a.im, bc2(fr), mul2(a.re, bc2(fi)))};
        }
    } else if (EPI == EPI_AXPY) {
        C2 xv[12];
        float2 xs;
        staged_operand<16>(s8, xv, &xs);
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const float gs  = (prm.e.gamma5 && c >= 6) ? -1.0f : 1.0f;
            const float2 fr = mul2(bc2(gs * (float)(c < 6 ? prm.e.f1re : prm.e.f2re)), xs);
            const float2 fi = mul2(bc2(gs * (float)(c < 6 ? prm.e.f1im : prm.e.f2im)), xs);
            const float2 nf = mul2(bc2(-gs * (float)(c < 6 ? prm.e.f1im : prm.e.f2im)), xs);
            const float ms  = -gs * sc;
            const C2 a      = acc[c];
            acc[c]          = C2{fma2(a.re, bc2(ms), fma2(xv[c].re, fr, mul2(xv[c].im, nf))),
                        fma2(a.im, bc2(ms), fma2(xv[c].im, fr, mul2(xv[c].re, fi)))};
        }
    }
    if (DOT != DOT_CGR) SlotF16::store(rr.out, rr.out_norm, ss, j, acc);

    if (DOT == DOT_CGR) {  // r -= alpha out (r FP32, passed as y), |r|^2
        const float ar = (float)rr.sc->alpha[0], ai = (float)rr.sc->alpha[1];
        float4* rw     = static_cast<float4*>(const_cast<void*>(rr.y));
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            C2 r       = c2_from(rw[(size_t)c * ss + j], false);
            const C2 v = acc[c];
            r.re       = fma2(v.re, bc2(-ar), fma2(v.im, bc2(ai), r.re));
            r.im       = fma2(v.im, bc2(-ar), fma2(v.re, bc2(-ai), r.im));
            __stcs(rw + (size_t)c * ss + j, c2_to(r));
            dre        = fma2(r.re, r.re, fma2(r.im, r.im, dre));
        }
    } else if (DOT == DOT_Y) {
        C2 yv[12];
        float2 ys;
        staged_operand<16>(s9, yv, &ys);
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            dre = fma2(yv[c].re, acc[c].re, fma2(yv[c].im, acc[c].im, dre));
            dim = fma2(yv[c].re, acc[c].im, dim);
            dq  = fma2(yv[c].im, acc[c].re, dq);
        }
        dre = mul2(dre, ys);
        dim = mul2(dim, ys);
        dq  = mul2(dq, ys);
    } else if (DOT == DOT_SELF) {
#pragma unroll
        for (int c = 0; c < 12; ++c) dre = fma2(acc[c].re, acc[c].re, fma2(acc[c].im, acc[c].im, dre));
    } else if (DOT == DOT_XUPD) {  // x += alpha p (x FP32, passed as y; p passed as x and staged)
        const float ar = (float)rr.sc->alpha[0], ai = (float)rr.sc->alpha[1];
        float4* xw     = static_cast<float4*>(const_cast<void*>(rr.y));
        C2 pv[12];
        float2 ps;
        staged_operand<16>(s8, pv, &ps);
        const float2 cr = mul2(bc2(ar), ps), ci = mul2(bc2(ai), ps), nci = mul2(bc2(-ai), ps);
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            C2 xv = c2_from(xw[(size_t)c * ss + j], false);
            xv.re = fma2(pv[c].re, cr, fma2(pv[c].im, nci, xv.re));
            xv.im = fma2(pv[c].im, cr, fma2(pv[c].re, ci, xv.im));
            __stcs(xw + (size_t)c * ss + j, c2_to(xv));
        }
    }
}

template <int NL, int EPI, int DOT>
__global__ void __launch_bounds__(PK_THREADS, Pk2Stage<NL>::MINB) pdslash2_kernel(const PkParams<16> prm)
{
    using S = Pk2Stage<NL>;
    static_assert(DOT != DOT_XUPD || EPI != EPI_AXPY, "the solution update shares the EPI_AXPY operand slot");
    constexpr bool RED = DOT != DOT_NONE && DOT != DOT_XUPD;
    constexpr int T    = PK_THREADS;
    pdl_enter();
    if (halted(prm.red)) return;  // a stopped device-driven solve: every block leaves
    extern __shared__ uint4 ring[];
    uint4* mine     = ring + threadIdx.x;
    const PkGeom& g = prm.g;
    const int npair = prm.nrhs / 2;
    const int pair  = npair == 1 ? 0 : (int)(blockIdx.x % (unsigned)npair);
    const int blk   = npair == 1 ? (int)blockIdx.x : (int)(blockIdx.x / (unsigned)npair);
    const int G     = (int)gridDim.x / npair;  // blocks per pair of right-hand sides
    const PkRhs& r0 = prm.r[2 * pair];
    const PkRhs& r1 = prm.r[2 * pair + 1];
    __shared__ double smem[2 * 32];

    for (int tile = blk; tile < prm.ntiles; tile += G) {
    const int j = tile * T + threadIdx.x;
    float2 dre[2] = {bc2(0.f), bc2(0.f)}, dim[2] = {bc2(0.f), bc2(0.f)}, dq[2] = {bc2(0.f), bc2(0.f)};

    if (j < g.H) {
        const unsigned q1 = fdiv((unsigned)j, g.div_nsh);
        const int xh      = j - (int)q1 * g.nsh;
        const unsigned q2 = fdiv(q1, g.div_ns);
        const int y       = (int)q1 - (int)q2 * g.ns;
        const int t       = (int)fdiv(q2, g.div_ns);
        const int z       = (int)q2 - t * g.ns;
        const int x       = 2 * xh + ((prm.out_parity + y + z + t) & 1);
        const int yzt     = j - xh;
        const int ss      = g.ss;

        const int po          = prm.out_parity;
        const size_t grp      = (size_t)pk_link_bytes<16, NL>() * ss;
        const char* gb        = static_cast<const char*>(prm.gauge);
        const char* fwd_links = gb + (size_t)(po * 4) * grp;
        const char* bwd_links = gb + (size_t)((1 - po) * 4) * grp;

        const bool fold_f = t + 1 == g.nt2, fold_b = t == 0;
        const int base    = j - g.vs_h * t;
        int nb[8];
        nb[0]         = fold_f ? base : j + g.vs_h;
        nb[1]         = fold_b ? base + g.vs_h * (g.nt2 - 1) : j - g.vs_h;
        const int xp  = x + 1 == g.ns ? 0 : x + 1, xm = x == 0 ? g.ns - 1 : x - 1;
        nb[2]         = (xp >> 1) + yzt;
        nb[3]         = (xm >> 1) + yzt;
        const int row = g.nsh, pl = g.nsh * g.ns;
        nb[4]         = y + 1 == g.ns ? j - (g.ns - 1) * row : j + row;
        nb[5]         = y == 0 ? j + (g.ns - 1) * row : j - row;
        nb[6]         = z + 1 == g.ns ? j - (g.ns - 1) * pl : j + pl;
        nb[7]         = z == 0 ? j + (g.ns - 1) * pl : j - pl;

        // stage q: hops 0..7 (two neighbour spinors, one link), then the
        // epilogue operands of both sources (q = 8: x / p, q = 9: y)
        auto issue = [&](auto qc) {
            constexpr int q = decltype(qc)::value;
            uint4* st       = mine + (size_t)((q % S::STAGES) * S::CH) * T;
            if constexpr (q < 8) {
                constexpr bool back = q & 1;
                stage_spinor<16>(st, r0.in, r0.in_norm, ss, nb[q]);
                stage_spinor<16>(st + S::SPC * T, r1.in, r1.in_norm, ss, nb[q]);
                // temporal gauge: the T links between inner slices are the identity
                if (q >= 2 || (back ? fold_b : fold_f))
                    stage_link<16, NL>(st + S::SPC * T, (back ? bwd_links : fwd_links) + (size_t)(q >> 1) * grp, ss,
                                       back ? nb[q] : j);
            } else if constexpr (q == 8) {
                if (EPI == EPI_AXPY || DOT == DOT_XUPD) {
                    stage_spinor<16>(st, r0.x, r0.x_norm, ss, j);
                    stage_spinor<16>(st + S::SPC * T, r1.x, r1.x_norm, ss, j);
                }
                if (DOT == DOT_CGR || DOT == DOT_XUPD) {
                    const float4* a = static_cast<const float4*>(r0.y) + j;
                    const float4* b = static_cast<const float4*>(r1.y) + j;
#pragma unroll
                    for (int c = 0; c < 12; ++c) {
                        prefetch_l2(a + (size_t)c * ss);
                        prefetch_l2(b + (size_t)c * ss);
                    }
                }
            } else {
                if (DOT == DOT_Y) {
                    stage_spinor<16>(st, r0.y, r0.y_norm, ss, j);
                    stage_spinor<16>(st + S::SPC * T, r1.y, r1.y_norm, ss, j);
                }
            }
            cp_commit();
        };

        C2 acc0[12], acc1[12];
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            acc0[c] = C2{bc2(0.f), bc2(0.f)};
            acc1[c] = C2{bc2(0.f), bc2(0.f)};
        }

        auto step = [&](auto hc) {
            constexpr int h = decltype(hc)::value;
            if constexpr (h + S::STAGES - 1 <= 9)
                issue(std::integral_constant<int, h + S::STAGES - 1>{});
            else
                cp_commit();
            cp_wait<S::STAGES - 1>();
            const uint4* st0    = mine + (size_t)((h % S::STAGES) * S::CH) * T;
            const uint4* st1    = st0 + S::SPC * T;
            const uint4* lk     = st0 + 2 * S::SPC * T;
            constexpr int mu    = h >> 1;
            constexpr bool back = h & 1;
            if constexpr (mu == 0) {
                if (back ? fold_b : fold_f) {
                    // across the last time slice: the stored link W with the weight
                    // lambda (forward) or conj(lambda) (backward) on one lane, the
                    // identity with weight 1 on the other (as pk_hop_tg_fold)
                    const float lr = (float)prm.lam_re, li = (float)prm.lam_im;
                    const Kc w     = back ? Kc{make_float2(lr, 1.0f), make_float2(-li, 0.0f), make_float2(-lr, -1.0f),
                                           make_float2(li, 0.0f)}
                                          : Kc{make_float2(1.0f, lr), make_float2(0.0f, li), make_float2(-1.0f, -lr),
                                           make_float2(0.0f, -li)};
                    C2 u[9];
                    staged_link<16, NL, back>(lk, u);
                    pk_hop_spinor<16, 0, back, true, false>(acc0, st0, u, w);
                    pk_hop_spinor<16, 0, back, true, false>(acc1, st1, u, w);
                } else {
                    pk_hop_id<16, back>(acc0, st0, 1.0f);
                    pk_hop_id<16, back>(acc1, st1, 1.0f);
                }
            } else {
                const Kc w = uniform_weight(prm.c.re[mu][back ? 1 : 0], prm.c.im[mu][back ? 1 : 0]);
                C2 u[9];
                staged_link<16, NL, false>(lk, u);
                pk_hop_spinor<16, mu, back, false, true>(acc0, st0, u, w);
                pk_hop_spinor<16, mu, back, false, true>(acc1, st1, u, w);
            }
        };
        issue(std::integral_constant<int, 0>{});
        if constexpr (S::STAGES > 2) issue(std::integral_constant<int, 1>{});
        step(std::integral_constant<int, 0>{});
        step(std::integral_constant<int, 1>{});
        step(std::integral_constant<int, 2>{});
        step(std::integral_constant<int, 3>{});
        step(std::integral_constant<int, 4>{});
        step(std::integral_constant<int, 5>{});
        step(std::integral_constant<int, 6>{});
        step(std::integral_constant<int, 7>{});
        if constexpr (S::STAGES == 2) issue(std::integral_constant<int, 9>{});
        cp_wait<0>();

        const uint4* s8 = mine + (size_t)((8 % S::STAGES) * S::CH) * T;
        const uint4* s9 = mine + (size_t)((9 % S::STAGES) * S::CH) * T;
        pk2_epilogue<EPI, DOT>(acc0, prm, r0, s8, s9, ss, j, dre[0], dim[0], dq[0]);
        pk2_epilogue<EPI, DOT>(acc1, prm, r1, s8 + S::SPC * T, s9 + S::SPC * T, ss, j, dre[1], dim[1], dq[1]);
    }
    if (RED) {  // one partial per tile and source, in tile order
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            double dv[2] = {(double)dre[r].x + (double)dre[r].y,
                            ((double)dim[r].x - (double)dq[r].x) + ((double)dim[r].y - (double)dq[r].y)};
            block_sum<2>(dv, smem);
            store_partial<2>(dv, prm.red, (size_t)tile * prm.nrhs + 2 * pair + r);
        }
    }
    }  // tiles
    if (RED) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const PkRhs& rr = r ? r1 : r0;
            RedArgs ra      = prm.red;
            if (rr.sc) ra.sc = rr.sc;
            if (rr.result) ra.result = rr.result;
            if (r) __syncthreads();  // every thread has read the first group's flag before it is set again
            finish_group<2, PK_FINISH_ROUND>(ra, smem, 2 * pair + r, prm.nrhs, prm.ntiles, G);
        }
    }
}

}  // namespace c2q
