// pdslash_inst.cuh -- compile-time dispatch of the paired-site dslash kernel
// over epilogue, fused reduction and phase pattern; included once per storage
// precision (pdslash32.cu, pdslash16.cu) so the instantiations compile in parallel.
#pragma once

#include "pdslash.cuh"

namespace c2q {

// Launch one instantiation with its shared-memory ring (the opt-in above
// 48 KB is set once per device and instantiation).
template <int P, int NL, int EPI, int DOT, int PH, int CFG>
static void pk_go(const PkParams<P>& prm, int blocks, cudaStream_t s)
{
    constexpr size_t smem = PkStage<P, NL, CFG>::BYTES;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        cudaFuncSetAttribute(pdslash_kernel<P, NL, EPI, DOT, PH, CFG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        attr_set[dev] = true;
    }
    launch_dep(prm.pdl != 0, pdslash_kernel<P, NL, EPI, DOT, PH, CFG>, dim3(blocks), dim3(PK_THREADS), smem, s, prm);
}

template <int P, int NL, int PH, int CFG>
static void pk_dispatch_ph(const PkParams<P>& prm, int epi, int dot, int blocks, cudaStream_t s)
{
    // (epilogue, reduction): 3 x 3 combinations, the CG residual update after
    // EPI_AXPY and the CG solution update after EPI_PLAIN / EPI_DIAG
    switch (dot == DOT_CGR ? 9 : dot == DOT_XUPD ? 10 + epi : epi * 3 + dot) {
        case 0: pk_go<P, NL, EPI_PLAIN, DOT_NONE, PH, CFG>(prm, blocks, s); break;
        case 1: pk_go<P, NL, EPI_PLAIN, DOT_Y, PH, CFG>(prm, blocks, s); break;
        case 2: pk_go<P, NL, EPI_PLAIN, DOT_SELF, PH, CFG>(prm, blocks, s); break;
        case 3: pk_go<P, NL, EPI_DIAG, DOT_NONE, PH, CFG>(prm, blocks, s); break;
        case 4: pk_go<P, NL, EPI_DIAG, DOT_Y, PH, CFG>(prm, blocks, s); break;
        case 5: pk_go<P, NL, EPI_DIAG, DOT_SELF, PH, CFG>(prm, blocks, s); break;
        case 6: pk_go<P, NL, EPI_AXPY, DOT_NONE, PH, CFG>(prm, blocks, s); break;
        case 7: pk_go<P, NL, EPI_AXPY, DOT_Y, PH, CFG>(prm, blocks, s); break;
        case 8: pk_go<P, NL, EPI_AXPY, DOT_SELF, PH, CFG>(prm, blocks, s); break;
        case 9: pk_go<P, NL, EPI_AXPY, DOT_CGR, PH, CFG>(prm, blocks, s); break;
        case 10: pk_go<P, NL, EPI_PLAIN, DOT_XUPD, PH, CFG>(prm, blocks, s); break;
        case 11: pk_go<P, NL, EPI_DIAG, DOT_XUPD, PH, CFG>(prm, blocks, s); break;
    }
}

// Temporal gauge: the sweeps of the mixed-precision CG on QplusQminus_eo
// (twisted mass and Wilson) only.
template <int P, int NL, int CFG>
static void pk_dispatch_tg(const PkParams<P>& prm, int epi, int dot, int blocks, cudaStream_t s)
{
    switch (dot == DOT_CGR ? 9 : dot == DOT_XUPD ? 10 + epi : epi * 3 + dot) {
        case 0: pk_go<P, NL, EPI_PLAIN, DOT_NONE, PH_TG, CFG>(prm, blocks, s); break;
        case 3: pk_go<P, NL, EPI_DIAG, DOT_NONE, PH_TG, CFG>(prm, blocks, s); break;
        case 6: pk_go<P, NL, EPI_AXPY, DOT_NONE, PH_TG, CFG>(prm, blocks, s); break;
        case 8: pk_go<P, NL, EPI_AXPY, DOT_SELF, PH_TG, CFG>(prm, blocks, s); break;
        case 9: pk_go<P, NL, EPI_AXPY, DOT_CGR, PH_TG, CFG>(prm, blocks, s); break;
        case 10: pk_go<P, NL, EPI_PLAIN, DOT_XUPD, PH_TG, CFG>(prm, blocks, s); break;
        case 11: pk_go<P, NL, EPI_DIAG, DOT_XUPD, PH_TG, CFG>(prm, blocks, s); break;
    }
}
// Phase pattern from HopCoef::real_mask: all real, only T complex, or general.
template <int P, int NL, int CFG>
static void pk_dispatch_nl(const PkParams<P>& prm, int epi, int dot, int blocks, cudaStream_t s)
{
    const unsigned m = prm.c.real_mask;
    if (prm.tg)
        pk_dispatch_tg<P, NL, CFG>(prm, epi, dot, blocks, s);
    else if (m == 0xFFu)
        pk_dispatch_ph<P, NL, PH_REAL, CFG>(prm, epi, dot, blocks, s);
    else if ((m & 0xFCu) == 0xFCu)
        pk_dispatch_ph<P, NL, PH_TCPLX, CFG>(prm, epi, dot, blocks, s);
    else
        pk_dispatch_ph<P, NL, PH_ANY, CFG>(prm, epi, dot, blocks, s);
}

}  // namespace c2q
