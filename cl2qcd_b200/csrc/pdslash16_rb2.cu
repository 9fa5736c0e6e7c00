// pdslash16_rb2.cu -- instantiations of the two-sources-per-thread FP16 sweep
// (pdslash2.cuh) for the temporal-gauge sweeps of the batched mixed-precision CG.
#include "pdslash2.cuh"

namespace c2q {

template <int NL, int EPI, int DOT>
static void pk2_go(const PkParams<16>& prm, int blocks, cudaStream_t s)
{
    constexpr size_t smem = Pk2Stage<NL>::BYTES;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        cudaFuncSetAttribute(pdslash2_kernel<NL, EPI, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set[dev] = true;
    }
    launch_dep(prm.pdl != 0, pdslash2_kernel<NL, EPI, DOT>, dim3(blocks), dim3(PK_THREADS), smem, s, prm);
}

template <int NL>
static bool pk2_dispatch_nl(const PkParams<16>& prm, int epi, int dot, int blocks, cudaStream_t s)
{
    switch (dot == DOT_CGR ? 9 : dot == DOT_XUPD ? 10 + epi : epi * 3 + dot) {
        case 0: pk2_go<NL, EPI_PLAIN, DOT_NONE>(prm, blocks, s); return true;
        case 3: pk2_go<NL, EPI_DIAG, DOT_NONE>(prm, blocks, s); return true;
        case 6: pk2_go<NL, EPI_AXPY, DOT_NONE>(prm, blocks, s); return true;
        case 8: pk2_go<NL, EPI_AXPY, DOT_SELF>(prm, blocks, s); return true;
        case 9: pk2_go<NL, EPI_AXPY, DOT_CGR>(prm, blocks, s); return true;
        case 10: pk2_go<NL, EPI_PLAIN, DOT_XUPD>(prm, blocks, s); return true;
        case 11: pk2_go<NL, EPI_DIAG, DOT_XUPD>(prm, blocks, s); return true;
    }
    return false;
}

// Launches the sweep for prm.nrhs (even) right-hand sides, two per thread;
// false if the shape has no instantiation here.
bool pk2_dispatch(const PkParams<16>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s)
{
    return nl == 6 ? pk2_dispatch_nl<6>(prm, epi, dot, blocks, s) : pk2_dispatch_nl<9>(prm, epi, dot, blocks, s);
}

}  // namespace c2q
