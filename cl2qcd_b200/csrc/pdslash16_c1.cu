// pdslash16_c1.cu -- instantiations of the paired-site dslash for FP16
// fixed-point fields (12-real and 18-real FP16 links), launch configuration 1.
#include "pdslash_inst.cuh"

namespace c2q {

void pk_dispatch16_c1(const PkParams<16>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s)
{
    if (nl == 6)
        pk_dispatch_nl<16, 6, 1>(prm, epi, dot, blocks, s);
    else
        pk_dispatch_nl<16, 9, 1>(prm, epi, dot, blocks, s);
}

}  // namespace c2q
