// pdslash32_c0.cu -- instantiations of the paired-site dslash for FP32 fields
// (18-real and 12-real FP32 links), launch configuration 0.
#include "pdslash_inst.cuh"

namespace c2q {

void pk_dispatch32_c0(const PkParams<32>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s)
{
    if (nl == 6)
        pk_dispatch_nl<32, 6, 0>(prm, epi, dot, blocks, s);
    else
        pk_dispatch_nl<32, 9, 0>(prm, epi, dot, blocks, s);
}

}  // namespace c2q
