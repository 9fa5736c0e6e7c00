// pdslash32_c1.cu -- instantiations of the paired-site dslash for FP32 fields
// (18-real and 12-real FP32 links), launch configuration 1.
#include "pdslash_inst.cuh"

namespace c2q {

void pk_dispatch32_c1(const PkParams<32>& prm, int nl, int epi, int dot, int blocks, cudaStream_t s)
{
    if (nl == 6)
        pk_dispatch_nl<32, 6, 1>(prm, epi, dot, blocks, s);
    else
        pk_dispatch_nl<32, 9, 1>(prm, epi, dot, blocks, s);
}

}  // namespace c2q
