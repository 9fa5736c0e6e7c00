// reduce.cuh -- deterministic global reductions fused into the producing kernel.
//
// Every reducing kernel writes one partial per block into a scratch array, in
// block order.  The last block to finish (an atomic ticket, reset by that
// block) sums the partials in a fixed order with a fixed tree, so the result
// is independent of block scheduling and bitwise reproducible for a given
// launch shape.  No floating-point atomics are used anywhere.
//
// The same last block then runs a small scalar "finisher" on the device
// (complex divisions for CG/BiCGStab coefficients), so solver iterations need
// no host round trip.
#pragma once

#include "c2q_internal.cuh"

namespace c2q {

constexpr int RED_THREADS = 256;

// Sum NV doubles across the block; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double v[NV], double* smem /* NV * 32 */)
{
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = lane < nw ? smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            v[k] = t;
        }
    }
    __syncthreads();
}

// Device scalars of the Krylov solvers (complex, as the reference keeps them
// in Scalar<hmc_complex>, physics/algorithms/solvers/cg.cpp:290-302).
struct SolverScalars {
    double omega[2];     // CG: (r,r) of the previous iteration | BiCGStab: omega
    double rho[2];       // CG: (p,Ap)                           | BiCGStab: rho
    double rho_next[2];  // CG: (r,r) new                        | BiCGStab: (rhat, r_new)
    double alpha[2];
    double beta[2];
    double tmp1[2], tmp2[2];
    double resid;        // last |r|^2 written by a reducing kernel
    double aux[2];       // extra reduction slot (BiCGStab (t,t), true residual, ...)
    int flag;            // nonzero: a division by zero / NaN was seen
    int halt;            // BiCGStab: nonzero stops every later predicated launch (HALT_*)
    int halt_next;       // BiCGStab: the next iteration's opening test, moved into halt at its start
    int pad_;
    double thr;          // BiCGStab: stopping threshold on |r|^2
};

// Why a device-driven BiCGStab stopped (SolverScalars::halt bits).
enum HaltBits : int {
    HALT_STUCK     = 1,   // (rhat, r_new) vanished: SolverStuck in this iteration
    HALT_NAN       = 2,   // |r|^2 is NaN at this iteration's test
    HALT_CONV      = 4,   // |r|^2 < thr at this iteration's test
    HALT_NAN_NEXT  = 8,   // the same two tests, due at the top of the next iteration
    HALT_CONV_NEXT = 16,
};

// What the last block does with the reduced value(s).
enum Finisher : int {
    FIN_STORE_RESULT = 0,  // result[0..NV) = sum
    FIN_CG_ALPHA     = 1,  // rho = sum; alpha = omega / rho
    FIN_CG_BETA      = 2,  // rho_next = (sum,0); resid = sum; beta = rho_next/omega; omega = rho_next
    FIN_CG_OMEGA     = 3,  // omega = (sum,0) ; resid = sum  (refresh iteration, (r,r))
    // BiCGStab, physics/algorithms/solvers/bicgstab.cpp:566-733 (fast) and :401-564 (save)
    FIN_BI_REFRESH = 4,  // <rhat,rn>, <rhat,rhat>: rho; resid; the iteration's opening test
    FIN_BI_ALPHA   = 5,  // tmp1 = (rhat, v); alpha = rho / tmp1
    FIN_BI_OMEGA   = 6,  // <t,s>, <t,t>: tmp1, tmp2; omega = tmp1 / tmp2
    FIN_BI_RESID   = 7,  // resid = |rn|^2 (fin_arg: apply the stopping test now -- save)
    FIN_BI_BETA    = 8,  // fast: rho_next = (rhat, rn), stuck test, beta, tmp2 = -beta omega, rho;
                         // fin_arg: the next iteration's opening test (it is no refresh)
    FIN_BIS_INIT   = 9,  // save refresh: alpha = omega = rho = 1
    FIN_BIS_RHO    = 10, // save: rho_next = (rhat, rn), stuck test, beta, tmp2 = -beta omega, rho
    FIN_BI_XR      = 11, // fast, NV = 4 (|rn|^2, 0, (rhat, rn)): FIN_BI_RESID then FIN_BI_BETA
    FIN_BI_RHO     = 12, // rho = (rhat, rn) (rn replaced by a true residual)
};

struct RedArgs {
    double* partials;      // >= gridDim.x * NV doubles of scratch
    unsigned* ticket;      // zero-initialised counter, reset by the last block
    double* result;        // FIN_STORE_RESULT destination (NV doubles)
    SolverScalars* sc;     // solver scalars for the CG finishers
    int fin;
    int fin_arg = 0;       // finisher option (FIN_BI_RESID, FIN_BI_BETA)
    // Launch predicate: when set and *halt is nonzero every block returns at
    // once (a stopped device-driven solve; nothing is read or written).
    const int* halt = nullptr;
};

__device__ __forceinline__ bool halted(const RedArgs& ra) { return ra.halt && *(volatile const int*)ra.halt; }

// Complex arithmetic of the BiCGStab finishers, rounded operation by operation
// (no contraction into FMAs) as the host's complexdivide / complexmult
// (common_header_files/operations_complex.hpp:35-66) round them.
__device__ __forceinline__ void cx_div(double* out, const double* n, const double* d, int* flag)
{
    const double norm = __dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1]));
    if (!(norm > 0.0)) *flag = 1;
    const double re = __dadd_rn(__dmul_rn(n[0], d[0]), __dmul_rn(n[1], d[1]));
    const double im = __dsub_rn(__dmul_rn(n[1], d[0]), __dmul_rn(n[0], d[1]));
    out[0]          = __ddiv_rn(re, norm);
    out[1]          = __ddiv_rn(im, norm);
}
__device__ __forceinline__ void cx_mul(double* out, const double* a, const double* b)
{
    const double re = __dsub_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1]));
    const double im = __dadd_rn(__dmul_rn(a[1], b[0]), __dmul_rn(a[0], b[1]));
    out[0]          = re;
    out[1]          = im;
}
// beta = (rho_next / rho)(alpha / omega), tmp1 = beta omega, tmp2 = -tmp1, rho = rho_next
// (bicgstab.cpp:712-720 fast, :473-479 save)
__device__ __forceinline__ void bicg_beta(SolverScalars* s)
{
    const double mone[2] = {-1.0, 0.0};
    cx_div(s->tmp1, s->rho_next, s->rho, &s->flag);
    cx_div(s->tmp2, s->alpha, s->omega, &s->flag);
    cx_mul(s->beta, s->tmp1, s->tmp2);
    cx_mul(s->tmp1, s->beta, s->omega);
    cx_mul(s->tmp2, mone, s->tmp1);
    s->rho[0] = s->rho_next[0];
    s->rho[1] = s->rho_next[1];
}
__device__ __forceinline__ bool bicg_stuck(const double* r)
{
    return fabs(r[0]) < 1e-25 && fabs(r[1]) < 1e-25;  // bicgstab.cpp:467, :705
}
// the stopping test on |r|^2 (NaN -> SolverStuck, below thr -> converged)
__device__ __forceinline__ int bicg_test(const SolverScalars* s, int nan_bit, int conv_bit)
{
    if (s->resid != s->resid) return nan_bit;
    return s->resid < s->thr ? conv_bit : 0;
}

__device__ __forceinline__ void cdiv_store(double* out, const double* n, const double* d, int* flag)
{
    const double norm = d[0] * d[0] + d[1] * d[1];
    if (!(norm > 0.0)) *flag = 1;
    out[0] = (n[0] * d[0] + n[1] * d[1]) / norm;
    out[1] = (n[1] * d[0] - n[0] * d[1]) / norm;
}

// Partial `index` of a reduction (thread 0 holds the block sum).
template <int NV>
__device__ __forceinline__ void store_partial(const double v[NV], const RedArgs& ra, size_t index)
{
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) ra.partials[index * NV + k] = v[k];
}

// What the last block's thread 0 does with the group's sum (RedArgs::fin).
template <int NV>
__device__ __forceinline__ void finish_apply(const RedArgs& ra, const double acc[NV])
{
    SolverScalars* s = ra.sc;
    switch (ra.fin) {
        case FIN_STORE_RESULT:
#pragma unroll
            for (int k = 0; k < NV; ++k) ra.result[k] = acc[k];
            break;
        case FIN_CG_ALPHA: {
            s->rho[0] = acc[0];
            s->rho[1] = NV > 1 ? acc[NV > 1 ? 1 : 0] : 0.0;
            cdiv_store(s->alpha, s->omega, s->rho, &s->flag);
            break;
        }
        case FIN_CG_BETA: {
            s->rho_next[0] = acc[0];
            s->rho_next[1] = 0.0;
            s->resid       = acc[0];
            cdiv_store(s->beta, s->rho_next, s->omega, &s->flag);
            s->omega[0] = s->rho_next[0];
            s->omega[1] = s->rho_next[1];
            break;
        }
        case FIN_CG_OMEGA: {
            s->omega[0] = acc[0];
            s->omega[1] = 0.0;
            s->resid    = acc[0];
            break;
        }
        case FIN_BI_REFRESH: {  // NV = 4: <rhat, rn>, <rhat, rhat> with rhat = rn
            s->rho[0] = acc[0];
            s->rho[1] = acc[NV > 1 ? 1 : 0];
            s->resid  = acc[NV > 2 ? 2 : 0];
            s->halt |= bicg_test(s, HALT_NAN, HALT_CONV);
            break;
        }
        case FIN_BI_ALPHA: {
            s->tmp1[0] = acc[0];
            s->tmp1[1] = acc[NV > 1 ? 1 : 0];
            cx_div(s->alpha, s->rho, s->tmp1, &s->flag);
            break;
        }
        case FIN_BI_OMEGA: {  // NV = 4: <t, s>, <t, t>
            s->tmp1[0] = acc[0];
            s->tmp1[1] = acc[NV > 1 ? 1 : 0];
            s->tmp2[0] = acc[NV > 2 ? 2 : 0];
            s->tmp2[1] = acc[NV > 3 ? 3 : 0];
            cx_div(s->omega, s->tmp1, s->tmp2, &s->flag);
            break;
        }
        case FIN_BI_RESID: {
            s->resid = acc[0];
            if (ra.fin_arg) s->halt |= bicg_test(s, HALT_NAN, HALT_CONV);
            break;
        }
        case FIN_BI_BETA: {
            s->rho_next[0] = acc[0];
            s->rho_next[1] = acc[NV > 1 ? 1 : 0];
            if (bicg_stuck(s->rho_next)) {
                s->halt |= HALT_STUCK;
                break;
            }
            bicg_beta(s);
            if (ra.fin_arg) s->halt_next |= bicg_test(s, HALT_NAN_NEXT, HALT_CONV_NEXT);
            break;
        }
        case FIN_BI_XR: {
            s->resid       = acc[0];
            s->rho_next[0] = acc[NV > 2 ? 2 : 0];
            s->rho_next[1] = acc[NV > 3 ? 3 : 0];
            if (bicg_stuck(s->rho_next)) {
                s->halt |= HALT_STUCK;
                break;
            }
            bicg_beta(s);
            if (ra.fin_arg) s->halt_next |= bicg_test(s, HALT_NAN_NEXT, HALT_CONV_NEXT);
            break;
        }
        case FIN_BI_RHO: {
            s->rho[0] = acc[0];
            s->rho[1] = acc[NV > 1 ? 1 : 0];
            break;
        }
        case FIN_BIS_INIT: {
            s->alpha[0] = s->omega[0] = s->rho[0] = 1.0;
            s->alpha[1] = s->omega[1] = s->rho[1] = 0.0;
            break;
        }
        case FIN_BIS_RHO: {
            s->rho_next[0] = acc[0];
            s->rho_next[1] = acc[NV > 1 ? 1 : 0];
            if (bicg_stuck(s->rho_next)) {
                s->halt |= HALT_STUCK;
                break;
            }
            bicg_beta(s);
            break;
        }
    }
}

// Called by every thread of every block after block_sum (value in thread 0).
// Batched launches reduce per group: block b belongs to group b % G (one
// group per right-hand side), each group has its own ticket ra.ticket[grp]
// and its last block sums that group's partials in block order.
template <int NV>
__device__ __forceinline__ void finish_reduction(const double v[NV], const RedArgs& ra, double* smem, int grp = 0,
                                                 int G = 1);

// The ticket and final sum of a group whose `nparts` partials sit at
// partials[(m * G + grp) * NV], m < nparts, written by the `nblocks` blocks of
// the group (grid-stride kernels write several partials per block).
// ROUND: partials loaded per thread before they are added (the order of the
// additions does not depend on it); wider rounds shorten this block's serial
// tail, at ROUND * NV registers.
template <int NV, int ROUND = 8>
__device__ __forceinline__ void finish_group(const RedArgs& ra, double* smem, int grp, int G, int nparts, int nblocks)
{
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(ra.ticket + grp, 1u);
        last             = (t == (unsigned)nblocks - 1u);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int nb = nparts;
    // fixed-order sum of the group's partials: thread j takes partials
    // j, j + blockDim.x, ... in rounds of ROUND independent loads (this block
    // runs alone at the end of the kernel, so its load latency is not hidden)
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    const int step = blockDim.x;
    for (int m0 = threadIdx.x; m0 < nb; m0 += ROUND * step) {
        double t[ROUND][NV];
#pragma unroll
        for (int u = 0; u < ROUND; ++u) {
            const int m = m0 + u * step;
#pragma unroll
            for (int k = 0; k < NV; ++k) t[u][k] = m < nb ? __ldcg(ra.partials + ((size_t)m * G + grp) * NV + k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < ROUND; ++u)
#pragma unroll
            for (int k = 0; k < NV; ++k) acc[k] += t[u][k];
    }
    block_sum<NV>(acc, smem);
    if (threadIdx.x == 0) {
        ra.ticket[grp] = 0u;
        finish_apply<NV>(ra, acc);
        __threadfence();
    }
}

template <int NV>
__device__ __forceinline__ void finish_reduction(const double v[NV], const RedArgs& ra, double* smem, int grp, int G)
{
    store_partial<NV>(v, ra, blockIdx.x);
    const int nb = (int)gridDim.x / G;  // blocks (= partials) of this group
    finish_group<NV>(ra, smem, grp, G, nb, nb);
}

}  // namespace c2q
