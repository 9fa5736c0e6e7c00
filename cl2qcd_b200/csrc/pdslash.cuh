// pdslash.cuh -- the eo hopping term with the fused tm epilogues for the
// reduced-precision (FP32, FP16 fixed point) fields, on the paired-site slots
// of pack.cuh, for a batch of right-hand sides that share one gauge field.
//
// One thread computes one slot (two output sites) of one right-hand side,
// with packed FP32 arithmetic throughout: each float2 holds the same quantity
// for the two sites, so every multiply-add, add and multiply of the stencil is
// one f32x2 instruction for two sites.  The operator and its epilogues are the
// ones of dslash.cuh (the reference's dslash_eo, ocl_kernel/fermionmatrix_eo.cl:30-253,
// fused with M_tm_inverse_sitediagonal and the Aee/saxpy_AND_gamma5 tail).
//
// Batches: block b works on right-hand side b % nrhs and slot block b / nrhs,
// so the blocks that read the same links run side by side and each link
// crosses HBM once per batch; reductions are kept per right-hand side.
//
// FP16 arithmetic: the neighbour's biased words are projected without first
// removing the bias (a - b of two biased values is exact; a + b subtracts the
// doubled bias first), all values stay integers in units of the site's scale,
// and the scale (norm / 32767) of the neighbour site and the link scale 1/32767
// are applied as one factor per hop and one per launch.
#pragma once

#include <type_traits>

#include "dslash.cuh"
#include "pack.cuh"
#include "reduce.cuh"

namespace c2q {

constexpr int PK_THREADS = 128;
// partials per thread and load round of the sweeps' reduction finisher (4096
// tiles at 32^3x64: two rounds for the 128 threads of the last block)
constexpr int PK_FINISH_ROUND = 16;

// Fields of one right-hand side of a batch.
struct PkRhs {
    void* out;
    float* out_norm;
    const void* in;
    const float* in_norm;
    const void* x;        // EPI_AXPY operand (same parity as out)
    const float* x_norm;
    const void* y;        // DOT_Y partner
    const float* y_norm;
    SolverScalars* sc;    // finisher target of this right-hand side
    double* result;       // FIN_STORE_RESULT target (2 doubles)
};

struct PkGeom {
    int ns, nsh, nt2;     // NS, NS/2, NT/2
    int H;                // slots = Seo/2
    int ss;               // lane stride in slots
    int vs_h;             // NS^3/2 (slots per time slice)
    FastDiv div_nsh, div_ns;
};

template <int P>
struct PkParams {
    PkRhs r[PK_MAX_RHS];
    int nrhs;
    const void* gauge;
    PkGeom g;
    HopCoef c;
    EpiArgs e;
    int out_parity;
    int ntiles;  // tiles of PK_THREADS slots per right-hand side
    int tg;                 // the gauge field is in the temporal gauge (PH_TG)
    double lam_re, lam_im;  // PH_TG: weight of the T hop leaving the last time slice
    RedArgs red;
    int pdl;                // launched as a dependent launch (launch_dep)
};

// hop weight k (pairs) and its negations
struct Kc {
    float2 re, im, nre, nim;
};

// -------------------------------------------------------------- projection
// h = a + c b, c in {1, -1, i, -i} = CK 0..3, from biased FP16 words
template <int CK>
__device__ __forceinline__ C2 proj_words(uint2 a, uint2 b)
{
    const float2 m1 = bc2(-1.0f), nb2 = bc2(-FIX_BIAS2);
    const float2 ar = blo(a), ai = bhi(a);
    if (CK == 0) return C2{add2(add2(ar, nb2), blo(b)), add2(add2(ai, nb2), bhi(b))};
    if (CK == 1) return C2{fma2(blo(b), m1, ar), fma2(bhi(b), m1, ai)};
    if (CK == 2) return C2{fma2(bhi(b), m1, ar), add2(add2(ai, nb2), blo(b))};
    return C2{add2(add2(ar, nb2), bhi(b)), fma2(blo(b), m1, ai)};
}
// same from FP32 values
template <int CK>
__device__ __forceinline__ C2 proj_vals(C2 a, C2 b)
{
    const float2 m1 = bc2(-1.0f);
    if (CK == 0) return C2{add2(a.re, b.re), add2(a.im, b.im)};
    if (CK == 1) return C2{fma2(b.re, m1, a.re), fma2(b.im, m1, a.im)};
    if (CK == 2) return C2{fma2(b.im, m1, a.re), add2(a.im, b.re)};
    return C2{add2(a.re, b.im), fma2(b.re, m1, a.im)};
}

// acc += k * (u s) with u = conj(c) in {1, -1, i, -i} = CU 0..3
template <int CU, bool KREAL>
__device__ __forceinline__ void acc_add(C2& a, float2 sre, float2 sim, const Kc& k)
{
    if (KREAL) {
        if (CU == 0) {
            a.re = fma2(sre, k.re, a.re);
            a.im = fma2(sim, k.re, a.im);
        } else if (CU == 1) {
            a.re = fma2(sre, k.nre, a.re);
            a.im = fma2(sim, k.nre, a.im);
        } else if (CU == 2) {  // i s = (-sim, sre)
            a.re = fma2(sim, k.nre, a.re);
            a.im = fma2(sre, k.re, a.im);
        } else {  // -i s = (sim, -sre)
            a.re = fma2(sim, k.re, a.re);
            a.im = fma2(sre, k.nre, a.im);
        }
    } else {
        if (CU == 0) {
            a.re = fma2(sre, k.re, fma2(sim, k.nim, a.re));
            a.im = fma2(sim, k.re, fma2(sre, k.im, a.im));
        } else if (CU == 1) {
            a.re = fma2(sre, k.nre, fma2(sim, k.im, a.re));
            a.im = fma2(sim, k.nre, fma2(sre, k.nim, a.im));
        } else if (CU == 2) {
            a.re = fma2(sim, k.nre, fma2(sre, k.nim, a.re));
            a.im = fma2(sre, k.re, fma2(sim, k.nim, a.im));
        } else {
            a.re = fma2(sim, k.re, fma2(sre, k.im, a.re));
            a.im = fma2(sre, k.nre, fma2(sim, k.im, a.im));
        }
    }
}

// One half-spinor channel: s = U h (or U^dagger h), acc_A += k s, acc_PP += conj(c) k s.
template <int A, int PP, int CK, bool DAG, bool KREAL>
__device__ __forceinline__ void pk_channel(C2 acc[12], const C2 h[3], const C2 u[9], const Kc& k)
{
    const float2 m1 = bc2(-1.0f);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        float2 sre, sim;
        if (!DAG) {  // s_r = sum_c U[r][c] h_c
            float2 p = mul2(u[3 * r].re, h[0].re), q = mul2(u[3 * r].im, h[0].im);
            p        = fma2(u[3 * r + 1].re, h[1].re, p);
            q        = fma2(u[3 * r + 1].im, h[1].im, q);
            p        = fma2(u[3 * r + 2].re, h[2].re, p);
            q        = fma2(u[3 * r + 2].im, h[2].im, q);
            sre      = fma2(q, m1, p);
            sim      = mul2(u[3 * r].re, h[0].im);
            sim      = fma2(u[3 * r].im, h[0].re, sim);
            sim      = fma2(u[3 * r + 1].re, h[1].im, sim);
            sim      = fma2(u[3 * r + 1].im, h[1].re, sim);
            sim      = fma2(u[3 * r + 2].re, h[2].im, sim);
            sim      = fma2(u[3 * r + 2].im, h[2].re, sim);
        } else {  // s_r = sum_c conj(U[c][r]) h_c
            sre      = mul2(u[r].re, h[0].re);
            sre      = fma2(u[r].im, h[0].im, sre);
            sre      = fma2(u[3 + r].re, h[1].re, sre);
            sre      = fma2(u[3 + r].im, h[1].im, sre);
            sre      = fma2(u[6 + r].re, h[2].re, sre);
            sre      = fma2(u[6 + r].im, h[2].im, sre);
            float2 p = mul2(u[r].re, h[0].im), q = mul2(u[r].im, h[0].re);
            p        = fma2(u[3 + r].re, h[1].im, p);
            q        = fma2(u[3 + r].im, h[1].re, q);
            p        = fma2(u[6 + r].re, h[2].im, p);
            q        = fma2(u[6 + r].im, h[2].re, q);
            sim      = fma2(q, m1, p);
        }
        acc_add<0, KREAL>(acc[3 * A + r], sre, sim, k);
        acc_add<ConjUnit<CK>::value, KREAL>(acc[3 * PP + r], sre, sim, k);
    }
}

// ------------------------------------------------------------------ staging
// Every thread streams the data of its next hops into its own slices of a
// shared-memory ring with cp.async (16 bytes per copy), so two or three hops
// of loads are in flight while it computes the current one, without holding
// them in registers.  A stage holds, as 16-byte chunks, the neighbour spinor
// (FP16: 6 chunks + one for the norm pair; FP32: 12) followed by its link
// (FP16: 3 chunks; FP32: NL).  Chunk c of stage s of thread t sits at
// ring[(s * CH + c) * PK_THREADS + t]: consecutive threads read consecutive
// 16-byte words.  Only the thread that copied a chunk reads it, so
// cp.async.wait_group alone orders the copies and the reads.
//
// Launch configurations (CFG), chosen per launch shape by the autotuner of
// pdslash.cu: ring depth STAGES and the resident blocks per SM (MINB) that
// the register budget is fitted to.
//   FP16: CFG 0 = 3 stages, 3 blocks/SM; CFG 1 = 2 stages, 4 blocks/SM
//   FP32: CFG 0 = 2 stages, 2 blocks/SM; CFG 1 = 2 stages, 3 blocks/SM
constexpr int PK_CONFIGS = 2;
template <int P, int NL>
struct PkChunks {
    static constexpr int SPC = P == 16 ? 7 : 12;
    // FP16 18-real: entries 0..7 in four chunks, entry 8 in half of a fifth
    static constexpr int LKC = P == 16 ? (NL == 6 ? 3 : 5) : NL;
    static constexpr int CH  = SPC + LKC;
};
template <int P, int NL, int CFG>
struct PkStage : PkChunks<P, NL> {
    static constexpr int STAGES   = (P == 16 && CFG == 0) ? 3 : 2;
    static constexpr int MINB     = P == 16 ? (CFG == 0 ? 3 : 4) : (CFG == 0 ? 2 : 3);
    static constexpr size_t BYTES = (size_t)STAGES * PkChunks<P, NL>::CH * 16 * PK_THREADS;
};

__device__ __forceinline__ void cp16(uint4* smem, const void* g)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp8(uint4* smem, const void* g)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// spinor of `slot` of field (d, norm) -> chunks [0, SPC) of a stage
template <int P>
__device__ __forceinline__ void stage_spinor(uint4* st, const void* d, const float* norm, int ss, int slot)
{
    const uint4* p  = static_cast<const uint4*>(d) + slot;
    constexpr int n = P == 16 ? 6 : 12;
#pragma unroll
    for (int c = 0; c < n; ++c) cp16(st + c * PK_THREADS, p + (size_t)c * ss);
    if (P == 16) cp8(st + 6 * PK_THREADS, reinterpret_cast<const float2*>(norm) + slot);
}
// link of `slot` of a (parity, mu) group -> chunks [SPC, CH)
template <int P, int NL>
__device__ __forceinline__ void stage_link(uint4* st, const char* links, int ss, int slot)
{
    constexpr int SPC = PkChunks<P, NL>::SPC, LKC = PkChunks<P, NL>::LKC;
    const uint4* p    = reinterpret_cast<const uint4*>(links) + slot;
    if constexpr (P == 16 && NL == 9) {
#pragma unroll
        for (int c = 0; c < 4; ++c) cp16(st + (SPC + c) * PK_THREADS, p + (size_t)c * ss);
        cp8(st + (SPC + 4) * PK_THREADS, reinterpret_cast<const uint2*>(links + (size_t)64 * ss) + slot);
    } else {
#pragma unroll
        for (int c = 0; c < LKC; ++c) cp16(st + (SPC + c) * PK_THREADS, p + (size_t)c * ss);
    }
}

// The fused CG updates stage the 12 chunks of the slot's FP32 residual
// (DOT_CGR) or solution increment (DOT_XUPD) in the two epilogue slots: the
// q = 9 slot (unused by these sweeps) from chunk 0, and, when it is shorter
// than 12 chunks, the rest of the q = 8 slot after the spinor operand there
// (the EPI_AXPY operand or the search direction; FP16: chunks 7 ..).
template <int P, int NL>
struct ResidualPlace {
    static constexpr int CH     = PkChunks<P, NL>::CH;
    static constexpr int IN9    = CH < 12 ? CH : 12;        // chunks in the q = 9 slot
    static constexpr int AFTER8 = P == 16 ? 7 : 12;        // first free chunk of the q = 8 slot
    static_assert(IN9 + (CH - AFTER8) >= 12, "residual does not fit the epilogue slots");
};
template <int P, int NL, int Q>
__device__ __forceinline__ void stage_residual(uint4* st, const void* r, int ss, int slot)
{
    using RP        = ResidualPlace<P, NL>;
    const uint4* p  = static_cast<const uint4*>(r) + slot;
    if constexpr (Q == 9) {
#pragma unroll
        for (int c = 0; c < RP::IN9; ++c) cp16(st + c * PK_THREADS, p + (size_t)c * ss);
    } else {
#pragma unroll
        for (int c = RP::IN9; c < 12; ++c) cp16(st + (RP::AFTER8 + c - RP::IN9) * PK_THREADS, p + (size_t)c * ss);
    }
}
template <int P, int NL>
__device__ __forceinline__ uint4 residual_chunk(const uint4* s8, const uint4* s9, int c)
{
    using RP = ResidualPlace<P, NL>;
    return c < RP::IN9 ? s9[c * PK_THREADS] : s8[(RP::AFTER8 + c - RP::IN9) * PK_THREADS];
}

__device__ __forceinline__ float4 as_f4(uint4 v)
{
    return make_float4(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z), __uint_as_float(v.w));
}

// decode a staged link (chunks at lk[c * PK_THREADS])
template <int P, int NL, bool SWP>
__device__ __forceinline__ void staged_link(const uint4* lk, C2 u[9])
{
    if constexpr (P == 16) {
        const float2 nb = bc2(-FIX_BIAS);
        constexpr int L2 = NL == 6 ? 3 : 4;
#pragma unroll
        for (int L = 0; L < L2; ++L) {
            const uint4 v  = lk[L * PK_THREADS];
            const uint2 wa = SWP ? make_uint2(v.y, v.x) : make_uint2(v.x, v.y);
            const uint2 wb = SWP ? make_uint2(v.w, v.z) : make_uint2(v.z, v.w);
            u[2 * L]       = C2{add2(blo(wa), nb), add2(bhi(wa), nb)};
            u[2 * L + 1]   = C2{add2(blo(wb), nb), add2(bhi(wb), nb)};
        }
        if constexpr (NL == 9) {
            const uint4 v  = lk[4 * PK_THREADS];
            const uint2 wa = SWP ? make_uint2(v.y, v.x) : make_uint2(v.x, v.y);
            u[8]           = C2{add2(blo(wa), nb), add2(bhi(wa), nb)};
        } else {
            reconstruct_row2_pk(u, 1.0f / 32767.0f);
        }
    } else {
#pragma unroll
        for (int e = 0; e < NL; ++e) u[e] = c2_from(as_f4(lk[e * PK_THREADS]), SWP);
        if (NL == 6) reconstruct_row2_pk(u, 1.0f);
    }
}
// FP16 words and norm pair of a staged spinor
template <bool SWP>
__device__ __forceinline__ void staged_words(const uint4* st, uint2 w[12], float2* nrm)
{
#pragma unroll
    for (int L = 0; L < 6; ++L) {
        const uint4 v = st[L * PK_THREADS];
        w[2 * L]      = SWP ? make_uint2(v.y, v.x) : make_uint2(v.x, v.y);
        w[2 * L + 1]  = SWP ? make_uint2(v.w, v.z) : make_uint2(v.z, v.w);
    }
    const float2 n = *reinterpret_cast<const float2*>(st + 6 * PK_THREADS);
    *nrm           = SWP ? swap2(n) : n;
}
// FP32 values of a staged spinor
template <bool SWP>
__device__ __forceinline__ void staged_vals(const uint4* st, C2 s[12])
{
#pragma unroll
    for (int c = 0; c < 12; ++c) s[c] = c2_from(as_f4(st[c * PK_THREADS]), SWP);
}
// a staged (unswapped) operand as values sc * q: FP16 exact integers and the
// per-site scale, FP32 values and scale 1
template <int P>
__device__ __forceinline__ void staged_operand(const uint4* st, C2 q[12], float2* sc)
{
    if constexpr (P == 16) {
        uint2 w[12];
        float2 n;
        staged_words<false>(st, w, &n);
        *sc             = mul2(n, bc2(1.0f / 32767.0f));
        const float2 nb = bc2(-FIX_BIAS);
#pragma unroll
        for (int c = 0; c < 12; ++c) q[c] = C2{add2(blo(w[c]), nb), add2(bhi(w[c]), nb)};
    } else {
        staged_vals<false>(st, q);
        *sc = bc2(1.0f);
    }
}

// The spinor half of one hop: the decoded link u applied to the staged
// neighbour spinor st (projection, SU(3) products, accumulation).  The
// neighbour slot may hold the two sites swapped -- SWP, set for the time hops
// across the fold.  w: the hop weight of each lane (the two sites) and its
// negations.
template <int P, int MU, bool BACK, bool SWP, bool KREAL>
__device__ __forceinline__ void pk_hop_spinor(C2 acc[12], const uint4* st, const C2 u[9], const Kc& w)
{
    using T          = Proj<MU>;
    constexpr int c0 = BACK ? NegUnit<T::c0>::value : T::c0;
    constexpr int c1 = BACK ? NegUnit<T::c1>::value : T::c1;
    Kc k;
    C2 h[3];
    if constexpr (P == 16) {
        uint2 wd[12];
        float2 nrm;
        staged_words<SWP>(st, wd, &nrm);
        k.re  = mul2(w.re, nrm);
        k.nre = mul2(w.nre, nrm);
        if (!KREAL) {
            k.im  = mul2(w.im, nrm);
            k.nim = mul2(w.nim, nrm);
        }
#pragma unroll
        for (int col = 0; col < 3; ++col) h[col] = proj_words<c0>(wd[col], wd[3 * T::p0 + col]);
        pk_channel<0, T::p0, c0, BACK, KREAL>(acc, h, u, k);
#pragma unroll
        for (int col = 0; col < 3; ++col) h[col] = proj_words<c1>(wd[3 + col], wd[3 * T::p1 + col]);
        pk_channel<1, T::p1, c1, BACK, KREAL>(acc, h, u, k);
    } else {
        C2 psi[12];
        staged_vals<SWP>(st, psi);
        k = w;
#pragma unroll
        for (int col = 0; col < 3; ++col) h[col] = proj_vals<c0>(psi[col], psi[3 * T::p0 + col]);
        pk_channel<0, T::p0, c0, BACK, KREAL>(acc, h, u, k);
#pragma unroll
        for (int col = 0; col < 3; ++col) h[col] = proj_vals<c1>(psi[3 + col], psi[3 * T::p1 + col]);
        pk_channel<1, T::p1, c1, BACK, KREAL>(acc, h, u, k);
    }
}

// One hop from a stage: its link (staged after the spinor) decoded, then the
// spinor half.  A forward hop's link sits at the output slot and is never
// swapped; a backward hop's link swaps with its neighbour slot.
template <int P, int NL, int MU, bool BACK, bool SWP, bool KREAL>
__device__ __forceinline__ void pk_hop(C2 acc[12], const uint4* st, const Kc& w)
{
    C2 u[9];
    staged_link<P, NL, BACK && SWP>(st + PkChunks<P, NL>::SPC * PK_THREADS, u);
    pk_hop_spinor<P, MU, BACK, SWP, KREAL>(acc, st, u, w);
}

// A half-spinor channel through an identity link: acc_A += k h, acc_PP += conj(c) k h.
template <int A, int PP, int CK>
__device__ __forceinline__ void pk_identity_channel(C2 acc[12], const C2 h[3], const Kc& k)
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        acc_add<0, true>(acc[3 * A + r], h[r].re, h[r].im, k);
        acc_add<ConjUnit<CK>::value, true>(acc[3 * PP + r], h[r].re, h[r].im, k);
    }
}
// A time hop inside the temporal gauge: the link is the identity (no link
// staged), the weight real and the same for both lanes.  FP16: the launch
// scale carries the link scale 1/32767 of a stored link, so the weight here
// carries 32767.
template <int P, bool BACK>
__device__ __forceinline__ void pk_hop_id(C2 acc[12], const uint4* st, float wt)
{
    using T          = Proj<0>;
    constexpr int c0 = BACK ? NegUnit<T::c0>::value : T::c0;
    constexpr int c1 = BACK ? NegUnit<T::c1>::value : T::c1;
    Kc k;
    C2 h[3];
    if constexpr (P == 16) {
        uint2 wd[12];
        float2 nrm;
        staged_words<false>(st, wd, &nrm);
        k.re  = mul2(bc2(wt * 32767.0f), nrm);
        k.nre = mul2(bc2(-wt * 32767.0f), nrm);
#pragma unroll
        for (int col = 0; col < 3; ++col) h[col] = proj_words<c0>(wd[col], wd[3 * T::p0 + col]);
        pk_identity_channel<0, T::p0, c0>(acc, h, k);
#pragma unroll
        for (int col = 0; col < 3; ++col) h[col] = proj_words<c1>(wd[3 + col], wd[3 * T::p1 + col]);
        pk_identity_channel<1, T::p1, c1>(acc, h, k);
    } else {
        C2 psi[12];
        staged_vals<false>(st, psi);
        k.re  = bc2(wt);
        k.nre = bc2(-wt);
#pragma unroll
        for (int col = 0; col < 3; ++col) h[col] = proj_vals<c0>(psi[col], psi[3 * T::p0 + col]);
        pk_identity_channel<0, T::p0, c0>(acc, h, k);
#pragma unroll
        for (int col = 0; col < 3; ++col) h[col] = proj_vals<c1>(psi[3 + col], psi[3 * T::p1 + col]);
        pk_identity_channel<1, T::p1, c1>(acc, h, k);
    }
}

__device__ __forceinline__ Kc uniform_weight(double re, double im)
{
    return Kc{bc2((float)re), bc2((float)im), bc2((float)-re), bc2((float)-im)};
}

// hop q = 2 mu + back, with the phase pattern resolved
template <int P, int NL, int MU, bool BACK, bool SWP, int PH>
__device__ __forceinline__ void pk_hop_ph(C2 acc[12], const PkParams<P>& prm, const uint4* st)
{
    const int d  = BACK ? 1 : 0;
    const Kc w   = uniform_weight(prm.c.re[MU][d], prm.c.im[MU][d]);
    if (PH == PH_REAL || PH == PH_TG || (PH == PH_TCPLX && MU != 0)) {
        pk_hop<P, NL, MU, BACK, SWP, true>(acc, st, w);
    } else if (PH == PH_TCPLX) {
        pk_hop<P, NL, MU, BACK, SWP, false>(acc, st, w);
    } else if ((prm.c.real_mask >> (2 * MU + d)) & 1u) {
        pk_hop<P, NL, MU, BACK, SWP, true>(acc, st, w);
    } else {
        pk_hop<P, NL, MU, BACK, SWP, false>(acc, st, w);
    }
}

// A time hop across the fold inside the temporal gauge: one lane crosses the
// last time slice through its stored link W with the weight lambda (forward)
// or conj(lambda) (backward), lambda the product of the T phases around the
// lattice; the other lane steps between two inner slices, where the stored
// link is the identity and the weight 1.
template <int P, int NL, bool BACK>
__device__ __forceinline__ void pk_hop_tg_fold(C2 acc[12], const PkParams<P>& prm, const uint4* st)
{
    const float lr = (float)prm.lam_re, li = (float)prm.lam_im;
    const Kc w     = BACK ? Kc{make_float2(lr, 1.0f), make_float2(-li, 0.0f), make_float2(-lr, -1.0f),
                           make_float2(li, 0.0f)}
                          : Kc{make_float2(1.0f, lr), make_float2(0.0f, li), make_float2(-1.0f, -lr),
                           make_float2(0.0f, -li)};
    pk_hop<P, NL, 0, BACK, true, false>(acc, st, w);
}

// bytes per slot of a (parity, mu) group of links in the slot layout
template <int P, int NL>
__host__ __device__ constexpr int pk_link_bytes()
{
    return P == 16 ? (NL == 6 ? 48 : 72) : 16 * NL;
}

template <int P, int NL, int EPI, int DOT, int PH, int CFG>
__global__ void __launch_bounds__(PK_THREADS, PkStage<P, NL, CFG>::MINB) pdslash_kernel(const PkParams<P> prm)
{
    using S = PkStage<P, NL, CFG>;
    static_assert(S::STAGES == 2 || S::STAGES == 3, "the prologue below issues one or two stages");
    static_assert(DOT != DOT_XUPD || EPI != EPI_AXPY, "the solution update shares the EPI_AXPY operand slot");
    constexpr bool RED = DOT != DOT_NONE && DOT != DOT_XUPD;  // a reduction is fused
    pdl_enter();
    if (halted(prm.red)) return;  // a stopped device-driven solve: every block leaves
    extern __shared__ uint4 ring[];
    uint4* mine     = ring + threadIdx.x;
    const PkGeom& g = prm.g;
    const int nrhs  = prm.nrhs;
    const int rhs   = nrhs == 1 ? 0 : (int)(blockIdx.x % (unsigned)nrhs);
    const int blk   = nrhs == 1 ? (int)blockIdx.x : (int)(blockIdx.x / (unsigned)nrhs);
    const int G     = (int)gridDim.x / nrhs;  // blocks per right-hand side
    const PkRhs& rr = prm.r[rhs];
    __shared__ double smem[2 * 32];

    // tiles of PK_THREADS slots; a block takes tiles blk, blk + G, ... (one
    // tile per block unless the grid is sized to the resident blocks)
    for (int tile = blk; tile < prm.ntiles; tile += G) {
    const int j = tile * PK_THREADS + threadIdx.x;
    float2 dre = bc2(0.f), dim = bc2(0.f), dq = bc2(0.f);

    if (j < g.H) {
        // coordinates of slot j (site 0 at time t < NT/2; site 1 at t + NT/2)
        const unsigned r1 = fdiv((unsigned)j, g.div_nsh);
        const int xh      = j - (int)r1 * g.nsh;
        const unsigned r2 = fdiv(r1, g.div_ns);
        const int y       = (int)r1 - (int)r2 * g.ns;
        const int t       = (int)fdiv(r2, g.div_ns);
        const int z       = (int)r2 - t * g.ns;
        const int x       = 2 * xh + ((prm.out_parity + y + z + t) & 1);
        const int yzt     = j - xh;
        const int ss      = g.ss;

        const int po          = prm.out_parity;
        const size_t grp      = (size_t)pk_link_bytes<P, NL>() * ss;
        const char* gb        = static_cast<const char*>(prm.gauge);
        const char* fwd_links = gb + (size_t)(po * 4) * grp;
        const char* bwd_links = gb + (size_t)((1 - po) * 4) * grp;

        // neighbour slot and link slot of the 8 hops (q = 2 mu + back); across
        // the fold in time the neighbour slot holds the pair swapped
        const bool fold_f = t + 1 == g.nt2, fold_b = t == 0;
        const int base    = j - g.vs_h * t;
        int nb[8];
        nb[0]        = fold_f ? base : j + g.vs_h;
        nb[1]        = fold_b ? base + g.vs_h * (g.nt2 - 1) : j - g.vs_h;
        const int xp = x + 1 == g.ns ? 0 : x + 1, xm = x == 0 ? g.ns - 1 : x - 1;
        nb[2]        = (xp >> 1) + yzt;
        nb[3]        = (xm >> 1) + yzt;
        const int row = g.nsh, pl = g.nsh * g.ns;
        nb[4]         = y + 1 == g.ns ? j - (g.ns - 1) * row : j + row;
        nb[5]         = y == 0 ? j + (g.ns - 1) * row : j - row;
        nb[6]         = z + 1 == g.ns ? j - (g.ns - 1) * pl : j + pl;
        nb[7]         = z == 0 ? j + (g.ns - 1) * pl : j - pl;

        // stage q: hops 0..7, then the epilogue operands x (q = 8) and y (q = 9);
        // every index below is a compile-time constant
        auto issue = [&](auto qc) {
            constexpr int q = decltype(qc)::value;
            uint4* st       = mine + (size_t)((q % S::STAGES) * S::CH) * PK_THREADS;
            if constexpr (q < 8) {
                constexpr bool back = q & 1;
                stage_spinor<P>(st, rr.in, rr.in_norm, ss, nb[q]);
                // temporal gauge: the T links between inner slices are the identity
                if (PH != PH_TG || q >= 2 || (back ? fold_b : fold_f))
                    stage_link<P, NL>(st, (back ? bwd_links : fwd_links) + (size_t)(q >> 1) * grp, ss,
                                      back ? nb[q] : j);
            } else if constexpr (q == 8) {
                if (EPI == EPI_AXPY || DOT == DOT_XUPD) stage_spinor<P>(st, rr.x, rr.x_norm, ss, j);
                if (DOT == DOT_CGR || DOT == DOT_XUPD) stage_residual<P, NL, 8>(st, rr.y, ss, j);
            } else {
                if (DOT == DOT_Y) stage_spinor<P>(st, rr.y, rr.y_norm, ss, j);
                if (DOT == DOT_CGR || DOT == DOT_XUPD) stage_residual<P, NL, 9>(st, rr.y, ss, j);
            }
            cp_commit();
        };

        C2 acc[12];
#pragma unroll
        for (int c = 0; c < 12; ++c) acc[c] = C2{bc2(0.f), bc2(0.f)};

        auto step = [&](auto hc) {
            constexpr int h = decltype(hc)::value;
            if constexpr (h + S::STAGES - 1 <= 9)
                issue(std::integral_constant<int, h + S::STAGES - 1>{});
            else
                cp_commit();
            cp_wait<S::STAGES - 1>();
            const uint4* st = mine + (size_t)((h % S::STAGES) * S::CH) * PK_THREADS;
            constexpr int mu = h >> 1;
            constexpr bool back = h & 1;
            if constexpr (mu == 0 && PH == PH_TG) {
                if (back ? fold_b : fold_f)
                    pk_hop_tg_fold<P, NL, back>(acc, prm, st);
                else
                    pk_hop_id<P, back>(acc, st, 1.0f);
            } else if constexpr (mu == 0) {
                if (back ? fold_b : fold_f)
                    pk_hop_ph<P, NL, 0, back, true, PH>(acc, prm, st);
                else
                    pk_hop_ph<P, NL, 0, back, false, PH>(acc, prm, st);
            } else {
                pk_hop_ph<P, NL, mu, back, false, PH>(acc, prm, st);
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

        // epilogue on h = scale * acc (scale = -kappa, times the FP16 scales)
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
            // [g5] (f x - sc acc); FP16 x as exact integers q with the per-site
            // scale folded into f, the sign of g5 folded into the coefficients
            C2 xv[12];
            float2 xs;
            staged_operand<P>(mine + (size_t)((8 % S::STAGES) * S::CH) * PK_THREADS, xv, &xs);
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
        if (DOT != DOT_CGR) {
            if constexpr (P == 16)
                SlotF16::store(rr.out, rr.out_norm, ss, j, acc);
            else
                SlotF32::store(rr.out, ss, j, acc);
        }

        if (DOT == DOT_CGR) {  // r -= alpha out (r FP32, passed as y, staged in the ring), |r|^2
            const float ar = (float)rr.sc->alpha[0], ai = (float)rr.sc->alpha[1];
            float4* rw     = static_cast<float4*>(const_cast<void*>(rr.y));
            const uint4* s8 = mine + (size_t)((8 % S::STAGES) * S::CH) * PK_THREADS;
            const uint4* s9 = mine + (size_t)((9 % S::STAGES) * S::CH) * PK_THREADS;
#pragma unroll
            for (int c = 0; c < 12; ++c) {
                C2 r        = c2_from(as_f4(residual_chunk<P, NL>(s8, s9, c)), false);
                const C2 v  = acc[c];
                r.re        = fma2(v.re, bc2(-ar), fma2(v.im, bc2(ai), r.re));
                r.im        = fma2(v.im, bc2(-ar), fma2(v.re, bc2(-ai), r.im));
                __stcs(rw + (size_t)c * ss + j, c2_to(r));
                dre         = fma2(r.re, r.re, fma2(r.im, r.im, dre));
            }
        } else if (DOT == DOT_Y) {  // conj(y) out, FP16 y as integers times the per-site scale
            C2 yv[12];
            float2 ys;
            staged_operand<P>(mine + (size_t)((9 % S::STAGES) * S::CH) * PK_THREADS, yv, &ys);
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
        } else if (DOT == DOT_XUPD) {  // x += alpha p (x FP32, passed as y; p passed as x; both staged)
            const float ar  = (float)rr.sc->alpha[0], ai = (float)rr.sc->alpha[1];
            float4* xw      = static_cast<float4*>(const_cast<void*>(rr.y));
            const uint4* s8 = mine + (size_t)((8 % S::STAGES) * S::CH) * PK_THREADS;
            const uint4* s9 = mine + (size_t)((9 % S::STAGES) * S::CH) * PK_THREADS;
            C2 pv[12];
            float2 ps;
            staged_operand<P>(s8, pv, &ps);
            const float2 cr = mul2(bc2(ar), ps), ci = mul2(bc2(ai), ps), nci = mul2(bc2(-ai), ps);
#pragma unroll
            for (int c = 0; c < 12; ++c) {
                C2 xv = c2_from(as_f4(residual_chunk<P, NL>(s8, s9, c)), false);
                xv.re = fma2(pv[c].re, cr, fma2(pv[c].im, nci, xv.re));
                xv.im = fma2(pv[c].im, cr, fma2(pv[c].re, ci, xv.im));
                __stcs(xw + (size_t)c * ss + j, c2_to(xv));
            }
        }
    }
    if (RED) {  // one partial per tile, in tile order
        double dv[2] = {(double)dre.x + (double)dre.y,
                        ((double)dim.x - (double)dq.x) + ((double)dim.y - (double)dq.y)};
        block_sum<2>(dv, smem);
        store_partial<2>(dv, prm.red, (size_t)tile * nrhs + rhs);
    }
    }  // tiles
    if (RED) {
        RedArgs ra = prm.red;
        if (rr.sc) ra.sc = rr.sc;
        if (rr.result) ra.result = rr.result;
        finish_group<2, PK_FINISH_ROUND>(ra, smem, rhs, nrhs, prm.ntiles, G);
    }
}

}  // namespace c2q
