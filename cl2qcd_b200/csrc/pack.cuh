// pack.cuh -- paired-site ("slot") storage of the reduced-precision fields and
// the packed FP32 arithmetic that works on it.
//
// Slot layout.  A reduced-precision (FP32 or FP16) eo field of Seo sites is
// stored as H = Seo/2 slots; slot j holds the eo sites j and j + H, i.e. the
// same (x, y, z) at times t and t + NT/2 (eo index = site/2 with t slowest, so
// the two halves of the eo index range are the two halves of the time axis).
// With NT/2 even both sites have the same parity pattern, so the Wilson
// stencil maps slot pairs onto slot pairs: every neighbour of slot j's two
// sites is again one slot, with its two sites in the same order -- except for
// the time hop across the fold (t = NT/2 - 1 -> NT/2 and t = 0 -> -1), where
// the neighbour slot holds the pair in swapped order.
//
// The two sites of a slot are adjacent in every 16-byte word, so one thread
// loads both with 128-bit loads and computes on them with Blackwell's packed
// FP32 instructions (fma/add/mul .f32x2): each float2 below holds one real
// quantity for site 0 (x) and site 1 (y) of a slot.
//
//   FP32 spinor: 12 lanes of float4 (re0, re1, im0, im1), one per colour-spin
//                component c = 3*spin + colour;
//   FP16 spinor: 6 lanes of uint4 (w[2L] site 0, w[2L] site 1, w[2L+1] site 0,
//                w[2L+1] site 1) with w[c] = re | im << 16 in the biased 16-bit
//                fixed point of c2q_internal.cuh; per-site norms as float2;
//   FP32 links : NL lanes (9 or 6 complex entries) of float4 per (parity, mu);
//   FP16 links : 12-real: rows 0 and 1 (6 entries) as 3 lanes of uint4 per
//                (parity, mu); 18-real: entries 0..7 as 4 uint4 lanes and entry 8
//                as one uint2 lane.
// Lane stride = `ss` slots (half the FP64 lane stride, a multiple of 32).
#pragma once

#include "c2q_internal.cuh"

namespace c2q {

// largest batch of right-hand sides one launch handles
constexpr int PK_MAX_RHS = 16;

// one complex number for each of the two sites of a slot
struct C2 {
    float2 re, im;
};

__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 swap2(float2 a) { return make_float2(a.y, a.x); }

// 2^23 + 32768: a biased 16-bit word u placed in the mantissa of 2^23 reads
// as BIAS + q (q = u - 32768)
constexpr float FIX_BIAS  = 8421376.0f;
constexpr float FIX_BIAS2 = 16842752.0f;

// biased floats (2^23 + u) of the low / high 16-bit halves of two words
__device__ __forceinline__ float2 blo(uint2 w)
{
    return make_float2(__int_as_float(__byte_perm(w.x, 0x4B000000u, 0x7610)),
                       __int_as_float(__byte_perm(w.y, 0x4B000000u, 0x7610)));
}
__device__ __forceinline__ float2 bhi(uint2 w)
{
    return make_float2(__int_as_float(__byte_perm(w.x, 0x4B000000u, 0x7632)),
                       __int_as_float(__byte_perm(w.y, 0x4B000000u, 0x7632)));
}

// Division by a fixed positive divisor d with one high multiply and one add
// (round-up multiplier, exact for numerators below 2^31).
struct FastDiv {
    unsigned d, m;
    int l;
};
inline FastDiv make_fastdiv(unsigned d)
{
    FastDiv f;
    f.d = d;
    f.l = 0;
    while ((1ull << f.l) < d) ++f.l;
    f.m = (unsigned)(((1ull << 32) * ((1ull << f.l) - d)) / d + 1);
    return f;
}
__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) { return (__umulhi(n, f.m) + n) >> f.l; }

// ------------------------------------------------------------------ FP32 slots
__device__ __forceinline__ C2 c2_from(float4 v, bool swp)
{
    return swp ? C2{make_float2(v.y, v.x), make_float2(v.w, v.z)} : C2{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ float4 c2_to(C2 v) { return make_float4(v.re.x, v.re.y, v.im.x, v.im.y); }

struct SlotF32 {
    template <bool SWP = false>
    static __device__ __forceinline__ void load(const void* d, int ss, int j, C2 s[12])
    {
        const float4* p = static_cast<const float4*>(d);
#pragma unroll
        for (int c = 0; c < 12; ++c) s[c] = c2_from(__ldg(p + (size_t)c * ss + j), SWP);
    }
    static __device__ __forceinline__ void store(void* d, int ss, int j, const C2 s[12])
    {
        float4* p = static_cast<float4*>(d);
#pragma unroll
        for (int c = 0; c < 12; ++c) p[(size_t)c * ss + j] = c2_to(s[c]);
    }
};

// ------------------------------------------------------------------ FP16 slots
struct SlotF16 {
    // the 12 word pairs (site 0, site 1) and the norm pair of slot j
    template <bool SWP = false>
    static __device__ __forceinline__ void load_words(const void* d, const float* norm, int ss, int j, uint2 w[12],
                                                      float2* nrm)
    {
        const uint4* p = static_cast<const uint4*>(d);
#pragma unroll
        for (int L = 0; L < 6; ++L) {
            const uint4 v = __ldg(p + (size_t)L * ss + j);
            w[2 * L]      = SWP ? make_uint2(v.y, v.x) : make_uint2(v.x, v.y);
            w[2 * L + 1]  = SWP ? make_uint2(v.w, v.z) : make_uint2(v.z, v.w);
        }
        const float2 n = __ldg(reinterpret_cast<const float2*>(norm) + j);
        *nrm           = SWP ? swap2(n) : n;
    }
    // the integers q (exact) and the per-site scales norm / 32767: v = sc q
    static __device__ __forceinline__ void load_q(const void* d, const float* norm, int ss, int j, C2 q[12],
                                                  float2* sc)
    {
        uint2 w[12];
        float2 n;
        load_words(d, norm, ss, j, w, &n);
        *sc             = mul2(n, bc2(1.0f / 32767.0f));
        const float2 nb = bc2(-FIX_BIAS);
#pragma unroll
        for (int c = 0; c < 12; ++c) q[c] = C2{add2(blo(w[c]), nb), add2(bhi(w[c]), nb)};
    }
    // decoded values v = sc q
    static __device__ __forceinline__ void load(const void* d, const float* norm, int ss, int j, C2 s[12])
    {
        float2 sc;
        load_q(d, norm, ss, j, s, &sc);
#pragma unroll
        for (int c = 0; c < 12; ++c) s[c] = C2{mul2(s[c].re, sc), mul2(s[c].im, sc)};
    }
    // Encode 12 complex values per site with a per-site norm = max |component|.
    // q = rint(v * 32767 / norm) is formed by one fused multiply-add onto
    // 2^23 + 32768, whose low 16 mantissa bits are then the biased word.
    static __device__ __forceinline__ void store(void* d, float* norm, int ss, int j, const C2 s[12])
    {
        float m0 = 0.f, m1 = 0.f;
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            m0 = fmaxf(m0, fmaxf(fabsf(s[c].re.x), fabsf(s[c].im.x)));
            m1 = fmaxf(m1, fmaxf(fabsf(s[c].re.y), fabsf(s[c].im.y)));
        }
        const float2 inv = make_float2(m0 > 0.f ? 32767.0f / m0 : 0.f, m1 > 0.f ? 32767.0f / m1 : 0.f);
        const float2 bias = bc2(FIX_BIAS);
        unsigned w0[12], w1[12];
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const float2 er = fma2(s[c].re, inv, bias), ei = fma2(s[c].im, inv, bias);
            w0[c] = __byte_perm(__float_as_uint(er.x), __float_as_uint(ei.x), 0x5410);
            w1[c] = __byte_perm(__float_as_uint(er.y), __float_as_uint(ei.y), 0x5410);
        }
        uint4* p = static_cast<uint4*>(d);
#pragma unroll
        for (int L = 0; L < 6; ++L) p[(size_t)L * ss + j] = make_uint4(w0[2 * L], w1[2 * L], w0[2 * L + 1], w1[2 * L + 1]);
        reinterpret_cast<float2*>(norm)[j] = make_float2(m0, m1);
    }
};

// ------------------------------------------------------------------ links
// row2 = s * conj(row0 x row1) on slot pairs; (a x b)_k = a_{k+1} b_{k+2} - a_{k+2} b_{k+1}
__device__ __forceinline__ void cross_conj(C2& out, C2 a, C2 b, C2 c, C2 d, float s)
{
    // z = a b - c d
    const float2 t1 = fma2(a.re, b.re, mul2(c.im, d.im));
    const float2 t2 = fma2(a.im, b.im, mul2(c.re, d.re));
    const float2 t3 = fma2(a.re, b.im, mul2(a.im, b.re));
    const float2 t4 = fma2(c.re, d.im, mul2(c.im, d.re));
    out.re          = fma2(t2, bc2(-s), mul2(t1, bc2(s)));  //  s Re z
    out.im          = fma2(t4, bc2(s), mul2(t3, bc2(-s)));  // -s Im z
}
__device__ __forceinline__ void reconstruct_row2_pk(C2 u[9], float s)
{
    cross_conj(u[6], u[1], u[5], u[2], u[4], s);
    cross_conj(u[7], u[2], u[3], u[0], u[5], s);
    cross_conj(u[8], u[0], u[4], u[1], u[3], s);
}

}  // namespace c2q
