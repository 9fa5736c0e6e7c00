// c2q_internal.cuh -- device-side building blocks of the tm-Wilson eo hot path.
//
// Data layout in HBM (all fields are one parity of the lattice, "eo fields"):
//   * site order = the reference's eo index i = site/2 with
//     site = x + NS*y + NS^2*z + NS^3*t (ocl_kernel/operations_geometry.cl:97-156,
//     297-300), so uploads/downloads are pure transpositions;
//   * structure of arrays: component lane k of site i lives at lane[k*stride + i],
//     stride = Seo rounded up to a multiple of 64 sites (>= 256 B alignment
//     for every lane in every precision), so a warp reads 32 consecutive sites
//     of one lane with one 128-bit (FP64, FP32) or 64/128-bit (FP16) load each;
//   * FP64 spinor: 12 double2 lanes (spin-major: k = 3*spin + colour);
//     FP32 spinor: 6 float4 lanes (complex 2k, 2k+1 in lane k);
//     FP16 spinor: 3 int4 lanes of 8 int16 fixed-point values each, scaled by a
//       per-site float norm (max |component|) held in a separate float array;
//   * gauge field: links are grouped by the parity of the site they start at,
//     [parity][mu][lane][stride], so the 4 forward links of an output site and
//     the 4 backward links (which start at opposite-parity neighbours) are both
//     read with consecutive-site coalesced loads.  18-real storage keeps 9
//     complex lanes, 12-real storage keeps rows 0 and 1 (6 lanes) and rebuilds
//     row 2 = conj(row0 x row1), which is exact for SU(3).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace c2q {

// ------------------------------------------------------------------------
// complex helpers (compute type R = double or float)
// ------------------------------------------------------------------------
template <typename R>
struct Cplx {
    R re, im;
};
template <typename R>
__host__ __device__ __forceinline__ Cplx<R> cmk(R a, R b)
{
    return Cplx<R>{a, b};
}
template <typename R>
__device__ __forceinline__ Cplx<R> operator+(Cplx<R> a, Cplx<R> b)
{
    return {a.re + b.re, a.im + b.im};
}
template <typename R>
__device__ __forceinline__ Cplx<R> operator-(Cplx<R> a, Cplx<R> b)
{
    return {a.re - b.re, a.im - b.im};
}
template <typename R>
__device__ __forceinline__ Cplx<R> cmul(Cplx<R> a, Cplx<R> b)
{
    return {a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im};
}
// conj(a) * b
template <typename R>
__device__ __forceinline__ Cplx<R> cmulc(Cplx<R> a, Cplx<R> b)
{
    return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}

// ------------------------------------------------------------------------
// lattice geometry and per-launch operator coefficients
// ------------------------------------------------------------------------
struct Geom {
    int ns, nt;     // extents (NS even, NT even)
    int nsh;        // NS/2
    int seo;        // V/2 eo sites
    int stride;     // SoA lane stride in sites
    int vs_h;       // NS^3/2
};

// Hop coefficient table for one dslash launch: coef[mu][0] forward,
// coef[mu][1] backward, already multiplied by -kappa (the kernel's overall sign)
// and, on T links, by the chemical-potential factors.
struct HopCoef {
    double re[4][2], im[4][2];
};

// Epilogue applied to the hopping sum h at each output site.
enum Epilogue : int {
    EPI_PLAIN = 0,  // out = h                                  (dslash_eo)
    EPI_DIAG  = 1,  // out = diag(f1,f2) h                      (dslash_AND_M_tm_inverse_sitediagonal)
    EPI_AXPY  = 2,  // out = [g5] (diag(f1,f2) x - h)            (Aee tail, saxpy[_AND_gamma5])
};

// Optional reduction fused into a sweep: <y, out> or |out|^2.
enum DotMode : int { DOT_NONE = 0, DOT_Y = 1, DOT_SELF = 2 };

struct EpiArgs {
    double f1re, f1im, f2re, f2im;  // spin 0,1 factor and spin 2,3 factor
    int gamma5;                      // flip the sign of spins 2,3 of the result
};

__host__ __device__ __forceinline__ int round_up(int n, int m) { return (n + m - 1) / m * m; }

// ------------------------------------------------------------------------
// field views.  P = storage precision (64, 32, 16); R = compute type.
// ------------------------------------------------------------------------
template <int P>
struct Prec;
template <>
struct Prec<64> {
    using R = double;
};
template <>
struct Prec<32> {
    using R = float;
};
template <>
struct Prec<16> {
    using R = float;
};

template <int P>
struct SpinorPtr {
    void* data;    // lanes
    float* norm;   // FP16 only: per-site scale
};

template <int P>
struct SpinorIO;

template <>
struct SpinorIO<64> {
    using R = double;
    static __device__ __forceinline__ void load(const SpinorPtr<64>& f, int stride, int i, Cplx<R> s[12])
    {
        const double2* p = static_cast<const double2*>(f.data);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            double2 v = __ldg(p + (size_t)k * stride + i);
            s[k]      = {v.x, v.y};
        }
    }
    static __device__ __forceinline__ void store(const SpinorPtr<64>& f, int stride, int i, const Cplx<R> s[12])
    {
        double2* p = static_cast<double2*>(f.data);
#pragma unroll
        for (int k = 0; k < 12; ++k) p[(size_t)k * stride + i] = make_double2(s[k].re, s[k].im);
    }
};

template <>
struct SpinorIO<32> {
    using R = float;
    static __device__ __forceinline__ void load(const SpinorPtr<32>& f, int stride, int i, Cplx<R> s[12])
    {
        const float4* p = static_cast<const float4*>(f.data);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float4 v     = __ldg(p + (size_t)k * stride + i);
            s[2 * k]     = {v.x, v.y};
            s[2 * k + 1] = {v.z, v.w};
        }
    }
    static __device__ __forceinline__ void store(const SpinorPtr<32>& f, int stride, int i, const Cplx<R> s[12])
    {
        float4* p = static_cast<float4*>(f.data);
#pragma unroll
        for (int k = 0; k < 6; ++k)
            p[(size_t)k * stride + i] = make_float4(s[2 * k].re, s[2 * k].im, s[2 * k + 1].re, s[2 * k + 1].im);
    }
};

// FP16 fixed point: value = q / 32767 * norm, norm = max |real component|.
template <>
struct SpinorIO<16> {
    using R = float;
    static __device__ __forceinline__ void load(const SpinorPtr<16>& f, int stride, int i, Cplx<R> s[12])
    {
        const int4* p    = static_cast<const int4*>(f.data);
        const float sc   = __ldg(f.norm + i) * (1.0f / 32767.0f);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int4 v                = __ldg(p + (size_t)k * stride + i);
            const int w[4]        = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const short lo = (short)(w[j] & 0xffff);
                const short hi = (short)(((unsigned)w[j]) >> 16);
                s[4 * k + j]   = {sc * (float)lo, sc * (float)hi};
            }
        }
    }
    static __device__ __forceinline__ void store(const SpinorPtr<16>& f, int stride, int i, const Cplx<R> s[12])
    {
        float mx = 0.f;
#pragma unroll
        for (int k = 0; k < 12; ++k) mx = fmaxf(mx, fmaxf(fabsf(s[k].re), fabsf(s[k].im)));
        const float inv = mx > 0.f ? 32767.0f / mx : 0.f;
        int4* p         = static_cast<int4*>(f.data);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int w[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int lo = __float2int_rn(s[4 * k + j].re * inv);
                const int hi = __float2int_rn(s[4 * k + j].im * inv);
                w[j]         = (lo & 0xffff) | (hi << 16);
            }
            p[(size_t)k * stride + i] = make_int4(w[0], w[1], w[2], w[3]);
        }
        f.norm[i] = mx;
    }
};

// ------------------------------------------------------------------------
// gauge links: NL = 9 (18-real) or 6 (12-real) complex lanes per link.
// ------------------------------------------------------------------------
template <int P, int NL>
struct LinkIO;

template <int NL>
struct LinkIO<64, NL> {
    using R = double;
    static __device__ __forceinline__ void load(const void* base, size_t lane_stride, size_t idx, Cplx<R> u[9])
    {
        const double2* p = static_cast<const double2*>(base);
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            double2 v = __ldg(p + k * lane_stride + idx);
            u[k]      = {v.x, v.y};
        }
    }
};

template <int NL>
struct LinkIO<32, NL> {
    using R = float;
    static __device__ __forceinline__ void load(const void* base, size_t lane_stride, size_t idx, Cplx<R> u[9])
    {
        const float2* p = static_cast<const float2*>(base);
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            float2 v = __ldg(p + k * lane_stride + idx);
            u[k]     = {v.x, v.y};
        }
    }
};

// FP16 links: entries of an SU(3) matrix are bounded by 1 in magnitude, so a
// fixed scale of 1/32767 is used (no per-link norm).
template <int NL>
struct LinkIO<16, NL> {
    using R = float;
    static __device__ __forceinline__ void load(const void* base, size_t lane_stride, size_t idx, Cplx<R> u[9])
    {
        const short2* p = static_cast<const short2*>(base);
        const float sc  = 1.0f / 32767.0f;
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            short2 v = __ldg(p + k * lane_stride + idx);
            u[k]     = {sc * (float)v.x, sc * (float)v.y};
        }
    }
};

// Rebuild row 2 of an SU(3) matrix from rows 0 and 1: row2 = conj(row0 x row1).
template <typename R>
__device__ __forceinline__ void reconstruct_row2(Cplx<R> u[9])
{
    // (a x b)_0 = a1 b2 - a2 b1, etc.
    Cplx<R> c0 = cmul(u[1], u[5]) - cmul(u[2], u[4]);
    Cplx<R> c1 = cmul(u[2], u[3]) - cmul(u[0], u[5]);
    Cplx<R> c2 = cmul(u[0], u[4]) - cmul(u[1], u[3]);
    u[6]       = {c0.re, -c0.im};
    u[7]       = {c1.re, -c1.im};
    u[8]       = {c2.re, -c2.im};
}

}  // namespace c2q
