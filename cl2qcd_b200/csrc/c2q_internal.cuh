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
//     FP32 and FP16 spinors (and their links) pair the sites i and i + Seo/2
//     in one "slot" (pack.cuh): FP32 12 float4 lanes, FP16 6 uint4 lanes of
//     16-bit fixed point with a per-site float norm (max |component|);
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

#include <utility>

namespace c2q {

// ---------------------------------------------------- dependent launches
// The kernels of the solver loops are launched with programmatic stream
// serialization: the next kernel on the stream may be scheduled while this one
// drains (its last wave, the last block's reduction finisher), and it waits on
// the device, at entry, until this one has completed and its writes are
// visible.  pdl_enter() is that wait (a no-op for an ordinary launch) followed
// by the signal that lets the next kernel be scheduled once every block of
// this one is running.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// Launch `kern` (whose blocks begin with pdl_enter) on stream s, as a
// dependent launch when pdl is set and s is not being captured into a graph
// (graph-replayed iterations of small lattices ran slower with the
// programmatic edges than with plain ones: 8^4 FP64 CG, 206-211 against
// 225-231 solves/s).
template <typename... K, typename... A>
inline cudaError_t launch_dep(bool pdl, void (*kern)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              A&&... args)
{
    if (pdl) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) pdl = false;
    }
    if (!pdl) {
        kern<<<grid, block, smem, s>>>(std::forward<A>(args)...);
        return cudaGetLastError();
    }
    cudaLaunchAttribute at[1];
    at[0].id                                         = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg                           = {};
    cfg.gridDim                                      = grid;
    cfg.blockDim                                     = block;
    cfg.dynamicSmemBytes                             = smem;
    cfg.stream                                       = s;
    cfg.attrs                                        = at;
    cfg.numAttrs                                     = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

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

// fused multiply-add in the compute type
__device__ __forceinline__ float fmad(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmad(double a, double b, double c) { return fma(a, b, c); }

// acc += a * b as four FMAs (a sum of complex products written as `s + a*b`
// would cost a multiply, an FMA and an add per real component)
template <typename R>
__device__ __forceinline__ void cmac(Cplx<R>& acc, Cplx<R> a, Cplx<R> b)
{
    acc.re = fmad(a.re, b.re, acc.re);
    acc.re = fmad(-a.im, b.im, acc.re);
    acc.im = fmad(a.re, b.im, acc.im);
    acc.im = fmad(a.im, b.re, acc.im);
}
// acc += conj(a) * b
template <typename R>
__device__ __forceinline__ void cmacc(Cplx<R>& acc, Cplx<R> a, Cplx<R> b)
{
    acc.re = fmad(a.re, b.re, acc.re);
    acc.re = fmad(a.im, b.im, acc.re);
    acc.im = fmad(a.re, b.im, acc.im);
    acc.im = fmad(-a.im, b.re, acc.im);
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

// Hop coefficients of one dslash launch.  Each hop is weighted by a phase
// (boundary phase e^{+/- i theta pi / N}, times the chemical-potential factor
// on T links): phase[mu][0] forward, phase[mu][1] backward.  The common factor
// -kappa (the kernel's overall sign; times the link dequantisation scale for
// FP16 links) is applied once per site, in the epilogue.  Bit 2*mu+dir of
// real_mask is set when that phase is real.
struct HopCoef {
    double re[4][2], im[4][2];
    double scale;
    unsigned real_mask;
};

// Epilogue applied to the hopping sum h at each output site.
enum Epilogue : int {
    EPI_PLAIN = 0,  // out = h                                  (dslash_eo)
    EPI_DIAG  = 1,  // out = diag(f1,f2) h                      (dslash_AND_M_tm_inverse_sitediagonal)
    EPI_AXPY  = 2,  // out = [g5] (diag(f1,f2) x - h)            (Aee tail, saxpy[_AND_gamma5])
};

// Optional reduction fused into a sweep: <y, out> or |out|^2.
// DOT_CGR (paired-site sweeps only): the CG residual update fused into the
// sweep -- r -= alpha out with r the FP32 field passed as y and alpha from the
// solver scalars, |r|^2 reduced; out itself is not stored.
// DOT_XUPD (paired-site EPI_PLAIN / EPI_DIAG sweeps only): no reduction; the
// CG solution update x += alpha p rides along, p the field passed as x (same
// precision as the sweep) and x the FP32 field passed as y, at the output slot.
enum DotMode : int { DOT_NONE = 0, DOT_Y = 1, DOT_SELF = 2, DOT_CGR = 3, DOT_XUPD = 4 };

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
    int half = 0;  // FP32 / FP16: H = Seo/2, the number of site pairs (slots)
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

// Per-site access to the paired-site ("slot") layout of the FP32 and FP16
// fields (pack.cuh): eo site i is half h = (i >= H) of slot j = i - h H, and
// its two words sit at offset h inside each pair.  The hot kernels work on
// whole slots; these accessors serve conversions and the generic BLAS.
__device__ __forceinline__ int slot_of(int i, int half, int* h)
{
    *h = i >= half;
    return i - (*h) * half;
}

template <>
struct SpinorIO<32> {
    using R = float;
    static __device__ __forceinline__ void load(const SpinorPtr<32>& f, int stride, int i, Cplx<R> s[12])
    {
        int h;
        const int j     = slot_of(i, f.half, &h);
        const float* p  = static_cast<const float*>(f.data) + (size_t)j * 4 + h;
        const size_t ls = (size_t)(stride >> 1) * 4;
#pragma unroll
        for (int k = 0; k < 12; ++k) s[k] = {__ldg(p + k * ls), __ldg(p + k * ls + 2)};
    }
    static __device__ __forceinline__ void store(const SpinorPtr<32>& f, int stride, int i, const Cplx<R> s[12])
    {
        int h;
        const int j     = slot_of(i, f.half, &h);
        float* p        = static_cast<float*>(f.data) + (size_t)j * 4 + h;
        const size_t ls = (size_t)(stride >> 1) * 4;
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            p[k * ls]     = s[k].re;
            p[k * ls + 2] = s[k].im;
        }
    }
};

// FP16 fixed point (16-bit integers with a per-site scale): a real component
// v of a site whose largest |component| is `norm` is stored as the biased
// 16-bit word u = q + 32768, q = rint(v * 32767 / norm) in [-32767, 32767].
// Decoding is exact and avoids the int->float conversion unit: one byte
// permute builds the float 2^23 + u, one add subtracts 2^23 + 32768 (= q).
__device__ __forceinline__ float dq_lo(unsigned w)
{
    return __int_as_float(__byte_perm(w, 0x4B000000u, 0x7610)) - 8421376.0f;
}
__device__ __forceinline__ float dq_hi(unsigned w)
{
    return __int_as_float(__byte_perm(w, 0x4B000000u, 0x7632)) - 8421376.0f;
}
__device__ __forceinline__ unsigned eq_pair(float re, float im, float inv)
{
    const int lo = __float2int_rn(re * inv) + 32768;
    const int hi = __float2int_rn(im * inv) + 32768;
    return (unsigned)(lo & 0xffff) | ((unsigned)hi << 16);
}

template <>
struct SpinorIO<16> {
    using R = float;
    // word of component k of (slot j, half h): lane k/2, position 2 (k & 1) + h
    static __device__ __forceinline__ void load(const SpinorPtr<16>& f, int stride, int i, Cplx<R> s[12])
    {
        int h;
        const int j       = slot_of(i, f.half, &h);
        const unsigned* p = static_cast<const unsigned*>(f.data) + (size_t)j * 4 + h;
        const size_t ls   = (size_t)(stride >> 1) * 4;
        const float sc    = __ldg(f.norm + 2 * j + h) * (1.0f / 32767.0f);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const unsigned w = __ldg(p + (k >> 1) * ls + 2 * (k & 1));
            s[k]             = {sc * dq_lo(w), sc * dq_hi(w)};
        }
    }
    static __device__ __forceinline__ void store(const SpinorPtr<16>& f, int stride, int i, const Cplx<R> s[12])
    {
        float mx = 0.f;
#pragma unroll
        for (int k = 0; k < 12; ++k) mx = fmaxf(mx, fmaxf(fabsf(s[k].re), fabsf(s[k].im)));
        const float inv = mx > 0.f ? 32767.0f / mx : 0.f;
        int h;
        const int j     = slot_of(i, f.half, &h);
        unsigned* p     = static_cast<unsigned*>(f.data) + (size_t)j * 4 + h;
        const size_t ls = (size_t)(stride >> 1) * 4;
#pragma unroll
        for (int k = 0; k < 12; ++k) p[(k >> 1) * ls + 2 * (k & 1)] = eq_pair(s[k].re, s[k].im, inv);
        f.norm[2 * j + h] = mx;
    }
};

// ------------------------------------------------------------------------
// FP64 gauge links: NL = 9 (18-real) or 6 (12-real) complex lanes per link.
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

// Rebuild row 2 of an SU(3) matrix from rows 0 and 1: row2 = conj(row0 x row1).
// With rows held in units of a scale s (U = s Q), row 2 in the same units is
// s * conj(q0 x q1): pass `s` for quantised links, 1 otherwise.
template <typename R>
__device__ __forceinline__ void reconstruct_row2(Cplx<R> u[9], R s = R(1))
{
    // (a x b)_0 = a1 b2 - a2 b1, etc., as FMA chains
    const Cplx<R> m2 = {-u[2].re, -u[2].im}, m0 = {-u[0].re, -u[0].im}, m1 = {-u[1].re, -u[1].im};
    Cplx<R> c0 = cmul(u[1], u[5]);
    cmac(c0, m2, u[4]);
    Cplx<R> c1 = cmul(u[2], u[3]);
    cmac(c1, m0, u[5]);
    Cplx<R> c2 = cmul(u[0], u[4]);
    cmac(c2, m1, u[3]);
    u[6]       = {s * c0.re, -s * c0.im};
    u[7]       = {s * c1.re, -s * c1.im};
    u[8]       = {s * c2.re, -s * c2.im};
}

}  // namespace c2q
