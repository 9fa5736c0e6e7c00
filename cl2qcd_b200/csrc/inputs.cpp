// inputs.cpp -- seeded synthetic inputs in the reference's host layouts.
//
// Gauge links: U = exp(i eps H), H traceless Hermitian 3x3 with N(0,1)
// entries (off-diagonal complex N(0,1), real diagonal N(0,1), trace removed),
// exponentiated by scaling-and-squaring Taylor series in FP64 and then
// reunitarised in FP64 (Gram-Schmidt on rows 0 and 1, row 2 = conj(row0 x row1),
// so det U = 1).
//
// Random numbers: counter-based.  Stream (seed, index) is SplitMix64
// (Steele, Lea, Flood 2014) started at seed ^ (index * golden ratio); normals
// come from the Box-Muller transform.  Every link / site has its own stream,
// so generation is parallel and independent of the thread count.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/cl2qcd_b200.h"

namespace {

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed, uint64_t idx) : s(seed ^ (idx * 0x9E3779B97F4A7C15ULL + 0xD1B54A32D192ED03ULL))
    {
        next();
    }
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z          = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    // uniform in (0, 1]
    double uniform() { return ((next() >> 11) + 1) * (1.0 / 9007199254740992.0); }
    void normal2(double* a, double* b)
    {
        const double u1 = uniform(), u2 = uniform();
        const double r = std::sqrt(-2.0 * std::log(u1)), ph = 6.283185307179586 * u2;
        *a             = r * std::cos(ph);
        *b             = r * std::sin(ph);
    }
};

struct C {
    double re, im;
};
inline C mul(C a, C b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C add(C a, C b) { return {a.re + b.re, a.im + b.im}; }

void matmul(const C a[9], const C b[9], C out[9])
{
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            C s{0, 0};
            for (int k = 0; k < 3; ++k) s = add(s, mul(a[3 * r + k], b[3 * k + c]));
            out[3 * r + c] = s;
        }
}

// exp(A) for a 3x3 complex A by scaling and squaring + 20-term Taylor series
void expm3(const C A[9], C out[9])
{
    double nrm = 0;
    for (int k = 0; k < 9; ++k) nrm += A[k].re * A[k].re + A[k].im * A[k].im;
    nrm       = std::sqrt(nrm);
    int s     = 0;
    while (nrm > 0.25 && s < 30) {
        nrm *= 0.5;
        ++s;
    }
    const double scale = std::ldexp(1.0, -s);
    C X[9], term[9], tmp[9];
    for (int k = 0; k < 9; ++k) X[k] = {A[k].re * scale, A[k].im * scale};
    for (int k = 0; k < 9; ++k) {
        out[k]  = {k % 4 == 0 ? 1.0 : 0.0, 0.0};
        term[k] = out[k];
    }
    for (int n = 1; n <= 20; ++n) {
        matmul(term, X, tmp);
        for (int k = 0; k < 9; ++k) {
            term[k] = {tmp[k].re / n, tmp[k].im / n};
            out[k]  = add(out[k], term[k]);
        }
    }
    for (int q = 0; q < s; ++q) {
        matmul(out, out, tmp);
        memcpy(out, tmp, sizeof tmp);
    }
}

void reunitarise(C u[9])
{
    // row 0 normalised
    double n0 = 0;
    for (int c = 0; c < 3; ++c) n0 += u[c].re * u[c].re + u[c].im * u[c].im;
    n0 = 1.0 / std::sqrt(n0);
    for (int c = 0; c < 3; ++c) u[c] = {u[c].re * n0, u[c].im * n0};
    // row 1 orthogonalised against row 0, normalised
    C d{0, 0};
    for (int c = 0; c < 3; ++c) d = add(d, mul({u[c].re, -u[c].im}, u[3 + c]));
    for (int c = 0; c < 3; ++c) u[3 + c] = {u[3 + c].re - (d.re * u[c].re - d.im * u[c].im),
                                            u[3 + c].im - (d.re * u[c].im + d.im * u[c].re)};
    double n1 = 0;
    for (int c = 0; c < 3; ++c) n1 += u[3 + c].re * u[3 + c].re + u[3 + c].im * u[3 + c].im;
    n1 = 1.0 / std::sqrt(n1);
    for (int c = 0; c < 3; ++c) u[3 + c] = {u[3 + c].re * n1, u[3 + c].im * n1};
    // row 2 = conj(row0 x row1)
    const C* a = u;
    const C* b = u + 3;
    C c0       = add(mul(a[1], b[2]), mul({-a[2].re, -a[2].im}, b[1]));
    C c1       = add(mul(a[2], b[0]), mul({-a[0].re, -a[0].im}, b[2]));
    C c2       = add(mul(a[0], b[1]), mul({-a[1].re, -a[1].im}, b[0]));
    u[6]       = {c0.re, -c0.im};
    u[7]       = {c1.re, -c1.im};
    u[8]       = {c2.re, -c2.im};
}

}  // namespace

extern "C" {

C2Q_EXPORT int c2q_gauge_generate(double* aos, int ns, int nt, double eps, unsigned long long seed)
{
    if (!aos || ns < 2 || nt < 2) return C2Q_BAD_ARG;
    const long long nlinks = 4LL * ns * ns * ns * nt;
#pragma omp parallel for schedule(static)
    for (long long l = 0; l < nlinks; ++l) {
        SplitMix64 rng(seed, (uint64_t)l);
        double g[10];
        for (int k = 0; k < 10; k += 2) rng.normal2(&g[k], &g[k + 1]);
        // H: real diagonal g0..g2 (trace removed), off-diagonal complex (g3,g4) (g5,g6) (g7,g8)
        const double tr = (g[0] + g[1] + g[2]) / 3.0;
        C H[9];
        H[0] = {g[0] - tr, 0};
        H[4] = {g[1] - tr, 0};
        H[8] = {g[2] - tr, 0};
        H[1] = {g[3], g[4]};
        H[3] = {g[3], -g[4]};
        H[2] = {g[5], g[6]};
        H[6] = {g[5], -g[6]};
        H[5] = {g[7], g[8]};
        H[7] = {g[7], -g[8]};
        C A[9], U[9];
        for (int k = 0; k < 9; ++k) A[k] = {-eps * H[k].im, eps * H[k].re};  // i eps H
        expm3(A, U);
        reunitarise(U);
        double* dst = aos + 18 * l;
        for (int k = 0; k < 9; ++k) {
            dst[2 * k]     = U[k].re;
            dst[2 * k + 1] = U[k].im;
        }
    }
    return C2Q_OK;
}

C2Q_EXPORT int c2q_source_generate(double* aos, size_t n_sites, int kind, unsigned long long seed)
{
    if (!aos || (kind != 0 && kind != 1)) return C2Q_BAD_ARG;
    const double h = 1.0 / std::sqrt(2.0);
#pragma omp parallel for schedule(static)
    for (long long s = 0; s < (long long)n_sites; ++s) {
        SplitMix64 rng(seed ^ 0x5350494E4F52ULL, (uint64_t)s);
        double* dst = aos + 24 * s;
        if (kind == 0) {
            const uint64_t bits = rng.next();
            for (int k = 0; k < 24; ++k) dst[k] = ((bits >> k) & 1) ? -h : h;
        } else {
            for (int k = 0; k < 24; k += 2) rng.normal2(&dst[k], &dst[k + 1]);
        }
    }
    return C2Q_OK;
}

}  // extern "C"
