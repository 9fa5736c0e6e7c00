/*
 * oracle_inputs.c -- TEST INFRASTRUCTURE ONLY (oracle input generators).
 *
 * The seeded synthetic workload inputs restated in plain C, so that the
 * CPU reference path (and the tests that check it) can build the gauge field
 * and sources of a workload without loading the product library.  The
 * definition is the workload's, shared with the product's host generator
 * (cl2qcd_b200/csrc/inputs.cpp); the tests assert that both produce
 * bit-identical arrays.
 *
 *   stream(seed, index): SplitMix64 (Steele, Lea, Flood 2014) started at
 *       seed ^ (index * 0x9E3779B97F4A7C15 + 0xD1B54A32D192ED03), one draw
 *       discarded; uniform in (0, 1] from the top 53 bits; normals by the
 *       Box-Muller transform, pairwise.
 *   link l: H traceless Hermitian from 10 normals (diagonal g0..g2 minus
 *       their mean, off-diagonal (g3,g4) (g5,g6) (g7,g8)); U = exp(i eps H)
 *       by scaling and squaring (halve until the Frobenius norm <= 1/4) and a
 *       20-term Taylor series; Gram-Schmidt on rows 0 and 1, row 2 =
 *       conj(row0 x row1).  Matrixsu3[4V] at link mu + 4 site.
 *   source site s: stream(seed ^ 0x5350494E4F52, s); Z2: bit k of one draw
 *       picks -1/sqrt2 or +1/sqrt2 for real k; Gaussian: 12 normal pairs.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define C2QO_API __attribute__((visibility("default")))

typedef struct {
    uint64_t s;
} sm64;

static uint64_t sm64_next(sm64* r)
{
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ULL);
    z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z          = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static sm64 sm64_stream(uint64_t seed, uint64_t idx)
{
    sm64 r = {seed ^ (idx * 0x9E3779B97F4A7C15ULL + 0xD1B54A32D192ED03ULL)};
    (void)sm64_next(&r);
    return r;
}

static double sm64_uniform(sm64* r) { return ((sm64_next(r) >> 11) + 1) * (1.0 / 9007199254740992.0); }

static void sm64_normal2(sm64* r, double* a, double* b)
{
    const double u1 = sm64_uniform(r);
    const double u2 = sm64_uniform(r);
    const double rad = sqrt(-2.0 * log(u1)), ph = 6.283185307179586 * u2;
    *a = rad * cos(ph);
    *b = rad * sin(ph);
}

typedef struct {
    double re, im;
} cx;

static cx cx_mul(cx a, cx b) { return (cx){a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
static cx cx_add(cx a, cx b) { return (cx){a.re + b.re, a.im + b.im}; }

static void mat_mul(const cx* a, const cx* b, cx* out)
{
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            cx s = {0, 0};
            for (int k = 0; k < 3; ++k) s = cx_add(s, cx_mul(a[3 * r + k], b[3 * k + c]));
            out[3 * r + c] = s;
        }
}

static void mat_exp(const cx* A, cx* out)
{
    double nrm = 0;
    for (int k = 0; k < 9; ++k) nrm += A[k].re * A[k].re + A[k].im * A[k].im;
    nrm   = sqrt(nrm);
    int s = 0;
    while (nrm > 0.25 && s < 30) {
        nrm *= 0.5;
        ++s;
    }
    const double scale = ldexp(1.0, -s);
    cx X[9], term[9], tmp[9];
    for (int k = 0; k < 9; ++k) X[k] = (cx){A[k].re * scale, A[k].im * scale};
    for (int k = 0; k < 9; ++k) {
        out[k]  = (cx){k % 4 == 0 ? 1.0 : 0.0, 0.0};
        term[k] = out[k];
    }
    for (int n = 1; n <= 20; ++n) {
        mat_mul(term, X, tmp);
        for (int k = 0; k < 9; ++k) {
            term[k] = (cx){tmp[k].re / n, tmp[k].im / n};
            out[k]  = cx_add(out[k], term[k]);
        }
    }
    for (int q = 0; q < s; ++q) {
        mat_mul(out, out, tmp);
        memcpy(out, tmp, sizeof tmp);
    }
}

static void gram_schmidt_rows(cx* u)
{
    double n0 = 0;
    for (int c = 0; c < 3; ++c) n0 += u[c].re * u[c].re + u[c].im * u[c].im;
    n0 = 1.0 / sqrt(n0);
    for (int c = 0; c < 3; ++c) u[c] = (cx){u[c].re * n0, u[c].im * n0};
    cx d = {0, 0};  /* <row0, row1> */
    for (int c = 0; c < 3; ++c) d = cx_add(d, cx_mul((cx){u[c].re, -u[c].im}, u[3 + c]));
    for (int c = 0; c < 3; ++c)
        u[3 + c] = (cx){u[3 + c].re - (d.re * u[c].re - d.im * u[c].im),
                        u[3 + c].im - (d.re * u[c].im + d.im * u[c].re)};
    double n1 = 0;
    for (int c = 0; c < 3; ++c) n1 += u[3 + c].re * u[3 + c].re + u[3 + c].im * u[3 + c].im;
    n1 = 1.0 / sqrt(n1);
    for (int c = 0; c < 3; ++c) u[3 + c] = (cx){u[3 + c].re * n1, u[3 + c].im * n1};
    const cx* a = u;
    const cx* b = u + 3;
    const cx c0 = cx_add(cx_mul(a[1], b[2]), cx_mul((cx){-a[2].re, -a[2].im}, b[1]));
    const cx c1 = cx_add(cx_mul(a[2], b[0]), cx_mul((cx){-a[0].re, -a[0].im}, b[2]));
    const cx c2 = cx_add(cx_mul(a[0], b[1]), cx_mul((cx){-a[1].re, -a[1].im}, b[0]));
    u[6] = (cx){c0.re, -c0.im};
    u[7] = (cx){c1.re, -c1.im};
    u[8] = (cx){c2.re, -c2.im};
}

C2QO_API int c2qo_gauge_generate(double* aos, int ns, int nt, double eps, unsigned long long seed)
{
    if (!aos || ns < 2 || nt < 2) return -5;
    const long long nlinks = 4LL * ns * ns * ns * nt;
#pragma omp parallel for schedule(static)
    for (long long l = 0; l < nlinks; ++l) {
        sm64 rng = sm64_stream(seed, (uint64_t)l);
        double g[10];
        for (int k = 0; k < 10; k += 2) sm64_normal2(&rng, &g[k], &g[k + 1]);
        const double tr = (g[0] + g[1] + g[2]) / 3.0;
        cx H[9];
        H[0] = (cx){g[0] - tr, 0};
        H[4] = (cx){g[1] - tr, 0};
        H[8] = (cx){g[2] - tr, 0};
        H[1] = (cx){g[3], g[4]};
        H[3] = (cx){g[3], -g[4]};
        H[2] = (cx){g[5], g[6]};
        H[6] = (cx){g[5], -g[6]};
        H[5] = (cx){g[7], g[8]};
        H[7] = (cx){g[7], -g[8]};
        cx A[9], U[9];
        for (int k = 0; k < 9; ++k) A[k] = (cx){-eps * H[k].im, eps * H[k].re};
        mat_exp(A, U);
        gram_schmidt_rows(U);
        double* dst = aos + 18 * l;
        for (int k = 0; k < 9; ++k) {
            dst[2 * k]     = U[k].re;
            dst[2 * k + 1] = U[k].im;
        }
    }
    return 0;
}

C2QO_API int c2qo_source_generate(double* aos, size_t n_sites, int kind, unsigned long long seed)
{
    if (!aos || (kind != 0 && kind != 1)) return -5;
    const double h = 1.0 / sqrt(2.0);
#pragma omp parallel for schedule(static)
    for (long long s = 0; s < (long long)n_sites; ++s) {
        sm64 rng    = sm64_stream(seed ^ 0x5350494E4F52ULL, (uint64_t)s);
        double* dst = aos + 24 * s;
        if (kind == 0) {
            const uint64_t bits = sm64_next(&rng);
            for (int k = 0; k < 24; ++k) dst[k] = ((bits >> k) & 1) ? -h : h;
        } else {
            for (int k = 0; k < 24; k += 2) sm64_normal2(&rng, &dst[k], &dst[k + 1]);
        }
    }
    return 0;
}
