/*
 * oracle_kernels_port.c -- TEST INFRASTRUCTURE ONLY (oracle, "port" backend).
 *
 * This project's own CPU restatement of the reference's hot-path kernels, in
 * the reference's host data formats (see oracle_kernels.h).  It is the checker
 * the CUDA path is compared against; it is never linked into the product.
 *
 * Conventions restated here (each cites the reference line it follows):
 *  - site index s = x + NS*y + NS^2*z + NS^3*t; eo index = s/2; a site is
 *    "even" when x+y+z+t is even (ocl_kernel/operations_geometry.cl:97-156,
 *    297-300, 378-385).  Because NS is even, the two sites 2i and 2i+1 differ
 *    only in x and have opposite parity, so the parity-p site of eo index i is
 *    whichever of 2i, 2i+1 has parity p.
 *  - dslash_eo(evenodd): evenodd == ODD(1) writes the even sites, EVEN(0) the
 *    odd sites (ocl_kernel/fermionmatrix_eo_dslash.cl:50-58).
 *  - out(x) = -sum_mu [ k_mu^+ (1 - g_mu) U_mu(x) psi(x+mu)
 *                      + k_mu^- (1 + g_mu) U_mu(x-mu)^dagger psi(x-mu) ],
 *    k^+ = kappa e^{+i theta pi/N}, k^- = kappa e^{-i theta pi/N}; on T links
 *    the chemical potential multiplies k^+ by e^{cp_re + i cp_im} and k^- by
 *    e^{-cp_re - i cp_im} (ocl_kernel/fermionmatrix_eo.cl:30-253,
 *    hardware/code/opencl_module.cpp:113-124,190-203).
 *  - gamma basis: each projector 1 -/+ g_mu is rank two.  With upper spin rows
 *    a = 0, 1 it is written h_a = psi_a + c psi_p (c -> -c for 1 + g_mu), and
 *    the lower rows receive conj(c) * (U h_a) in row p.  The (p, c) pairs for
 *    the forward hop are read off fermionmatrix_eo.cl:56-136:
 *        T: (2, 1), (3, 1)     X: (3, i), (2, i)
 *        Y: (3, 1), (2, -1)    Z: (2, i), (3, -i)
 *  - g5 = diag(1, 1, -1, -1) in spin (ocl_kernel/fermionmatrix.cl:41-49);
 *    M_diag_tm_local multiplies spins 0,1 by f1 and spins 2,3 by f2
 *    (ocl_kernel/fermionmatrix.cl:28-36).
 *  - saxpy(out, a, x, y) = y - a x (ocl_kernel/spinorfield_eo_saxpy.cl:20-37);
 *    saxsbypz = a x + b y + z (spinorfield_eo_saxsbypz.cl:22-43);
 *    scalar product = sum conj(x) y (ocl_kernel/operations_su3vec.cl:40-48).
 *  - cold eo field: every component 1/sqrt(12 V) real
 *    (ocl_kernel/spinorfield_eo_cold.cl:22-33).
 */
#include "oracle_kernels.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PI_REF 3.14159265358979 /* common_header_files/globaldefs.hpp */

static c2qo_lattice g_lat = {4, 4, 0., 0., 0, 0, 0., 0.};
/* hop coefficients: [dir][0 = forward, 1 = backward] as (re, im) */
static double g_hop[4][2][2];
/* the plain boundary phase e^{i theta pi / N} per direction, and the chemical
 * potential factors of the T link in the fermion force (forward, backward) */
static double g_phase[4][2];
static double g_cp_link[2][2];

static double as_build_option(double v)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%.16g", v);
    return strtod(buf, NULL);
}

void ok_set_lattice(const c2qo_lattice* lat)
{
    g_lat = *lat;
    for (int mu = 0; mu < 4; ++mu) {
        const double ang = mu == 0 ? (lat->theta_t * PI_REF) / (double)lat->nt : (lat->theta_s * PI_REF) / (double)lat->ns;
        double c = as_build_option(cos(ang)), s = as_build_option(sin(ang));
        g_hop[mu][0][0] = c;
        g_hop[mu][0][1] = s;
        g_hop[mu][1][0] = c;
        g_hop[mu][1][1] = -s;
        g_phase[mu][0]  = c;
        g_phase[mu][1]  = s;
    }
    {
        /* hardware/code/opencl_module.cpp:113-124: EXPCPR, MEXPCPR, COSCPI, SINCPI */
        const double er  = lat->use_cp_re ? as_build_option(exp(lat->cp_re)) : 1.;
        const double emr = lat->use_cp_re ? as_build_option(exp(-lat->cp_re)) : 1.;
        const double cc  = lat->use_cp_im ? as_build_option(cos(lat->cp_im)) : 1.;
        const double ss  = lat->use_cp_im ? as_build_option(sin(lat->cp_im)) : 0.;
        g_cp_link[0][0] = er * cc;
        g_cp_link[0][1] = er * ss;
        g_cp_link[1][0] = emr * cc;
        g_cp_link[1][1] = emr * ss;
    }
    if (lat->use_cp_re || lat->use_cp_im) {
        double er = lat->use_cp_re ? exp(lat->cp_re) : 1., emr = lat->use_cp_re ? exp(-lat->cp_re) : 1.;
        double cc = lat->use_cp_im ? cos(lat->cp_im) : 1., ss = lat->use_cp_im ? sin(lat->cp_im) : 0.;
        /* forward: k * e^{cp_re} * e^{i cp_im}; backward: k * e^{-cp_re} * e^{-i cp_im} */
        double f_re = er * cc, f_im = er * ss, b_re = emr * cc, b_im = -emr * ss;
        double* fw = g_hop[0][0];
        double* bw = g_hop[0][1];
        double r0 = fw[0] * f_re - fw[1] * f_im, i0 = fw[0] * f_im + fw[1] * f_re;
        double r1 = bw[0] * b_re - bw[1] * b_im, i1 = bw[0] * b_im + bw[1] * b_re;
        fw[0] = r0;
        fw[1] = i0;
        bw[0] = r1;
        bw[1] = i1;
    }
}
const c2qo_lattice* ok_lattice(void) { return &g_lat; }
size_t ok_vol(void) { return (size_t)g_lat.ns * g_lat.ns * g_lat.ns * g_lat.nt; }
size_t ok_seo(void) { return ok_vol() / 2; }
const char* ok_backend_name(void) { return "port"; }

/* ---------------- small complex helpers on (re,im) double pairs ---------------- */
typedef struct {
    double r, i;
} cplx;
static inline cplx cmul(cplx a, cplx b) { return (cplx){a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
static inline cplx cadd(cplx a, cplx b) { return (cplx){a.r + b.r, a.i + b.i}; }
static inline cplx cconj(cplx a) { return (cplx){a.r, -a.i}; }
static inline cplx cld(const double* p) { return (cplx){p[0], p[1]}; }

/* ---------------- geometry ---------------- */
static inline void site_coords(size_t s, int c[4])
{
    const size_t ns = (size_t)g_lat.ns;
    c[1] = (int)(s % ns);
    c[2] = (int)((s / ns) % ns);
    c[3] = (int)((s / (ns * ns)) % ns);
    c[0] = (int)(s / (ns * ns * ns));
}
static inline size_t site_index(const int c[4])
{
    const size_t ns = (size_t)g_lat.ns;
    return (size_t)c[1] + ns * ((size_t)c[2] + ns * ((size_t)c[3] + ns * (size_t)c[0]));
}
/* parity-p site that carries eo index i */
static inline size_t eo_site(size_t i, int p)
{
    int c[4];
    site_coords(2 * i, c);
    int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    return par == p ? 2 * i : 2 * i + 1;
}
static inline size_t shift_site(size_t s, int mu, int dir)
{
    int c[4];
    site_coords(s, c);
    const int n = mu == 0 ? g_lat.nt : g_lat.ns;
    c[mu]       = (c[mu] + dir + n) % n;
    return site_index(c);
}

/* forward-hop projector table: for mu and upper row a, partner row p and coefficient c */
static const int PROJ_P[4][2] = {{2, 3}, {3, 2}, {3, 2}, {2, 3}};
static const double PROJ_C[4][2][2] = {
    {{1., 0.}, {1., 0.}},  /* T */
    {{0., 1.}, {0., 1.}},  /* X */
    {{1., 0.}, {-1., 0.}}, /* Y */
    {{0., 1.}, {0., -1.}}, /* Z */
};

/* acc += k * [(1 -/+ g_mu) applied through U (or U^dagger)] to the spinor at psi */
static void hop_accumulate(double acc[24], const double* psi, const double* U, int mu, int backward, cplx k)
{
    for (int a = 0; a < 2; ++a) {
        const int p = PROJ_P[mu][a];
        cplx c      = {PROJ_C[mu][a][0], PROJ_C[mu][a][1]};
        if (backward) c = (cplx){-c.r, -c.i};
        cplx h[3], uh[3];
        for (int col = 0; col < 3; ++col) h[col] = cadd(cld(psi + 6 * a + 2 * col), cmul(c, cld(psi + 6 * p + 2 * col)));
        for (int r = 0; r < 3; ++r) {
            cplx s = {0., 0.};
            for (int col = 0; col < 3; ++col) {
                cplx u = backward ? cconj(cld(U + 2 * (3 * col + r))) : cld(U + 2 * (3 * r + col));
                s      = cadd(s, cmul(u, h[col]));
            }
            uh[r] = cmul(k, s);
        }
        const cplx d = cconj(c);
        for (int r = 0; r < 3; ++r) {
            acc[6 * a + 2 * r] += uh[r].r;
            acc[6 * a + 2 * r + 1] += uh[r].i;
            cplx lo = cmul(d, uh[r]);
            acc[6 * p + 2 * r] += lo.r;
            acc[6 * p + 2 * r + 1] += lo.i;
        }
    }
}

/* the hopping sum -sum_mu(...) at full-lattice site s; nb(site) gives the input spinor */
static void hopping_at(double out[24], size_t s, const double* gauge, double kappa, const double* in_field, int eo)
{
    double acc[24] = {0};
    for (int mu = 0; mu < 4; ++mu) {
        size_t sp = shift_site(s, mu, +1), sm = shift_site(s, mu, -1);
        const double* psi_p = in_field + 24 * (eo ? sp / 2 : sp);
        const double* psi_m = in_field + 24 * (eo ? sm / 2 : sm);
        cplx kf             = {kappa * g_hop[mu][0][0], kappa * g_hop[mu][0][1]};
        cplx kb             = {kappa * g_hop[mu][1][0], kappa * g_hop[mu][1][1]};
        hop_accumulate(acc, psi_p, gauge + 18 * (mu + 4 * s), mu, 0, kf);
        hop_accumulate(acc, psi_m, gauge + 18 * (mu + 4 * sm), mu, 1, kb);
    }
    for (int k = 0; k < 24; ++k) out[k] = -acc[k];
}

static void diag_factors(double mubar, int which, cplx* f1, cplx* f2, double* scale)
{
    *scale = 1.;
    switch (which) {
        case C2QO_DIAG_M: *f1 = (cplx){1., mubar}; *f2 = (cplx){1., -mubar}; break;
        case C2QO_DIAG_MINV: *f1 = (cplx){1., -mubar}; *f2 = (cplx){1., mubar}; *scale = 1. / (1. + mubar * mubar); break;
        case C2QO_DIAG_M_MINUS: *f1 = (cplx){1., -mubar}; *f2 = (cplx){1., mubar}; break;
        case C2QO_DIAG_MINV_MINUS: *f1 = (cplx){1., mubar}; *f2 = (cplx){1., -mubar}; *scale = 1. / (1. + mubar * mubar); break;
        case C2QO_DIAG_M_G5: *f1 = (cplx){1., mubar}; *f2 = (cplx){-1., mubar}; break;
        case C2QO_DIAG_M_MINUS_G5: *f1 = (cplx){1., -mubar}; *f2 = (cplx){-1., -mubar}; break;
        default: abort();
    }
}

static void diag_site(double* o, const double* in, cplx f1, cplx f2, double scale)
{
    double tmp[24];
    for (int sp = 0; sp < 4; ++sp)
        for (int col = 0; col < 3; ++col) {
            cplx v = cmul(sp < 2 ? f1 : f2, cld(in + 6 * sp + 2 * col));
            tmp[6 * sp + 2 * col]     = v.r * scale;
            tmp[6 * sp + 2 * col + 1] = v.i * scale;
        }
    memcpy(o, tmp, sizeof tmp);
}

void ok_dslash_eo(double* out, const double* in, const double* gauge, int evenodd, double kappa)
{
    const long n  = (long)ok_seo();
    const int par = evenodd == 1 ? 0 : 1;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) hopping_at(out + 24 * i, eo_site((size_t)i, par), gauge, kappa, in, 1);
}

void ok_dslash_tm_inv_eo(double* out, const double* in, const double* gauge, int evenodd, double kappa, double mubar,
                         int minus)
{
    const long n  = (long)ok_seo();
    const int par = evenodd == 1 ? 0 : 1;
    cplx f1, f2;
    double scale;
    diag_factors(mubar, minus ? C2QO_DIAG_MINV_MINUS : C2QO_DIAG_MINV, &f1, &f2, &scale);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        double h[24];
        hopping_at(h, eo_site((size_t)i, par), gauge, kappa, in, 1);
        diag_site(out + 24 * i, h, f1, f2, scale);
    }
}

void ok_tm_diag(double* out, const double* in, double mubar, int which)
{
    cplx f1, f2;
    double scale;
    diag_factors(mubar, which, &f1, &f2, &scale);
    const long n = (long)ok_seo();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) diag_site(out + 24 * i, in + 24 * i, f1, f2, scale);
}

void ok_gamma5_eo(double* inout)
{
    const long n = (long)ok_seo();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i)
        for (int k = 12; k < 24; ++k) inout[24 * i + k] = -inout[24 * i + k];
}

void ok_gamma5_full(double* inout)
{
    const long n = (long)ok_vol();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i)
        for (int k = 12; k < 24; ++k) inout[24 * i + k] = -inout[24 * i + k];
}

static void saxpy_impl(double* out, c2qo_complex alpha, const double* x, const double* y, int g5)
{
    const long n = (long)ok_seo() * 12;
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; ++j) {
        cplx ax   = cmul((cplx){alpha.re, alpha.im}, cld(x + 2 * j));
        double sg = (g5 && (j % 12) >= 6) ? -1. : 1.;
        out[2 * j]     = sg * (y[2 * j] - ax.r);
        out[2 * j + 1] = sg * (y[2 * j + 1] - ax.i);
    }
}
void ok_saxpy(double* out, c2qo_complex alpha, const double* x, const double* y) { saxpy_impl(out, alpha, x, y, 0); }
void ok_saxpy_gamma5(double* out, c2qo_complex alpha, const double* x, const double* y)
{
    saxpy_impl(out, alpha, x, y, 1);
}

void ok_sax(double* out, c2qo_complex alpha, const double* x)
{
    const long n = (long)ok_seo() * 12;
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; ++j) {
        cplx ax        = cmul((cplx){alpha.re, alpha.im}, cld(x + 2 * j));
        out[2 * j]     = ax.r;
        out[2 * j + 1] = ax.i;
    }
}

void ok_saxsbypz(double* out, c2qo_complex alpha, const double* x, c2qo_complex beta, const double* y,
                 const double* z)
{
    const long n = (long)ok_seo() * 12;
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; ++j) {
        cplx ax        = cmul((cplx){alpha.re, alpha.im}, cld(x + 2 * j));
        cplx by        = cmul((cplx){beta.re, beta.im}, cld(y + 2 * j));
        out[2 * j]     = ax.r + by.r + z[2 * j];
        out[2 * j + 1] = ax.i + by.i + z[2 * j + 1];
    }
}

/* Fixed-block two-level sums: deterministic for any thread count. */
#define RBLOCK 512
c2qo_complex ok_scalar_product(const double* x, const double* y)
{
    const long n   = (long)ok_seo();
    const long nb  = (n + RBLOCK - 1) / RBLOCK;
    double* part   = calloc((size_t)(2 * nb), sizeof(double));
#pragma omp parallel for schedule(static)
    for (long b = 0; b < nb; ++b) {
        double re = 0., im = 0.;
        for (long i = b * RBLOCK; i < n && i < (b + 1) * RBLOCK; ++i)
            for (int k = 0; k < 12; ++k) {
                const double* a = x + 24 * i + 2 * k;
                const double* c = y + 24 * i + 2 * k;
                re += a[0] * c[0] + a[1] * c[1];
                im += a[0] * c[1] - a[1] * c[0];
            }
        part[2 * b]     = re;
        part[2 * b + 1] = im;
    }
    c2qo_complex r = {0., 0.};
    for (long b = 0; b < nb; ++b) {
        r.re += part[2 * b];
        r.im += part[2 * b + 1];
    }
    free(part);
    return r;
}

static double sqnorm_n(const double* x, long n)
{
    const long nb = (n + RBLOCK - 1) / RBLOCK;
    double* part  = calloc((size_t)nb, sizeof(double));
#pragma omp parallel for schedule(static)
    for (long b = 0; b < nb; ++b) {
        double s = 0.;
        for (long i = b * RBLOCK; i < n && i < (b + 1) * RBLOCK; ++i)
            for (int k = 0; k < 24; ++k) s += x[24 * i + k] * x[24 * i + k];
        part[b] = s;
    }
    double r = 0.;
    for (long b = 0; b < nb; ++b) r += part[b];
    free(part);
    return r;
}
double ok_squarenorm(const double* x) { return sqnorm_n(x, (long)ok_seo()); }
double ok_squarenorm_full(const double* x) { return sqnorm_n(x, (long)ok_vol()); }

double ok_saxpy_squarenorm(double* out, c2qo_complex alpha, const double* x, const double* y)
{
    ok_saxpy(out, alpha, x, y);
    return ok_squarenorm(out);
}

void ok_zero(double* x) { memset(x, 0, ok_seo() * 24 * sizeof(double)); }
void ok_cold(double* x)
{
    const double norm = 1. / sqrt(12. * (double)ok_vol());
    const long n      = (long)ok_seo() * 12;
    for (long j = 0; j < n; ++j) {
        x[2 * j]     = norm;
        x[2 * j + 1] = 0.;
    }
}
void ok_copy(double* dst, const double* src) { memcpy(dst, src, ok_seo() * 24 * sizeof(double)); }

void ok_convert_to_eo(double* even, double* odd, const double* full)
{
    const long n = (long)ok_seo();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        memcpy(even + 24 * i, full + 24 * eo_site((size_t)i, 0), 24 * sizeof(double));
        memcpy(odd + 24 * i, full + 24 * eo_site((size_t)i, 1), 24 * sizeof(double));
    }
}

void ok_convert_from_eo(double* full, const double* even, const double* odd)
{
    const long n = (long)ok_seo();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        memcpy(full + 24 * eo_site((size_t)i, 0), even + 24 * i, 24 * sizeof(double));
        memcpy(full + 24 * eo_site((size_t)i, 1), odd + 24 * i, 24 * sizeof(double));
    }
}

static void m_tm_full(double* out, const double* in, const double* gauge, double kappa, double mubar, int minus)
{
    cplx f1, f2;
    double scale;
    diag_factors(mubar, minus ? C2QO_DIAG_M_MINUS : C2QO_DIAG_M, &f1, &f2, &scale);
    const long n = (long)ok_vol();
#pragma omp parallel for schedule(static)
    for (long s = 0; s < n; ++s) {
        double h[24], d[24];
        hopping_at(h, (size_t)s, gauge, kappa, in, 0);
        diag_site(d, in + 24 * s, f1, f2, scale);
        for (int k = 0; k < 24; ++k) out[24 * s + k] = d[k] + h[k];
    }
}
void ok_m_tm_plus(double* out, const double* in, const double* gauge, double kappa, double mubar)
{
    m_tm_full(out, in, gauge, kappa, mubar, 0);
}
void ok_m_tm_minus(double* out, const double* in, const double* gauge, double kappa, double mubar)
{
    m_tm_full(out, in, gauge, kappa, mubar, 1);
}

/* ---------------- fermion force (eo) ----------------
 * The four kernels fermion_force_eo_0..3 (ocl_kernel/force_fermion_eo.cl:31-459)
 * in one pass.  At every site x of the parity selected by evenodd (ODD = 1: the
 * even sites, as get_even_st_idx; EVEN = 0: the odd ones) with y = g5 Y(x):
 *   forward hop : the upper rows a, b of phi = (1 - g_mu) y and of
 *                 psi = (1 - g_mu) X(x + mu) give v = phi_a psi_a^+ + phi_b psi_b^+
 *                 (tr_v_times_u_dagger, operations_su3vec.cl:228-250) and
 *                 F(x, mu) += tr_lambda(bc_mu U_mu(x) v^+);
 *   backward hop: with (1 + g_mu) and X(x - mu), v = psi_a phi_a^+ + psi_b phi_b^+
 *                 and F(x - mu, mu) += tr_lambda(bc_mu U_mu(x - mu) v^+);
 * bc_mu = 2 kappa e^{i theta pi / N} for both hops; on T links U is multiplied by
 * e^{cp_re} e^{i cp_im} (forward) or e^{-cp_re} e^{i cp_im} (backward).
 * tr_lambda(M)_k = Tr[i T_k (M - M^+)] with T_k = lambda_k / 2
 * (tr_lambda_u, operations_gaugemomentum.cl:68-88, including its 1/sqrt(3)
 * literal).  Gauge momenta: ae[4 V] at link mu + 4 site, 8 doubles each.  Every
 * link gets at most one contribution per call, so the site loop is parallel. */
static void tr_lambda(const cplx M[9], double ae[8])
{
    ae[0] = -M[3].i - M[1].i;
    ae[1] = M[3].r - M[1].r;
    ae[2] = -M[0].i + M[4].i;
    ae[3] = -M[6].i - M[2].i;
    ae[4] = M[6].r - M[2].r;
    ae[5] = -M[7].i - M[5].i;
    ae[6] = M[7].r - M[5].r;
    ae[7] = (-M[0].i - M[4].i + 2.0 * M[8].i) * 0.577350269189625;
}

void ok_fermion_force_eo(double* gm, const double* Y, const double* X, const double* gauge, int evenodd, double kappa)
{
    const int par = evenodd == 1 ? 0 : 1;
    const long n  = (long)ok_seo();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        const size_t s = eo_site((size_t)i, par);
        double y[24];
        for (int k = 0; k < 24; ++k) y[k] = k < 12 ? Y[24 * i + k] : -Y[24 * i + k];
        for (int mu = 0; mu < 4; ++mu) {
            const cplx bc = {2. * kappa * g_phase[mu][0], 2. * kappa * g_phase[mu][1]};
            for (int back = 0; back < 2; ++back) {
                const size_t sn    = shift_site(s, mu, back ? -1 : +1);
                const size_t ls    = back ? sn : s; /* the link's site */
                const double* plus = X + 24 * (sn / 2);
                cplx U[9];
                for (int e = 0; e < 9; ++e) {
                    U[e] = cld(gauge + 18 * (mu + 4 * ls) + 2 * e);
                    if (mu == 0) U[e] = cmul(U[e], (cplx){g_cp_link[back][0], g_cp_link[back][1]});
                }
                cplx psi[2][3], phi[2][3];
                for (int a = 0; a < 2; ++a) {
                    const int p = PROJ_P[mu][a];
                    cplx c      = {PROJ_C[mu][a][0], PROJ_C[mu][a][1]};
                    if (back) c = (cplx){-c.r, -c.i};
                    for (int col = 0; col < 3; ++col) {
                        psi[a][col] = cadd(cld(plus + 6 * a + 2 * col), cmul(c, cld(plus + 6 * p + 2 * col)));
                        phi[a][col] = cadd(cld(y + 6 * a + 2 * col), cmul(c, cld(y + 6 * p + 2 * col)));
                    }
                }
                cplx v[9], w[9];
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q) {
                        cplx acc = {0., 0.};
                        for (int a = 0; a < 2; ++a)
                            acc = cadd(acc, back ? cmul(psi[a][r], cconj(phi[a][q])) : cmul(phi[a][r], cconj(psi[a][q])));
                        v[3 * r + q] = acc;
                    }
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q) {
                        cplx acc = {0., 0.};
                        for (int k = 0; k < 3; ++k) acc = cadd(acc, cmul(U[3 * r + k], cconj(v[3 * q + k])));
                        w[3 * r + q] = cmul(acc, bc);
                    }
                double ae[8];
                tr_lambda(w, ae);
                double* dst = gm + 8 * (mu + 4 * ls);
                for (int k = 0; k < 8; ++k) dst[k] += ae[k];
            }
        }
    }
}

/* the non-eo force (ocl_kernel/force_fermion.cl) sums the same two hops over
 * every site: the eo force of the even sites plus that of the odd ones */
void ok_fermion_force_full(double* gm, const double* Y, const double* X, const double* gauge, double kappa)
{
    const size_t seo = ok_seo();
    double* ye       = malloc(24 * seo * sizeof(double));
    double* yo       = malloc(24 * seo * sizeof(double));
    double* xe       = malloc(24 * seo * sizeof(double));
    double* xo       = malloc(24 * seo * sizeof(double));
    ok_convert_to_eo(ye, yo, Y);
    ok_convert_to_eo(xe, xo, X);
    ok_fermion_force_eo(gm, ye, xo, gauge, 1 /*ODD: the even sites*/, kappa);
    ok_fermion_force_eo(gm, yo, xe, gauge, 0 /*EVEN: the odd sites*/, kappa);
    free(ye);
    free(yo);
    free(xe);
    free(xo);
}
