/*
 * oracle_kernels.h -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 * The kernel-level interface the oracle's control flow (c2q_oracle.c) runs on.
 * Two backends implement it:
 *   oracle_kernels_port.c -- this project's own C restatement of the
 *                            reference kernels ("port");
 *   oracle_kernels_ref.c  -- the reference's own OpenCL-C kernels compiled as C
 *                            through ref_shim.h ("reference").
 *
 * Every field argument uses the reference's host formats:
 *   eo spinor field : spinor[Seo], AoS, 24 doubles per site ordered
 *                     [spin 0..3][colour 0..2][re,im]
 *                     (common_header_files/types_fermions.hpp:31-55), at the
 *                     eo index site/2 (ocl_kernel/operations_geometry.cl:297-300);
 *   full spinor     : spinor[V] in site order x + NS*y + NS^2*z + NS^3*t;
 *   gauge field     : Matrixsu3[4*V] at link mu + 4*site, TDIR = 0
 *                     (ocl_kernel/operations_geometry.cl:192-211), each matrix
 *                     row-major e00..e22 as (re,im) pairs (types.hpp:165-177).
 */
#ifndef C2Q_ORACLE_KERNELS_H
#define C2Q_ORACLE_KERNELS_H

#include <stddef.h>

typedef struct {
    double re, im;
} c2qo_complex;

/* Lattice extents, boundary phases (theta in units of pi) and chemical potential. */
typedef struct {
    int ns, nt;
    double theta_t, theta_s;
    int use_cp_re, use_cp_im;
    double cp_re, cp_im;
} c2qo_lattice;

/* tm site-diagonal variants (ocl_kernel/fermionmatrix_eo_m.cl:22-109 and
 * fermionmatrix_eo_m_merged.cl:22-64 of the reference) */
enum {
    C2QO_DIAG_M            = 0, /* (1 + i mubar g5)                 */
    C2QO_DIAG_MINV         = 1, /* (1 - i mubar g5) / (1 + mubar^2) */
    C2QO_DIAG_M_MINUS      = 2, /* (1 - i mubar g5)                 */
    C2QO_DIAG_MINV_MINUS   = 3, /* (1 + i mubar g5) / (1 + mubar^2) */
    C2QO_DIAG_M_G5         = 4, /* g5 (1 + i mubar g5)              */
    C2QO_DIAG_M_MINUS_G5   = 5  /* g5 (1 - i mubar g5)              */
};

void ok_set_lattice(const c2qo_lattice* lat);
const c2qo_lattice* ok_lattice(void);
size_t ok_seo(void); /* eo sites = V/2 */
size_t ok_vol(void); /* V */

void ok_dslash_eo(double* out, const double* in, const double* gauge, int evenodd, double kappa);
void ok_dslash_tm_inv_eo(double* out, const double* in, const double* gauge, int evenodd, double kappa, double mubar,
                         int minus);
void ok_tm_diag(double* out, const double* in, double mubar, int which);
void ok_gamma5_eo(double* inout);
void ok_saxpy(double* out, c2qo_complex alpha, const double* x, const double* y);
void ok_saxpy_gamma5(double* out, c2qo_complex alpha, const double* x, const double* y);
void ok_sax(double* out, c2qo_complex alpha, const double* x);
void ok_saxsbypz(double* out, c2qo_complex alpha, const double* x, c2qo_complex beta, const double* y,
                 const double* z);
c2qo_complex ok_scalar_product(const double* x, const double* y);
double ok_squarenorm(const double* x);
double ok_saxpy_squarenorm(double* out, c2qo_complex alpha, const double* x, const double* y);
void ok_zero(double* x);
void ok_cold(double* x);
void ok_copy(double* dst, const double* src);
void ok_convert_to_eo(double* even, double* odd, const double* full);
void ok_convert_from_eo(double* full, const double* even, const double* odd);
void ok_m_tm_plus(double* out, const double* in, const double* gauge, double kappa, double mubar);
void ok_m_tm_minus(double* out, const double* in, const double* gauge, double kappa, double mubar);
void ok_gamma5_full(double* inout);
double ok_squarenorm_full(const double* x);

/* fermion_force_eo_0..3 (ocl_kernel/force_fermion_eo.cl): gm (ae[4V], link
 * mu + 4*site, 8 doubles) += the eo fermion force of Y (on the sites evenodd
 * selects: ODD the even ones) and X (the other parity). */
void ok_fermion_force_eo(double* gm, const double* Y, const double* X, const double* gauge, int evenodd, double kappa);
/* fermion_force (ocl_kernel/force_fermion.cl): the same on full fields spinor[V]. */
void ok_fermion_force_full(double* gm, const double* Y, const double* X, const double* gauge, double kappa);

/* Name of the backend ("port" or "reference"). */
const char* ok_backend_name(void);

#endif
