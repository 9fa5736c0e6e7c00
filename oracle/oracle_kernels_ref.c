/*
 * oracle_kernels_ref.c -- TEST INFRASTRUCTURE ONLY (oracle, "reference" backend).
 *
 * Implements oracle_kernels.h by running the reference's own OpenCL-C kernels,
 * compiled as C through ref_shim.h.  The kernel sources are #included from the
 * reference tree in place (the include path points at it; nothing is copied).
 * Launch model = the reference's OpenCL CPU device: local size 1, one
 * work-item per OpenMP thread, AoS storage, blocked loops
 * (hardware/device_info.cpp:39-40,111-127).  Two-stage reductions follow
 * hardware/code/spinors.cpp:670-789: per-work-item partial sums, then the
 * *_reduction kernel on work-item 0.
 *
 * The boundary phases are produced exactly as hardware/code/opencl_module.cpp:
 * 190-203 does: theta*PI/N with PI = 3.14159265358979, then printed with 16
 * significant digits into the build options and parsed back.
 */
#include "ref_shim.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

__thread size_t c2qref_gid   = 0;
__thread size_t c2qref_gsize = 1;
unsigned c2qref_ns = 4, c2qref_nt = 4;
double c2qref_spatial_re = 1., c2qref_spatial_im = 0., c2qref_temporal_re = 1., c2qref_temporal_im = 0.;
double c2qref_expcpr = 1., c2qref_mexpcpr = 1., c2qref_coscpi = 1., c2qref_sincpi = 0.;

/* ---- the reference's hot-path device code, in the order the reference's own
 *      kernel builder concatenates it (hardware/code/fermions.cpp:36-123,
 *      hardware/code/spinors.cpp) ---- */
#include "ocl_kernel/opencl_header.cl"
#include "common_header_files/globaldefs.hpp"
#include "common_header_files/types.hpp"
#include "common_header_files/operations_complex.hpp"
#include "ocl_kernel/operations_geometry.cl"
#include "common_header_files/types_fermions.hpp"
#include "ocl_kernel/operations_matrix_su3.cl"
#include "ocl_kernel/operations_matrix.cl"
#include "ocl_kernel/operations_gaugefield.cl"
#include "ocl_kernel/operations_su3vec.cl"
#include "ocl_kernel/operations_spinor.cl"
#include "ocl_kernel/spinorfield.cl"
#include "ocl_kernel/operations_spinorfield_eo.cl"
#include "ocl_kernel/fermionmatrix.cl"
#include "ocl_kernel/fermionmatrix_eo.cl"
#include "ocl_kernel/fermionmatrix_eo_dslash.cl"
#include "ocl_kernel/fermionmatrix_eo_dslash_AND_M_tm_inverse_sitediagonal.cl"
#include "ocl_kernel/fermionmatrix_eo_dslash_AND_M_tm_inverse_sitediagonal_minus.cl"
#include "ocl_kernel/fermionmatrix_eo_m.cl"
#include "ocl_kernel/fermionmatrix_eo_m_merged.cl"
#include "ocl_kernel/fermionmatrix_eo_gamma5.cl"
#include "ocl_kernel/fermionmatrix_saxpy_AND_gamma5_eo.cl"
#include "ocl_kernel/fermionmatrix_m_tm_plus.cl"
#include "ocl_kernel/fermionmatrix_m_tm_minus.cl"
#include "ocl_kernel/fermionmatrix_gamma5.cl"
#include "ocl_kernel/spinorfield_eo_saxpy.cl"
#include "ocl_kernel/spinorfield_eo_sax.cl"
#include "ocl_kernel/spinorfield_eo_saxsbypz.cl"
#include "ocl_kernel/spinorfield_eo_scalar_product.cl"
#include "ocl_kernel/spinorfield_scalar_product_reduction.cl"
#include "ocl_kernel/spinorfield_eo_squarenorm.cl"
#include "ocl_kernel/spinorfield_squarenorm.cl"
#include "ocl_kernel/spinorfield_squarenorm_reduction.cl"
#include "ocl_kernel/spinorfield_eo_saxpy_AND_squarenorm.cl"
#include "ocl_kernel/spinorfield_eo_zero.cl"
#include "ocl_kernel/spinorfield_eo_cold.cl"
#include "ocl_kernel/spinorfield_eo_convert.cl"
#include "ocl_kernel/operations_gaugemomentum.cl"
#include "ocl_kernel/force_fermion_eo.cl"
#include "ocl_kernel/force_fermion.cl"

#include "oracle_kernels.h"

static c2qo_lattice g_lat = {4, 4, 0., 0., 0, 0, 0., 0.};

/* %.16g round trip, as std::ostringstream with precision(16) writes the -D options. */
static double as_build_option(double v)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%.16g", v);
    return strtod(buf, NULL);
}

void ok_set_lattice(const c2qo_lattice* lat)
{
    g_lat     = *lat;
    c2qref_ns = (unsigned)lat->ns;
    c2qref_nt = (unsigned)lat->nt;
    /* opencl_module.cpp:190-203; PI as globaldefs.hpp defines it */
    double tmp_spatial  = (lat->theta_s * PI) / ((double)lat->ns);
    double tmp_temporal = (lat->theta_t * PI) / ((double)lat->nt);
    c2qref_spatial_re   = as_build_option(cos(tmp_spatial));
    c2qref_spatial_im   = as_build_option(sin(tmp_spatial));
    c2qref_temporal_re  = as_build_option(cos(tmp_temporal));
    c2qref_temporal_im  = as_build_option(sin(tmp_temporal));
    /* opencl_module.cpp:113-124 */
    c2qref_expcpr  = lat->use_cp_re ? as_build_option(exp(lat->cp_re)) : 1.;
    c2qref_mexpcpr = lat->use_cp_re ? as_build_option(exp(-1. * lat->cp_re)) : 1.;
    c2qref_coscpi  = lat->use_cp_im ? as_build_option(cos(lat->cp_im)) : 1.;
    c2qref_sincpi  = lat->use_cp_im ? as_build_option(sin(lat->cp_im)) : 0.;
}
const c2qo_lattice* ok_lattice(void) { return &g_lat; }
size_t ok_seo(void) { return (size_t)VOL4D_MEM / 2; }
size_t ok_vol(void) { return (size_t)VOL4D_MEM; }
const char* ok_backend_name(void) { return "reference"; }

/* Run one "NDRange" of the CPU device: global size = #threads, local size 1. */
#define LAUNCH(CALL)                                              \
    do {                                                          \
        _Pragma("omp parallel")                                   \
        {                                                         \
            c2qref_gid   = (size_t)omp_get_thread_num();          \
            c2qref_gsize = (size_t)omp_get_num_threads();         \
            CALL;                                                 \
        }                                                         \
    } while (0)

void ok_dslash_eo(double* out, const double* in, const double* gauge, int evenodd, double kappa)
{
    LAUNCH(dslash_eo((const spinor*)in, (spinor*)out, (const Matrixsu3*)gauge, evenodd, kappa));
}

void ok_dslash_tm_inv_eo(double* out, const double* in, const double* gauge, int evenodd, double kappa, double mubar,
                         int minus)
{
    if (minus)
        LAUNCH(dslash_AND_M_tm_inverse_sitediagonal_minus_eo((const spinor*)in, (spinor*)out,
                                                             (const Matrixsu3*)gauge, evenodd, kappa, mubar));
    else
        LAUNCH(dslash_AND_M_tm_inverse_sitediagonal_eo((const spinor*)in, (spinor*)out, (const Matrixsu3*)gauge,
                                                       evenodd, kappa, mubar));
}

void ok_tm_diag(double* out, const double* in, double mubar, int which)
{
    const spinor* i = (const spinor*)in;
    spinor* o       = (spinor*)out;
    switch (which) {
        case C2QO_DIAG_M: LAUNCH(M_tm_sitediagonal(i, o, mubar)); break;
        case C2QO_DIAG_MINV: LAUNCH(M_tm_inverse_sitediagonal(i, o, mubar)); break;
        case C2QO_DIAG_M_MINUS: LAUNCH(M_tm_sitediagonal_minus(i, o, mubar)); break;
        case C2QO_DIAG_MINV_MINUS: LAUNCH(M_tm_inverse_sitediagonal_minus(i, o, mubar)); break;
        case C2QO_DIAG_M_G5: LAUNCH(M_tm_sitediagonal_AND_gamma5_eo(i, o, mubar)); break;
        case C2QO_DIAG_M_MINUS_G5: LAUNCH(M_tm_sitediagonal_minus_AND_gamma5_eo(i, o, mubar)); break;
        default: abort();
    }
}

void ok_gamma5_eo(double* inout) { LAUNCH(gamma5_eo((spinor*)inout)); }

void ok_saxpy(double* out, c2qo_complex alpha, const double* x, const double* y)
{
    hmc_complex a = {alpha.re, alpha.im};
    LAUNCH(saxpy_eoprec((const spinor*)x, (const spinor*)y, &a, (spinor*)out));
}

void ok_saxpy_gamma5(double* out, c2qo_complex alpha, const double* x, const double* y)
{
    LAUNCH(saxpy_AND_gamma5_eo((const spinor*)x, (const spinor*)y, alpha.re, alpha.im, (spinor*)out));
}

void ok_sax(double* out, c2qo_complex alpha, const double* x)
{
    hmc_complex a = {alpha.re, alpha.im};
    LAUNCH(sax_eoprec((const spinor*)x, &a, (spinor*)out));
}

void ok_saxsbypz(double* out, c2qo_complex alpha, const double* x, c2qo_complex beta, const double* y,
                 const double* z)
{
    hmc_complex a = {alpha.re, alpha.im};
    hmc_complex b = {beta.re, beta.im};
    LAUNCH(saxsbypz_eoprec((const spinor*)x, (const spinor*)y, (const spinor*)z, &a, &b, (spinor*)out));
}

c2qo_complex ok_scalar_product(const double* x, const double* y)
{
    int nthr             = omp_get_max_threads();
    hmc_complex* partial = calloc((size_t)nthr, sizeof(hmc_complex));
    hmc_complex res      = {0., 0.};
    int used             = 0;
#pragma omp parallel
    {
        c2qref_gid   = (size_t)omp_get_thread_num();
        c2qref_gsize = (size_t)omp_get_num_threads();
        scalar_product_eoprec((const spinor*)x, (const spinor*)y, partial, NULL);
#pragma omp single
        used = omp_get_num_threads();
    }
    c2qref_gid   = 0;
    c2qref_gsize = (size_t)used;
    scalar_product_reduction(partial, &res, (uint)used);
    c2qref_gsize = 1;
    free(partial);
    return (c2qo_complex){res.re, res.im};
}

static double squarenorm_generic(const double* x, int full)
{
    int nthr          = omp_get_max_threads();
    hmc_float* partial = calloc((size_t)nthr, sizeof(hmc_float));
    hmc_float res     = 0.;
    int used          = 0;
#pragma omp parallel
    {
        c2qref_gid   = (size_t)omp_get_thread_num();
        c2qref_gsize = (size_t)omp_get_num_threads();
        if (full)
            global_squarenorm((const spinor*)x, partial, NULL);
        else
            global_squarenorm_eoprec((const spinor*)x, partial, NULL);
#pragma omp single
        used = omp_get_num_threads();
    }
    c2qref_gid   = 0;
    c2qref_gsize = 1;
    global_squarenorm_reduction(&res, partial, (uint)used);
    free(partial);
    return res;
}

double ok_squarenorm(const double* x) { return squarenorm_generic(x, 0); }
double ok_squarenorm_full(const double* x) { return squarenorm_generic(x, 1); }

double ok_saxpy_squarenorm(double* out, c2qo_complex alpha, const double* x, const double* y)
{
    int nthr           = omp_get_max_threads();
    hmc_float* partial = calloc((size_t)nthr, sizeof(hmc_float));
    hmc_float res      = 0.;
    hmc_complex a      = {alpha.re, alpha.im};
    int used           = 0;
#pragma omp parallel
    {
        c2qref_gid   = (size_t)omp_get_thread_num();
        c2qref_gsize = (size_t)omp_get_num_threads();
        saxpy_AND_squarenorm_eo((const spinor*)x, (const spinor*)y, &a, (spinor*)out, partial, NULL);
#pragma omp single
        used = omp_get_num_threads();
    }
    c2qref_gid   = 0;
    c2qref_gsize = 1;
    global_squarenorm_reduction(&res, partial, (uint)used);
    free(partial);
    return res;
}

void ok_zero(double* x) { LAUNCH(set_zero_spinorfield_eoprec((spinor*)x)); }
void ok_cold(double* x) { LAUNCH(set_eoprec_spinorfield_cold((spinor*)x)); }
void ok_copy(double* dst, const double* src) { memcpy(dst, src, ok_seo() * 24 * sizeof(double)); }

void ok_convert_to_eo(double* even, double* odd, const double* full)
{
    LAUNCH(convert_to_eoprec((spinor*)even, (spinor*)odd, (const spinor*)full));
}

void ok_convert_from_eo(double* full, const double* even, const double* odd)
{
    LAUNCH(convert_from_eoprec((const spinor*)even, (const spinor*)odd, (spinor*)full));
}

void ok_m_tm_plus(double* out, const double* in, const double* gauge, double kappa, double mubar)
{
    LAUNCH(M_tm_plus((const spinor*)in, (const Matrixsu3*)gauge, (spinor*)out, kappa, mubar));
}

void ok_m_tm_minus(double* out, const double* in, const double* gauge, double kappa, double mubar)
{
    LAUNCH(M_tm_minus((const spinor*)in, (const Matrixsu3*)gauge, (spinor*)out, kappa, mubar));
}

void ok_gamma5_full(double* inout) { LAUNCH(gamma5((spinor*)inout)); }

/* hardware/code/molecular_dynamics.cpp:543-625 fermion_force_eo_device: the four
 * direction kernels one after the other on the same momenta */
void ok_fermion_force_eo(double* gm, const double* Y, const double* X, const double* gauge, int evenodd, double kappa)
{
    LAUNCH(fermion_force_eo_0((const Matrixsu3*)gauge, (const spinor*)Y, (const spinor*)X, (ae*)gm, evenodd, kappa));
    LAUNCH(fermion_force_eo_1((const Matrixsu3*)gauge, (const spinor*)Y, (const spinor*)X, (ae*)gm, evenodd, kappa));
    LAUNCH(fermion_force_eo_2((const Matrixsu3*)gauge, (const spinor*)Y, (const spinor*)X, (ae*)gm, evenodd, kappa));
    LAUNCH(fermion_force_eo_3((const Matrixsu3*)gauge, (const spinor*)Y, (const spinor*)X, (ae*)gm, evenodd, kappa));
}

/* molecular_dynamics.cpp fermion_force_device: the non-eo kernel on full fields */
void ok_fermion_force_full(double* gm, const double* Y, const double* X, const double* gauge, double kappa)
{
    LAUNCH(fermion_force((const Matrixsu3*)gauge, (const spinor*)Y, (const spinor*)X, (ae*)gm, kappa));
}
