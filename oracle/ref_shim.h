/*
 * ref_shim.h -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 * A small OpenCL-C -> GNU C11 shim so that the reference's own hot-path kernel
 * sources (the ocl_kernel .cl files of CL2QCD, read in place from the reference tree at
 * build time, never copied) compile into a host shared library under
 * oracle/_ref/.  That library runs the reference kernels the way the reference
 * runs them on an OpenCL CPU device: AoS storage (no _USE_SOA_), blocked loops
 * (_USE_BLOCKED_LOOPS_), local size 1, one work-item per OpenMP thread
 * (hardware/device_info.cpp:39-40,111-127 of the reference).
 *
 * The build-time -D constants that hardware/code/opencl_module.cpp:61-224 of the
 * reference passes to the OpenCL compiler are turned into process globals here,
 * so one library serves every lattice size; the library is therefore not
 * thread-safe across concurrent calls (it is only used by the tests and by the
 * CPU baseline, one call at a time).
 *
 * Nothing in the product links against this: only tests/, the smoke check and
 * the CPU-baseline leg of bench.py load oracle/_ref.
 */
#ifndef C2Q_REF_SHIM_H
#define C2Q_REF_SHIM_H

#include <stdbool.h>
#include <stddef.h>
#include <math.h>
#include <stdio.h>

/* ---- OpenCL address-space / function qualifiers ---- */
#define __kernel
#define __global
#define __local
#define __private
#define __constant const

/* ---- OpenCL scalar / vector types used by the hot-path files ---- */
typedef unsigned int uint;
typedef struct { uint x, y, z; } uint3;
typedef struct { uint x, y, z, w; } uint4;
typedef struct { int x, y, z, w; } int4;
typedef struct { float x, y; } float2;
typedef struct { float x, y, z, w; } float4;

/* ---- work-item functions: one work-item per OpenMP thread, local size 1 ---- */
extern __thread size_t c2qref_gid;
extern __thread size_t c2qref_gsize;
static inline size_t get_global_id(int d) { (void)d; return c2qref_gid; }
static inline size_t get_global_size(int d) { (void)d; return c2qref_gsize; }
static inline size_t get_local_id(int d) { (void)d; return 0; }
static inline size_t get_local_size(int d) { (void)d; return 1; }
static inline size_t get_group_id(int d) { (void)d; return c2qref_gid; }
static inline size_t get_num_groups(int d) { (void)d; return c2qref_gsize; }
#define CLK_LOCAL_MEM_FENCE 0
#define CLK_GLOBAL_MEM_FENCE 0
static inline void barrier(int f) { (void)f; }

/* ---- the -D build options of opencl_module.cpp, as runtime globals ---- */
extern unsigned c2qref_ns, c2qref_nt;
extern double c2qref_spatial_re, c2qref_spatial_im, c2qref_temporal_re, c2qref_temporal_im;
extern double c2qref_expcpr, c2qref_mexpcpr, c2qref_coscpi, c2qref_sincpi;

#define _INKERNEL_
#define _USEDOUBLEPREC_
#define _USE_BLOCKED_LOOPS_
#define _TWISTEDMASS_
/* Both chemical-potential branches are always compiled in; with the neutral
 * values (exp(0)=1, cos 0=1, sin 0=0) they are bitwise no-ops. */
#define _CP_REAL_
#define _CP_IMAG_

#define NSPACE (c2qref_ns)
#define NTIME_GLOBAL (c2qref_nt)
#define NTIME_LOCAL (c2qref_nt)
#define NTIME_MEM (c2qref_nt)
#define NTIME_OFFSET 0
#define VOLSPACE (c2qref_ns * c2qref_ns * c2qref_ns)
#define VOL4D_GLOBAL (VOLSPACE * c2qref_nt)
#define VOL4D_LOCAL (VOLSPACE * c2qref_nt)
#define VOL4D_MEM (VOLSPACE * c2qref_nt)
#define T_EXTENT_LOCAL (c2qref_nt)
#define GRID_POS_LOCAL 0
#define SU3SIZE 9
#define STAPLEMATRIXSIZE 9
#define EOPREC_SPINORFIELDSIZE_GLOBAL (VOL4D_MEM / 2)
#define EOPREC_SPINORFIELDSIZE_LOCAL (VOL4D_MEM / 2)
#define EOPREC_SPINORFIELDSIZE_MEM (VOL4D_MEM / 2)
#define SPINORFIELDSIZE_GLOBAL (VOL4D_MEM)
#define SPINORFIELDSIZE_LOCAL (VOL4D_MEM)
#define SPINORFIELDSIZE_MEM (VOL4D_MEM)
#define GAUGEMOMENTASIZE_GLOBAL (VOL4D_MEM * 4)
#define GAUGEMOMENTASIZE_LOCAL (VOL4D_MEM * 4)
#define GAUGEMOMENTASIZE_MEM (VOL4D_MEM * 4)
#define SPATIAL_RE (c2qref_spatial_re)
#define MSPATIAL_RE (-c2qref_spatial_re)
#define SPATIAL_IM (c2qref_spatial_im)
#define MSPATIAL_IM (-c2qref_spatial_im)
#define TEMPORAL_RE (c2qref_temporal_re)
#define MTEMPORAL_RE (-c2qref_temporal_re)
#define TEMPORAL_IM (c2qref_temporal_im)
#define MTEMPORAL_IM (-c2qref_temporal_im)
#define EXPCPR (c2qref_expcpr)
#define MEXPCPR (c2qref_mexpcpr)
#define COSCPI (c2qref_coscpi)
#define SINCPI (c2qref_sincpi)

#endif
