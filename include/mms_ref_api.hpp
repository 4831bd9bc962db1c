/*
 * Drop-in C++ entry points with the reference's exact signatures (C++ linkage,
 * fptype = float, Vector3 = three packed floats), implemented on top of the C
 * ABI in mms_b200.h.  Linking libmms_refapi.so in place of the reference's
 * fmm_kernel.o + ode_functions.o lets the reference's main.cpp driver run its
 * whole demag / LLG path on the B200 unchanged.
 *
 *   fmm_calc                   helper_functions.hpp:24-29   (fmm_calc.cu:295-408)
 *   calc_potential_exact       helper_functions.hpp:31-35   (fmm_calc.cu:412-461)
 *   calc_potential_exact_gpu   helper_functions.hpp:37-40   (potential_calc.cu:120-188)
 *   Hfield                     ode_functions.hpp:8-15       (ode_functions.cpp:21-70)
 *   rk4_step                   ode_functions.cpp:76-87      (no header upstream)
 *   time_marching              ode_functions.hpp:17-24      (ode_functions.cpp:158-365)
 *
 * Semantics kept: host arrays owned by the caller; potential without 1/(4 pi);
 * EXIT_SUCCESS / EXIT_FAILURE returns; the library keeps per-process state
 * sized by the last grid (re-created when the grid changes; the reference
 * silently assumes the first call's grid forever).  Differences, by design:
 * every path runs on the GPU (use_gpu is accepted and ignored: the library has
 * no CPU path); the FMM is a full FMM (P2M/M2M/M2L/L2L/L2P + near-field P2P)
 * valid for any grid, not the reference's tree code restricted to square
 * power-of-two grids; the RK4 state is FP64 inside a step; time_marching
 * never waits on getchar().  Not thread-safe, like the reference.
 */
#ifndef MMS_REF_API_HPP
#define MMS_REF_API_HPP

#include <stdio.h>

#ifndef _MYDEFS_H_
typedef float fptype;
typedef unsigned char byte;
#endif

#ifndef _VECTOR3_H_
struct Vector3;  /* the reference's three-float value type (Vector3.hpp:10-12) */
#endif

int fmm_calc(const fptype *charge, fptype *potential,
             const int xdim, const int ydim, const int zdim,
             const fptype dx, const fptype dy, const fptype dz,
             const int P, const int use_gpu, const int verbosity);

int calc_potential_exact(const fptype *charge,
                         const int xdim, const int ydim, const int zdim,
                         const fptype dx, const fptype dy, const fptype dz,
                         fptype *potential, int use_gpu, const int verbosity);

int calc_potential_exact_gpu(const fptype *charge,
                             const int xdim, const int ydim, const int zdim,
                             const fptype dx, const fptype dy, const fptype dz,
                             fptype *potential);

int Hfield(const Vector3 *M, Vector3 *H, fptype *charge, fptype *potential,
           const fptype t,
           const int xdim, const int ydim, const int zdim,
           const fptype dx, const fptype dy, const fptype dz,
           const int P,
           const fptype mu_0, const fptype Ms, const fptype Aexch,
           const int demag, const int exchange, const int external, const int use_fmm,
           const int use_gpu, const int verbosity);

int rk4_step(const fptype t, const fptype dt, fptype *t2,
             const byte *material, const Vector3 *M, Vector3 *M2,
             Vector3 *H, Vector3 *slope, Vector3 *this_slope,
             fptype *charge, fptype *potential,
             const int xdim, const int ydim, const int zdim,
             const fptype dx, const fptype dy, const fptype dz,
             const int P,
             const fptype mu_0, const fptype Ms, const fptype Aexch, const fptype alfa, const fptype gamma,
             const int demag, const int exchange, const int external, const int use_fmm,
             const int normalize, const int use_gpu, const int verbosity);

int time_marching(byte *material, Vector3 *M,
                  const fptype finaltime, const fptype timestep,
                  const int xdim, const int ydim, const int zdim,
                  const fptype dx, const fptype dy, const fptype dz,
                  const int P,
                  const fptype mu_0, const fptype Ms, const fptype Aexch, const fptype alfa, const fptype gamma,
                  const int coupling, const int exchange, const int external, const int use_fmm,
                  const int use_gpu, const char *sim_name, const int verbosity);

#endif
