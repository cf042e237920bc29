/*
 * efdc_oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU FP64 restatement of EFDC+ 8.5's external mode (and its bottom-stress
 * and explicit-momentum producers), used by tests/ and by
 * bench.py's CPU-baseline leg to check and time the CUDA library.  Nothing in
 * the shipped library links or calls this code.
 *
 * Parity status: UNPINNED by the reference.  EFDC+ is Intel-Fortran-only
 * (IFPORT, Windows NetCDF libraries), no Fortran compiler exists in this
 * build environment, and the reference ships no tests, golden vectors or
 * result files for this path.  The restatement is instead cross-checked by
 * independent properties (direct sparse solve of the assembled system, lake
 * at rest, mirror symmetry, volume telescoping, thread-count invariance); see
 * tests/test_oracle_*.py.
 *
 * Arithmetic rules followed so that the statement-level rounding matches the
 * ReleaseDP64 build (/real_size:64 /fp:source, no /Qx => SSE2, no FMA):
 *   - FP64 everywhere, compiled with -ffp-contract=off, no -ffast-math;
 *   - Fortran left-to-right evaluation of each statement, same statement order;
 *   - serial, L-ordered dot products (congrad.f90:118-149);
 *   - libm sin/cos/sqrt/fmod.
 */
#ifndef EFDC_ORACLE_H
#define EFDC_ORACLE_H

#include "../include/efdc_xm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

/* nthreads: NTHREADS of the reference; noptimal_cap: the "8" of
 * NOPTIMAL=MIN(NTHREADS,8,MAX(LA/100,1)) (calpuv2c.f90:61); pass 8 for the
 * reference behaviour, or a larger cap to use more host cores. */
oracle_ctx *oracle_create(const efdc_xm_grid *grid, int nthreads, int noptimal_cap);
void oracle_destroy(oracle_ctx *c);
int oracle_noptimal(const oracle_ctx *c);

/* One CALPUV2C call (calpuv2c.f90:128-1187 with ISITB=0, ISVEG=0, ISGWIE=0,
 * IGRIDV=0; sub-grid channels and the baroclinic terms where set), or, with
 * prm->tl3_istl = 3 or 2, one CALPUV9C(ISTL_) call (calpuv9c.f90:105-1069).
 * Returns the status code. */
int oracle_step(oracle_ctx *c, const efdc_xm_params *prm, efdc_xm_fields *f,
                efdc_xm_stats *st);

/* CONGRAD on a caller-assembled scaled system (congrad.f90:54-187). */
/* Sub-grid channels of the basin (efdc_xm_set_channels' contract); n = 0
 * removes them.  Returns 0, or EFDC_XM_BAD_ARGUMENT. */
int oracle_set_channels(oracle_ctx *c, const efdc_xm_channels *ch);

/* Layers of the standard sigma grid for CALEBI (efdc_xm_set_layers' contract). */
int oracle_set_layers(oracle_ctx *c, const efdc_xm_layers *ly);

/* The bed of the bottom-stress producer (efdc_xm_set_bed's contract). */
int oracle_set_bed(oracle_ctx *c, const efdc_xm_bed *bed);

/* CALTBXY's drag coefficients and the bottom stresses of hdmt2t.f90:670-684
 * (efdc_xm_bottom_stress_batch's contract) on the state `st` the last
 * oracle_step left (HU, HV, LMASKDRY; its entry mask is the context's);
 * TBX, TBY in/out in f. */
int oracle_bottom_stress(oracle_ctx *c, const efdc_xm_drag_params *p, const efdc_xm_fields *st,
                         efdc_xm_drag_fields *f);

/* CALEXP2T's external-mode terms (efdc_xm_set_momentum / efdc_xm_explicit_batch
 * for one basin). */
int oracle_set_momentum(oracle_ctx *c, const efdc_xm_momentum *mo);
int oracle_explicit(oracle_ctx *c, const efdc_xm_explicit_params *p, efdc_xm_explicit_fields *f);
int oracle_congrad(oracle_ctx *c, const double *ccc, const double *ccs,
                   const double *ccn, const double *ccw, const double *cce,
                   const double *ccci, const double *fptmp, double *p,
                   double rsqm, int iterm, int *iters, double *rsq);

#ifdef __cplusplus
}
#endif
#endif
