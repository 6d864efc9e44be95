/*
 * sw2_refglue.h -- the B200 SW2 path behind the reference's own signatures.
 *
 * sw2_refglue.c is compiled into the reference (it includes the reference's adh.h)
 * in place of src/residual/assemble_residual.c and src/jacobian/assemble_jacobian.c.
 * It defines, with the reference's signatures,
 *   void assemble_residual(SMODEL_SUPER *sm, SGRID *grid)   -- src/residual/residual.h:5
 *   void assemble_jacobian(SMODEL_SUPER *sm)                -- src/jacobian/jacobian.h:5
 * so that the reference's own fe_newton (src/newton/fe_newton.c:351,360, its only
 * callers) assembles on the GPU, and a stepper with fe_newton's signature
 *   int fe_newton_gpu(SMODEL_SUPER *sm)                     -- src/newton/newton.h:19
 * that runs the whole Newton solve on the GPU; install it as
 * adh_time_stepper[FE_NEWTON] (src/models/set_function_pointers.c:64) and the
 * reference's time_loop (src/timeloop/time_loop.c:14) drives it.
 *
 * One device model (sw2g_model) per SMODEL_SUPER, built on the first call from
 * sm->grid and checked against sm->lin_sys's CSR.  Covered: SW2 triangles
 * (fe_sw2_body_resid) and the two compiled SW2 boundary plugins, fe_sw2_bc_vel and
 * fe_sw2_bc_h, with one velocity series pair for all velocity strings and
 * nsubsteps = 1; anything else stops with tl_error, as the reference stops on a
 * model it cannot run.
 */
#ifndef SW2_REFGLUE_H
#define SW2_REFGLUE_H
#include "adh_sw2_gpu.h"

/* builds (or finds) the device model of sm; SW2G_OK or an SW2G_ERR_* code */
int sw2_gpu_attach(SMODEL_SUPER *sm);
/* the device model of sm (NULL before sw2_gpu_attach) */
sw2g_model *sw2_gpu_model(SMODEL_SUPER *sm);
/* Newton options fe_newton_gpu hands to sw2g_fe_newton after copying tol_nonlin,
 * inc_nonlin, max_nonlin_it and max_nonlin_linesearch_cuts from sm (NULL: the defaults). */
void sw2_gpu_set_newton_opts(const sw2g_newton_opts *opts);
/* statistics of the last fe_newton_gpu call */
const sw2g_newton_stats *sw2_gpu_last_stats(void);
int fe_newton_gpu(SMODEL_SUPER *sm);
void sw2_gpu_detach_all(void);
#endif
