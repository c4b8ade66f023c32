/*
 * pastix_b200_sched.h -- the B200 backend as a PaStiX scheduler.
 *
 * With iparm[IPARM_SCHEDULER] set to one of the two values below, PaStiX's own
 * entry points (pastix_task_numfact, pastix_task_solve, pastix_task_refine and the
 * solve subtasks) run the numerical factorization, the triangular solves and the
 * iterative refinement on one B200 through libpastix_b200.so (include/pastix_b200.h)
 * instead of the CPU schedulers of pastix_scheduler_t (include/pastix/api.h:289-295).
 * PaStiX's analysis (ordering, symbolic factorization, blend) is unchanged and its
 * SolverMatrix is reused bit-exact; the factor lives on the GPU (no host coeftab).
 *
 * The hooks are called from a build of PaStiX's sources in which each entry point
 * tests pastix_b200_scheduler() first (pastix_b200/refhost/build_sched.py).
 */
#ifndef PASTIX_B200_SCHED_H
#define PASTIX_B200_SCHED_H

#include "common.h"

/* Scheduler ids after PastixSchedDynamic = 4 */
#define PastixSchedB200      5 /* factor in the matrix's own precision on the GPU: the drop-in */
#define PastixSchedB200Mixed 6 /* FP32 factor with 3xTF32 tensor-core updates; solve and
                                  refinement vectors in double */

/* 1 if the instance's scheduler is one of the B200 ids */
int pastix_b200_scheduler( const pastix_data_t *pastix_data );

/* pastix_subtask_bcsc2ctab (sopalin/pastix_task_sopalin.c:196): the bcsc's values go
 * to the GPU factor instance (created from the SolverMatrix on first use). */
int pastix_b200_subtask_bcsc2ctab( pastix_data_t *pastix_data );

/* pastix_subtask_sopalin (sopalin/pastix_task_sopalin.c:355): the factorization on
 * the GPU; sets diagthreshold, IPARM_STATIC_PIVOTING, DPARM_FACT_TIME/FLOPS and the
 * steps as the CPU path does. */
int pastix_b200_subtask_sopalin( pastix_data_t *pastix_data );

/* pastix_task_solve (sopalin/pastix_task_solve.c:550): b (original numbering,
 * matrix precision) overwritten by x; permutations and sweeps on the GPU. */
int pastix_b200_task_solve( pastix_data_t *pastix_data, pastix_int_t nrhs, void *b,
                            pastix_int_t ldb );

/* pastix_subtask_solve / _trsm / _diag (sopalin/pastix_task_solve.c:194-516) on a
 * permuted b. */
int pastix_b200_subtask_solve( pastix_data_t *pastix_data, pastix_int_t nrhs, void *b,
                               pastix_int_t ldb );
int pastix_b200_subtask_trsm( pastix_data_t *pastix_data, pastix_coeftype_t flttype,
                              pastix_side_t side, pastix_uplo_t uplo, pastix_trans_t trans,
                              pastix_diag_t diag, pastix_int_t nrhs, void *b, pastix_int_t ldb );
int pastix_b200_subtask_diag( pastix_data_t *pastix_data, pastix_coeftype_t flttype,
                              pastix_int_t nrhs, void *b, pastix_int_t ldb );

/* pastix_task_refine (refinement/pastix_task_refine.c:226), after PaStiX has set
 * DPARM_EPSILON_REFINEMENT: IPARM_REFINEMENT's method (GMRES, CG or SR) on the GPU,
 * all right-hand sides together, each with its own stopping rule. */
int pastix_b200_task_refine( pastix_data_t *pastix_data, pastix_int_t n, pastix_int_t nrhs,
                             void *b, pastix_int_t ldb, void *x, pastix_int_t ldx );

/* pastixFinalize (common/api.c:868): releases the instance's GPU factor. */
void pastix_b200_finalize( pastix_data_t *pastix_data );

/* The GPU factor instance (a b200_solver_t *) of a PaStiX instance, NULL before
 * its first bcsc2ctab: for b200_* calls on the same factor (factor download,
 * device solves). */
void *pastix_b200_solver( pastix_data_t *pastix_data );

#endif /* PASTIX_B200_SCHED_H */
