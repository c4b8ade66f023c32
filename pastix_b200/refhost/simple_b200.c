/*
 * simple_b200.c -- PaStiX's example/simple.c sequence as a callable function, for
 * running the same program under any scheduler (the CPU ones or the B200 ids of
 * pastix_b200_sched.h) and comparing the results.
 *
 *   pastixInitParam -> iparm/dparm -> pastixInit
 *   -> analysis: pastix_task_analyze's four subtasks (blend/pastix_task_analyze.c:52-102)
 *      with the ordering given by pastixOrderGrid (grid nested dissection; Scotch
 *      and Metis are not part of this build)
 *   -> pastix_task_numfact -> x = b -> pastix_task_solve -> pastix_task_refine
 *   -> pastixFinalize
 *
 * The matrix is a 0-based CSC (lower triangle for symmetric matrices) of doubles.
 */
#include "common.h"
#include "spm.h"
#include "blend/solver.h"
#include "bcsc/bcsc.h"
#include "pastix/order.h"
#include "pastix_b200.h"
#include "pastix_b200_sched.h"
#include <string.h>

/* out[] = { DPARM_FACT_TIME, DPARM_SOLV_TIME, DPARM_REFINE_TIME, diagthreshold,
 *           IPARM_STATIC_PIVOTING, IPARM_NBITER, DPARM_RELATIVE_ERROR, DPARM_FACT_FLOPS,
 *           DPARM_A_NORM, return code of the first failing task (0: none) }.
 * L, U (may be NULL): the factor in PaStiX's coeftab layout after numfact (the
 * host coeftab for the CPU schedulers, the GPU factor for the B200 ids).
 * Returns 0 or the PaStiX error code of the failing step. */
int
pb_simple( int64_t n, const int64_t *colptr, const int64_t *rowind, const double *values, int symmetric,
           int facto, int64_t nx, int64_t ny, int64_t nz, int scheduler, int nthreads, int refinement,
           double epsilon_magn_ctrl, int64_t nrhs, const double *b, double *x, double *L, double *U,
           double *out )
{
    pastix_data_t  *pastix_data = NULL;
    pastix_int_t    iparm[IPARM_SIZE];
    double          dparm[DPARM_SIZE];
    spmatrix_t      spm;
    pastix_order_t *ord;
    int64_t nnz = colptr[n] - colptr[0];
    int rc;

    /* the matrix */
    spmInit( &spm );
    spm.mtxtype = symmetric ? SpmSymmetric : SpmGeneral;
    spm.flttype = SpmDouble;
    spm.fmttype = SpmCSC;
    spm.n       = n;
    spm.nnz     = nnz;
    spm.dof     = 1;
    spm.colptr  = malloc( (n + 1) * sizeof(spm_int_t) );
    spm.rowptr  = malloc( nnz * sizeof(spm_int_t) );
    spm.values  = malloc( nnz * sizeof(double) );
    memcpy( spm.colptr, colptr, (n + 1) * sizeof(int64_t) );
    memcpy( spm.rowptr, rowind, nnz * sizeof(int64_t) );
    memcpy( spm.values, values, nnz * sizeof(double) );
    spmUpdateComputedFields( &spm );

    /* parameters and startup */
    pastixInitParam( iparm, dparm );
    iparm[IPARM_VERBOSE]       = PastixVerboseNot;
    iparm[IPARM_FACTORIZATION] = facto;
    iparm[IPARM_SCHEDULER]     = scheduler;
    iparm[IPARM_THREAD_NBR]    = nthreads > 0 ? nthreads : 1;
    iparm[IPARM_ORDERING]      = PastixOrderPersonal;
    iparm[IPARM_REFINEMENT]    = refinement;
    dparm[DPARM_EPSILON_MAGN_CTRL] = epsilon_magn_ctrl;
    pastixInit( &pastix_data, MPI_COMM_WORLD, iparm, dparm );

    /* ordering, symbolic factorization, reordering, blend */
    ord = calloc( 1, sizeof(pastix_order_t) );
    rc  = pastixOrderGrid( &ord, nx, ny, nz );
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_order( pastix_data, &spm, ord );
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_symbfact( pastix_data );
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_reordering( pastix_data );
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_blend( pastix_data );
    pastixOrderExit( ord );
    free( ord );

    /* numerical factorization */
    if ( rc == PASTIX_SUCCESS ) rc = pastix_task_numfact( pastix_data, &spm );
    if ( (rc == PASTIX_SUCCESS) && (L != NULL) ) {
        if ( pastix_b200_scheduler( pastix_data ) ) {
            rc = b200_factor_download( pastix_b200_solver( pastix_data ), L, U );
        }
        else {
            SolverMatrix *s = pastix_data->solvmatr;
            double *pl = L, *pu = U;
            for ( pastix_int_t k = 0; k < s->cblknbr; k++ ) {
                SolverCblk *c = s->cblktab + k;
                size_t cnt = (size_t)c->stride * (size_t)cblk_colnbr( c );
                memcpy( pl, c->lcoeftab, cnt * sizeof(double) );
                pl += cnt;
                if ( (pu != NULL) && (c->ucoeftab != NULL) ) {
                    memcpy( pu, c->ucoeftab, cnt * sizeof(double) );
                    pu += cnt;
                }
            }
        }
    }

    /* solve and refinement (b is kept for the refinement) */
    if ( rc == PASTIX_SUCCESS ) {
        memcpy( x, b, (size_t)n * nrhs * sizeof(double) );
        rc = pastix_task_solve( pastix_data, nrhs, x, n );
    }
    if ( rc == PASTIX_SUCCESS ) {
        rc = pastix_task_refine( pastix_data, n, nrhs, (void *)b, n, x, n );
    }

    out[0] = dparm[DPARM_FACT_TIME];
    out[1] = dparm[DPARM_SOLV_TIME];
    out[2] = dparm[DPARM_REFINE_TIME];
    out[3] = pastix_data->solvmatr ? pastix_data->solvmatr->diagthreshold : 0.;
    out[4] = (double)iparm[IPARM_STATIC_PIVOTING];
    out[5] = (double)iparm[IPARM_NBITER];
    out[6] = dparm[DPARM_RELATIVE_ERROR];
    out[7] = dparm[DPARM_FACT_FLOPS];
    out[8] = dparm[DPARM_A_NORM];
    out[9] = rc;

    pastixFinalize( &pastix_data );
    spmExit( &spm );
    return rc;
}
