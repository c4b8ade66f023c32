/*
 * ref_driver.c -- TEST INFRASTRUCTURE (oracle).  Runs PaStiX's own CPU
 * numerical factorization, solve and refinement on an analysis produced by the
 * host library, and exports PaStiX's factor so the restated oracle and the GPU
 * path can be compared against it.  Built into oracle/_ref/ by
 * oracle/build_oracle.py; only tests, the smoke check and the benchmark's CPU
 * baseline may load it.
 *
 * Entry points follow PaStiX's public API:
 *   rd_numfact  -> pastix_task_numfact  (sopalin/pastix_task_sopalin.c:563)
 *   rd_solve    -> pastix_task_solve    (sopalin/pastix_task_solve.c:550)
 *   rd_refine   -> pastix_task_refine   (refinement/pastix_task_refine.c:226)
 *   rd_export_coeftab copies every cblk's lcoeftab/ucoeftab (2D layout,
 *   kernels/cpucblk_zinit.c:48-139) into one array in cblk order.
 */
#include "common.h"
#include "spm.h"
#include "blend/solver.h"
#include "bcsc/bcsc.h"
#include <string.h>

int
rd_numfact( pastix_data_t *pastix_data, spmatrix_t *spm, int scheduler )
{
    pastix_data->iparm[IPARM_SCHEDULER] = scheduler;
    return pastix_task_numfact( pastix_data, spm );
}

int
rd_solve( pastix_data_t *pastix_data, int64_t nrhs, void *b, int64_t ldb )
{
    return pastix_task_solve( pastix_data, nrhs, b, ldb );
}

int
rd_refine( pastix_data_t *pastix_data, int64_t n, int64_t nrhs, void *b, int64_t ldb,
           void *x, int64_t ldx )
{
    return pastix_task_refine( pastix_data, n, nrhs, b, ldb, x, ldx );
}

/* Copy PaStiX's factor: L (and U for LU) of every cblk, concatenated in cblk
 * order, each cblk stride*ncols entries in its 2D block layout. */
void
rd_export_coeftab( pastix_data_t *pastix_data, void *L, void *U )
{
    SolverMatrix *s = pastix_data->solvmatr;
    size_t esz = (pastix_data->bcsc->flttype == PastixFloat) ? sizeof(float) : sizeof(double);
    char *pl = L, *pu = U;
    for ( pastix_int_t k = 0; k < s->cblknbr; k++ ) {
        SolverCblk *c = s->cblktab + k;
        size_t cnt = (size_t)c->stride * (size_t)cblk_colnbr( c );
        memcpy( pl, c->lcoeftab, cnt * esz );
        pl += cnt * esz;
        if ( pu && c->ucoeftab ) {
            memcpy( pu, c->ucoeftab, cnt * esz );
            pu += cnt * esz;
        }
    }
}

/* out = { fact time, solve time, refine time, static pivots, refinement iters,
 *         diagthreshold } */
void
rd_stats( pastix_data_t *pastix_data, double *out )
{
    out[0] = pastix_data->dparm[DPARM_FACT_TIME];
    out[1] = pastix_data->dparm[DPARM_SOLV_TIME];
    out[2] = pastix_data->dparm[DPARM_REFINE_TIME];
    out[3] = (double)pastix_data->iparm[IPARM_STATIC_PIVOTING];
    out[4] = (double)pastix_data->iparm[IPARM_NBITER];
    out[5] = pastix_data->solvmatr->diagthreshold;
}
