/*
 * refhost.c -- host side of the B200 backend that stays PaStiX's own code.
 *
 * PaStiX's analysis (ordering, symbolic factorization, blend) produces the
 * SolverMatrix that the numerical factorization walks.  The B200 backend keeps
 * that analysis as PaStiX's C code and reuses its integer structure bit-exact.
 * This file is compiled together with the (unmodified) PaStiX sources and
 * exposes, through plain C types, the calls a host program needs:
 *
 *   rh_analyze()        spm from CSC arrays -> pastixOrderGrid (grid nested
 *                       dissection) -> pastix_subtask_order / symbfact /
 *                       reordering / blend   (example/ordering_grid.c:87-110)
 *   rh_export_solver()  SolverMatrix cblktab/bloktab/browtab as int64 arrays
 *                       (blend/solver.h:83-213)
 *   rh_bcsc()           pastix_subtask_spm2bcsc (sopalin/pastix_task_sopalin.c:82)
 *   rh_export_bcsc()    the permuted blocked CSC (bcsc/bcsc.h:28-53) flattened
 *
 * Nothing here computes numerical factors; that is the GPU library's job.
 */
#include "common.h"
#include "spm.h"
#include "blend/solver.h"
#include "graph/graph.h"
#include "symbol/symbol.h"
#include "bcsc/bcsc.h"
#include "pastix/order.h"
#include <string.h>

typedef struct rh_s {
    pastix_data_t *pastix_data;
    pastix_int_t   iparm[IPARM_SIZE];
    double         dparm[DPARM_SIZE];
    spmatrix_t     spm;
    int            have_bcsc;
} rh_t;

/* Create the spm (CSC, 0-based) and run the PaStiX analysis with a grid
 * nested-dissection ordering.  mtxtype: 0 general, 1 symmetric (lower CSC).
 * flttype: 2 float, 3 double.  facto: PastixFactPOTRF=0, SYTRF=1, GETRF=2.
 * kv is a list of nkv (index,value) pairs applied to iparm before pastixInit;
 * the indices come from rh_param_ids(). */
/* Same with a Schur complement (pastixSetSchurUnknownList, sopalin/schur.c): the
 * nschur unknowns of schur_list (0-based, original numbering) must be the last ones
 * of the grid ordering, as PaStiX requires of a personal ordering
 * (order/pastix_subtask_order.c:145-153); the symbolic factorization then starts the
 * Schur part at column n - nschur and blend marks those cblks CBLK_IN_SCHUR. */
void *
rh_analyze_schur( int64_t n, const int64_t *colptr, const int64_t *rowind, const void *values,
                  int mtxtype, int flttype, int facto, int64_t nx, int64_t ny, int64_t nz,
                  int nthreads, int verbose, int nkv, const int64_t *kv, int64_t nschur,
                  const int64_t *schur_list, int *info );

int rh_write_order( const pastix_order_t *o, const char *path );

void *
rh_analyze( int64_t n, const int64_t *colptr, const int64_t *rowind, const void *values,
            int mtxtype, int flttype, int facto, int64_t nx, int64_t ny, int64_t nz,
            int nthreads, int verbose, int nkv, const int64_t *kv, int *info )
{
    return rh_analyze_schur( n, colptr, rowind, values, mtxtype, flttype, facto, nx, ny, nz, nthreads,
                             verbose, nkv, kv, 0, NULL, info );
}

void *
rh_analyze_schur( int64_t n, const int64_t *colptr, const int64_t *rowind, const void *values,
                  int mtxtype, int flttype, int facto, int64_t nx, int64_t ny, int64_t nz,
                  int nthreads, int verbose, int nkv, const int64_t *kv, int64_t nschur,
                  const int64_t *schur_list, int *info )
{
    rh_t *h = calloc( 1, sizeof(rh_t) );
    pastix_order_t *ord = NULL;
    int64_t nnz = colptr[n] - colptr[0];
    size_t  esz = (flttype == 2) ? sizeof(float) : sizeof(double);
    int rc;

    spmInit( &h->spm );
    h->spm.mtxtype = (mtxtype == 0) ? SpmGeneral : SpmSymmetric;
    h->spm.flttype = (flttype == 2) ? SpmFloat : SpmDouble;
    h->spm.fmttype = SpmCSC;
    h->spm.n       = n;
    h->spm.nnz     = nnz;
    h->spm.dof     = 1;
    h->spm.colptr  = malloc( (n + 1) * sizeof(spm_int_t) );
    h->spm.rowptr  = malloc( nnz * sizeof(spm_int_t) );
    h->spm.values  = malloc( nnz * esz );
    memcpy( h->spm.colptr, colptr, (n + 1) * sizeof(int64_t) );
    memcpy( h->spm.rowptr, rowind, nnz * sizeof(int64_t) );
    if ( values ) {
        memcpy( h->spm.values, values, nnz * esz );
    }
    else {
        memset( h->spm.values, 0, nnz * esz );
    }
    spmUpdateComputedFields( &h->spm );

    pastixInitParam( h->iparm, h->dparm );
    h->iparm[IPARM_VERBOSE]       = verbose ? PastixVerboseYes : PastixVerboseNot;
    h->iparm[IPARM_FACTORIZATION] = facto;
    h->iparm[IPARM_THREAD_NBR]    = nthreads > 0 ? nthreads : 1;
    h->iparm[IPARM_ORDERING]      = PastixOrderPersonal;
    for ( int i = 0; i < nkv; i++ ) {
        h->iparm[kv[2 * i]] = kv[2 * i + 1];
    }
    pastixInit( &h->pastix_data, MPI_COMM_WORLD, h->iparm, h->dparm );
    if ( nschur > 0 ) {
        pastixSetSchurUnknownList( h->pastix_data, nschur, schur_list );
        h->iparm[IPARM_SCHUR_SOLV_MODE] = PastixSolvModeInterface;
    }

    /* pastixOrderGrid fills a caller-allocated order (order/order_grids.c:306);
     * grid vertex (i,j,k) is numbered i + nx*j + nx*ny*k. */
    ord = calloc( 1, sizeof(pastix_order_t) );
    rc = pastixOrderGrid( &ord, nx, ny, nz );
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_order( h->pastix_data, &h->spm, ord );
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_symbfact( h->pastix_data );
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_reordering( h->pastix_data );
    if ( (rc == PASTIX_SUCCESS) && (h->iparm[IPARM_IO_STRATEGY] & PastixIOSave) &&
         (h->pastix_data->dir_global != NULL) ) {
        /* the reordered ordering, beside the symbol file the reordering step saved
         * (before blend, which splits the ordering's column blocks) */
        char path[4096];
        snprintf( path, sizeof(path), "%s/ordergen", h->pastix_data->dir_global );
        rc = rh_write_order( h->pastix_data->ordemesh, path );
    }
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_blend( h->pastix_data );
    if ( ord ) {
        pastixOrderExit( ord );
        free( ord );
    }
    *info = rc;
    return h;
}

/* The symbolic-factorization step of an analysis loaded from files: what
 * pastix_subtask_symbfact does under PastixIOLoad (symbol/pastix_subtask_symbfact.c:157-165,
 * then :248-330), with two gaps of that path filled.  Its symbol structure is
 * malloc'ed and never initialised (:150-155; pastixSymbolInit sets dof, schurfcol and
 * the row tables), and pastixSymbolLoad (symbol/symbol_io.c:50-130) does not restore
 * the blocks' lcblknm, which pastixSymbolCheck (symbol/symbol_check.c:88-95) and the
 * solver build read.  Here the structure is initialised, lcblknm is set from the
 * column blocks' block ranges and the Schur start from the graph, then the steps after
 * the fax follow (rebase, row tables, selevtx, NNZ and flop counts, step bits). */
static int
rh_symbol_load( pastix_data_t *pd, const char *path )
{
    symbol_matrix_t *s;
    FILE *f;
    pastix_int_t k, b;

    if ( !(pd->steps & STEP_ORDERING) || (pd->graph == NULL) || (pd->ordemesh == NULL) ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    pastixOrderBase( pd->ordemesh, 0 );
    s = malloc( sizeof(symbol_matrix_t) );
    pastixSymbolInit( NULL, NULL, s );
    f = fopen( path, "r" );
    if ( f == NULL ) {
        free( s );
        return PASTIX_ERR_FILE;
    }
    if ( pastixSymbolLoad( s, f ) != 0 ) {
        fclose( f );
        free( s );
        return PASTIX_ERR_FILE;
    }
    fclose( f );
    if ( s->nodenbr != pd->graph->gN ) {
        pastixSymbolExit( s );
        free( s );
        return PASTIX_ERR_BADPARAMETER;
    }
    for ( k = 0; k < s->cblknbr; k++ ) {
        for ( b = s->cblktab[k].bloknum; b < s->cblktab[k + 1].bloknum; b++ ) {
            s->bloktab[b - s->baseval].lcblknm = k + s->baseval;
        }
    }
    s->schurfcol = pd->graph->gN - pd->schur_n + s->baseval;
    pastixSymbolBase( s, 0 );
    pastixSymbolBuildRowtab( s );
    pastixSymbolRealloc( s );
    if ( pd->ordemesh->selevtx != NULL ) {
        for ( k = 0; k < s->cblknbr; k++ ) {
            s->cblktab[k].selevtx = pd->ordemesh->selevtx[k];
        }
    }
    if ( pastixSymbolCheck( s ) != 0 ) {
        pastixSymbolExit( s );
        free( s );
        return PASTIX_ERR_BADPARAMETER;
    }
    pd->symbmtx = s;
    pd->iparm[IPARM_NNZEROS] = pastixSymbolGetNNZ( s );
    pastixSymbolGetFlops( s, pd->iparm[IPARM_FLOAT], pd->iparm[IPARM_FACTORIZATION],
                          &(pd->dparm[DPARM_FACT_THFLOPS]), &(pd->dparm[DPARM_FACT_RLFLOPS]) );
    pd->steps &= ~( STEP_ANALYSE | STEP_CSC2BCSC | STEP_BCSC2CTAB | STEP_NUMFACT | STEP_SOLVE | STEP_REFINE );
    pd->steps |= STEP_SYMBFACT;
    return PASTIX_SUCCESS;
}

/* The analysis from PaStiX's own saved files: the working directory holds
 * "ordername" and "symbname" as written by an analysis run with IPARM_IO_STRATEGY =
 * PastixIOSave ("ordergen" and "symbgen" of its pastix-XXXXXX directory, renamed to
 * the names the loaders read).  pastix_subtask_order loads the ordering
 * (order/pastix_subtask_order.c:310-315), rh_symbol_load the symbol matrix, and blend
 * builds the SolverMatrix; the reordering step is not run again, the saved
 * ordering and symbol being the reordered ones (symbol/pastix_subtask_reordering.c:102-106).
 * No ordering or symbolic factorization is computed. */
void *
rh_analyze_load( int64_t n, const int64_t *colptr, const int64_t *rowind, const void *values,
                 int mtxtype, int flttype, int facto, int nthreads, int verbose, int nkv, const int64_t *kv,
                 int *info )
{
    rh_t *h = calloc( 1, sizeof(rh_t) );
    int64_t nnz = colptr[n] - colptr[0];
    size_t  esz = (flttype == 2) ? sizeof(float) : sizeof(double);
    int rc;

    spmInit( &h->spm );
    h->spm.mtxtype = (mtxtype == 0) ? SpmGeneral : SpmSymmetric;
    h->spm.flttype = (flttype == 2) ? SpmFloat : SpmDouble;
    h->spm.fmttype = SpmCSC;
    h->spm.n       = n;
    h->spm.nnz     = nnz;
    h->spm.dof     = 1;
    h->spm.colptr  = malloc( (n + 1) * sizeof(spm_int_t) );
    h->spm.rowptr  = malloc( nnz * sizeof(spm_int_t) );
    h->spm.values  = malloc( nnz * esz );
    memcpy( h->spm.colptr, colptr, (n + 1) * sizeof(int64_t) );
    memcpy( h->spm.rowptr, rowind, nnz * sizeof(int64_t) );
    if ( values ) {
        memcpy( h->spm.values, values, nnz * esz );
    }
    else {
        memset( h->spm.values, 0, nnz * esz );
    }
    spmUpdateComputedFields( &h->spm );

    pastixInitParam( h->iparm, h->dparm );
    h->iparm[IPARM_VERBOSE]       = verbose ? PastixVerboseYes : PastixVerboseNot;
    h->iparm[IPARM_FACTORIZATION] = facto;
    h->iparm[IPARM_THREAD_NBR]    = nthreads > 0 ? nthreads : 1;
    h->iparm[IPARM_ORDERING]      = PastixOrderPersonal;
    for ( int i = 0; i < nkv; i++ ) {
        h->iparm[kv[2 * i]] = kv[2 * i + 1];
    }
    h->iparm[IPARM_IO_STRATEGY] = PastixIOLoad;
    pastixInit( &h->pastix_data, MPI_COMM_WORLD, h->iparm, h->dparm );
    rc = pastix_subtask_order( h->pastix_data, &h->spm, NULL );
    if ( rc == PASTIX_SUCCESS ) rc = rh_symbol_load( h->pastix_data, "symbname" );
    if ( rc == PASTIX_SUCCESS ) rc = pastix_subtask_blend( h->pastix_data );
    h->iparm[IPARM_IO_STRATEGY] = PastixIONo;
    *info = rc;
    return h;
}

/* Write an ordering (rangtab, permtab, treetab) to path in the text format
 * pastixOrderLoad reads (order/order_io.c:40-110: version 1, cblknbr, vertnbr, then
 * the three arrays).  PaStiX's own pastixOrderSave writes only when procnbr == 0
 * (order/order_io.c:321), which never holds, so an analysis run with PastixIOSave
 * leaves its symbol file but not its ordering; rh_analyze writes it instead. */
int
rh_write_order( const pastix_order_t *o, const char *path )
{
    FILE *f;
    pastix_int_t i;
    if ( (o == NULL) || (o->permtab == NULL) || (o->rangtab == NULL) || (o->treetab == NULL) ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    f = fopen( path, "w" );
    if ( f == NULL ) {
        return PASTIX_ERR_FILE;
    }
    fprintf( f, "1\n%ld\t%ld\n", (long)o->cblknbr, (long)o->vertnbr );
    for ( i = 0; i <= o->cblknbr; i++ ) {
        fprintf( f, "%ld%c", (long)o->rangtab[i], ((i & 7) == 7) ? '\n' : '\t' );
    }
    fputc( '\n', f );
    for ( i = 0; i < o->vertnbr; i++ ) {
        fprintf( f, "%ld%c", (long)o->permtab[i], ((i & 7) == 7) ? '\n' : '\t' );
    }
    fputc( '\n', f );
    for ( i = 0; i < o->cblknbr; i++ ) {
        fprintf( f, "%ld%c", (long)o->treetab[i], ((i & 7) == 7) ? '\n' : '\t' );
    }
    fputc( '\n', f );
    return fclose( f ) == 0 ? PASTIX_SUCCESS : PASTIX_ERR_FILE;
}

/* The directory where an analysis run with PastixIOSave wrote its files (NULL if
 * none). */
const char *
rh_io_dir( void *vh )
{
    return ((rh_t *)vh)->pastix_data->dir_global;
}

/* Index of the iparm/dparm entries a host program sets or reads, in a fixed
 * order: MIN_BLOCKSIZE, MAX_BLOCKSIZE, SCHEDULER, THREAD_NBR, TASKS2D_LEVEL,
 * REFINEMENT, ITERMAX, GMRES_IM, FACTORIZATION, NBITER, STATIC_PIVOTING,
 * NNZEROS, IO_STRATEGY, IPARM_SIZE | DPARM_EPSILON_REFINEMENT, DPARM_EPSILON_MAGN_CTRL,
 * DPARM_A_NORM, DPARM_FACT_TIME, DPARM_SOLV_TIME, DPARM_REFINE_TIME,
 * DPARM_FACT_THFLOPS, DPARM_RELATIVE_ERROR, DPARM_SIZE. */
void
rh_param_ids( int64_t *ids )
{
    int64_t v[] = { IPARM_MIN_BLOCKSIZE, IPARM_MAX_BLOCKSIZE, IPARM_SCHEDULER, IPARM_THREAD_NBR,
                    IPARM_TASKS2D_LEVEL, IPARM_REFINEMENT, IPARM_ITERMAX, IPARM_GMRES_IM,
                    IPARM_FACTORIZATION, IPARM_NBITER, IPARM_STATIC_PIVOTING, IPARM_NNZEROS,
                    IPARM_IO_STRATEGY, IPARM_SIZE,
                    DPARM_EPSILON_REFINEMENT, DPARM_EPSILON_MAGN_CTRL, DPARM_A_NORM,
                    DPARM_FACT_TIME, DPARM_SOLV_TIME, DPARM_REFINE_TIME, DPARM_FACT_THFLOPS,
                    DPARM_RELATIVE_ERROR, DPARM_SIZE };
    memcpy( ids, v, sizeof(v) );
}

/* Direct access to the instance's iparm/dparm arrays (read or write). */
int64_t *
rh_iparm( void *vh )
{
    return ((rh_t *)vh)->iparm;
}

double *
rh_dparm( void *vh )
{
    return ((rh_t *)vh)->dparm;
}

/* sizes[0..10] = n, cblknbr, bloknbr, brownbr, coefnbr, bcsc nnz, facto, flttype, gN, cblkmaxblk,
 * cblkschur (first cblk of the Schur complement; cblknbr without one) */
void
rh_sizes( void *vh, int64_t *sizes )
{
    rh_t *h = vh;
    SolverMatrix *s = h->pastix_data->solvmatr;
    sizes[0] = h->spm.n;
    sizes[1] = s->cblknbr;
    sizes[2] = s->bloknbr;
    sizes[3] = s->brownbr;
    sizes[4] = s->coefnbr;
    sizes[5] = (h->have_bcsc && h->pastix_data->bcsc->cscfnbr > 0)
        ? h->pastix_data->bcsc->cscftab[h->pastix_data->bcsc->cscfnbr - 1].coltab[
              h->pastix_data->bcsc->cscftab[h->pastix_data->bcsc->cscfnbr - 1].colnbr]
        : -1;
    sizes[6] = h->iparm[IPARM_FACTORIZATION];
    sizes[7] = h->spm.flttype;
    sizes[8] = h->spm.gN;
    sizes[9] = s->cblkmaxblk;
    sizes[10] = s->cblkschur;
}

/* cblk arrays have cblknbr+1 entries (the sentinel cblk is exported too);
 * blok arrays have bloknbr+1 entries; browtab has brownbr entries.
 * cblk_fblok is the index of the first block of each cblk (fblokptr - bloktab). */
void
rh_export_solver( void *vh, int64_t *cblk_fcolnum, int64_t *cblk_lcolnum, int64_t *cblk_fblok,
                  int64_t *cblk_stride, int64_t *cblk_lcolidx, int64_t *cblk_brownum,
                  int64_t *cblk_brown2d, int32_t *cblk_type,
                  int64_t *blok_frownum, int64_t *blok_lrownum, int64_t *blok_lcblknm,
                  int64_t *blok_fcblknm, int64_t *blok_coefind, int64_t *blok_browind,
                  int64_t *browtab )
{
    rh_t *h = vh;
    SolverMatrix *s = h->pastix_data->solvmatr;
    for ( pastix_int_t k = 0; k <= s->cblknbr; k++ ) {
        SolverCblk *c = s->cblktab + k;
        cblk_fcolnum[k] = c->fcolnum;
        cblk_lcolnum[k] = c->lcolnum;
        cblk_fblok[k]   = c->fblokptr - s->bloktab;
        cblk_stride[k]  = c->stride;
        cblk_lcolidx[k] = c->lcolidx;
        cblk_brownum[k] = c->brownum;
        cblk_brown2d[k] = c->brown2d;
        cblk_type[k]    = c->cblktype;
    }
    for ( pastix_int_t b = 0; b <= s->bloknbr; b++ ) {
        SolverBlok *bl = s->bloktab + b;
        blok_frownum[b] = bl->frownum;
        blok_lrownum[b] = bl->lrownum;
        blok_lcblknm[b] = bl->lcblknm;
        blok_fcblknm[b] = bl->fcblknm;
        blok_coefind[b] = bl->coefind;
        blok_browind[b] = bl->browind;
    }
    for ( pastix_int_t i = 0; i < s->brownbr; i++ ) {
        browtab[i] = s->browtab[i];
    }
}

void
rh_export_perm( void *vh, int64_t *permtab, int64_t *peritab )
{
    rh_t *h = vh;
    pastix_order_t *o = h->pastix_data->ordemesh;
    memcpy( permtab, o->permtab, o->vertnbr * sizeof(int64_t) );
    memcpy( peritab, o->peritab, o->vertnbr * sizeof(int64_t) );
}

/* dparm[DPARM_FACT_THFLOPS] computed by blend (symbol/symbol_cost.c) */
double
rh_thflops( void *vh )
{
    rh_t *h = vh;
    return h->dparm[DPARM_FACT_THFLOPS];
}

/* Replace the spm values (same pattern) and build the blocked CSC. */
int
rh_bcsc( void *vh, const void *values )
{
    rh_t *h = vh;
    size_t esz = (h->spm.flttype == SpmFloat) ? sizeof(float) : sizeof(double);
    if ( values ) {
        memcpy( h->spm.values, values, h->spm.nnz * esz );
    }
    int rc = pastix_subtask_spm2bcsc( h->pastix_data, &h->spm );
    h->have_bcsc = (rc == PASTIX_SUCCESS);
    return rc;
}

double
rh_anorm( void *vh )
{
    rh_t *h = vh;
    return h->dparm[DPARM_A_NORM];
}

/* colptr: n+1 entries over the permuted column numbering (cblk order);
 * Lvalues: the bcsc values (A, both triangles for symmetric matrices);
 * Uvalues: A^T values (LU only; may be NULL). */
void
rh_export_bcsc( void *vh, int64_t *colptr, int64_t *rowtab, void *Lvalues, void *Uvalues )
{
    rh_t *h = vh;
    pastix_bcsc_t *b = h->pastix_data->bcsc;
    size_t esz = (b->flttype == PastixFloat) ? sizeof(float) : sizeof(double);
    int64_t col = 0, nnz;
    for ( pastix_int_t k = 0; k < b->cscfnbr; k++ ) {
        for ( pastix_int_t j = 0; j < b->cscftab[k].colnbr; j++ ) {
            colptr[col++] = b->cscftab[k].coltab[j];
        }
    }
    nnz = b->cscftab[b->cscfnbr - 1].coltab[b->cscftab[b->cscfnbr - 1].colnbr];
    colptr[col] = nnz;
    memcpy( rowtab, b->rowtab, nnz * sizeof(int64_t) );
    memcpy( Lvalues, b->Lvalues, nnz * esz );
    if ( Uvalues && b->Uvalues ) {
        memcpy( Uvalues, b->Uvalues, nnz * esz );
    }
}

/* The pastix_data handle, for the oracle driver that runs PaStiX's own
 * numerical factorization on the same analysis. */
void *
rh_pastix_data( void *vh )
{
    return ((rh_t *)vh)->pastix_data;
}

void *
rh_spm( void *vh )
{
    return &((rh_t *)vh)->spm;
}

void
rh_free( void *vh )
{
    rh_t *h = vh;
    if ( !h ) return;
    pastixFinalize( &h->pastix_data );
    spmExit( &h->spm );
    free( h );
}
