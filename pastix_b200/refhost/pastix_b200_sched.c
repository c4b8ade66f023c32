/*
 * pastix_b200_sched.c -- the B200 backend behind PaStiX's own entry points.
 *
 * Compiled into a build of PaStiX's sources whose task entry points call these hooks
 * when iparm[IPARM_SCHEDULER] is PastixSchedB200 or PastixSchedB200Mixed
 * (pastix_b200/refhost/build_sched.py inserts the calls), and linked against
 * libpastix_b200.so.  Every hook reads what the CPU path reads (the SolverMatrix, the
 * bcsc, ordemesh->peritab, iparm/dparm) and writes what it writes (diagthreshold,
 * nbpivots, IPARM_STATIC_PIVOTING, IPARM_NBITER, the times, the step bits), so a
 * PaStiX program switches backends by one iparm entry.
 *
 * The GPU factor instance of each pastix_data_t is kept in a small table here (the
 * pastix_data_t layout is left as it is); pastixFinalize releases it.
 */
#include "common.h"
#include "spm.h"
#include "blend/solver.h"
#include "bcsc/bcsc.h"
#include "pastix/order.h"
#include "pastix_b200.h"
#include "pastix_b200_sched.h"
#include <pthread.h>
#include <string.h>
#include <time.h>

typedef struct b200_entry_s {
    const pastix_data_t *pastix_data;
    b200_solver_t       *solver;
    int                  facto, precision;
    struct b200_entry_s *next;
} b200_entry_t;

static b200_entry_t   *b200_entries = NULL;
static pthread_mutex_t b200_lock    = PTHREAD_MUTEX_INITIALIZER;

static double
b200_wtime( void )
{
    struct timespec t;
    clock_gettime( CLOCK_MONOTONIC, &t );
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static b200_entry_t *
b200_entry( const pastix_data_t *pastix_data, int create )
{
    b200_entry_t *e;
    pthread_mutex_lock( &b200_lock );
    for ( e = b200_entries; e != NULL; e = e->next ) {
        if ( e->pastix_data == pastix_data ) {
            break;
        }
    }
    if ( (e == NULL) && create ) {
        e = calloc( 1, sizeof(b200_entry_t) );
        e->pastix_data = pastix_data;
        e->next        = b200_entries;
        b200_entries   = e;
    }
    pthread_mutex_unlock( &b200_lock );
    return e;
}

int
pastix_b200_scheduler( const pastix_data_t *pastix_data )
{
    pastix_int_t s = pastix_data->iparm[IPARM_SCHEDULER];
    return (s == PastixSchedB200) || (s == PastixSchedB200Mixed);
}

void *
pastix_b200_solver( pastix_data_t *pastix_data )
{
    b200_entry_t *e = b200_entry( pastix_data, 0 );
    return e ? e->solver : NULL;
}

/* PaStiX's factorization kinds for real arithmetic: LL^t and LL^h are the same
 * Cholesky, LDL^t and LDL^h the same LDL^t (include/pastix/api.h:271-283) */
static int
b200_facto( pastix_int_t f )
{
    switch ( f ) {
    case PastixFactPOTRF:
    case PastixFactPXTRF:
        return B200_FACTO_POTRF;
    case PastixFactSYTRF:
    case PastixFactHETRF:
        return B200_FACTO_SYTRF;
    case PastixFactGETRF:
        return B200_FACTO_GETRF;
    default:
        return -1;
    }
}

static int
b200_precision( const pastix_data_t *pastix_data )
{
    if ( pastix_data->iparm[IPARM_SCHEDULER] == PastixSchedB200Mixed ) {
        return B200_PREC_TF32X3;
    }
    return ( pastix_data->bcsc->flttype == PastixFloat ) ? B200_PREC_FP32 : B200_PREC_FP64;
}

/* The SolverMatrix tables (blend/solver.h:83-213) as the int64 arrays of b200_symbol_t,
 * and the GPU instance built from them. */
static int
b200_create( pastix_data_t *pastix_data, int facto, int precision, b200_solver_t **out )
{
    const SolverMatrix *s = pastix_data->solvmatr;
    pastix_int_t C = s->cblknbr, B = s->bloknbr, k, b;
    int64_t *buf = malloc( sizeof(int64_t) * ( 6 * (C + 1) + 4 * (B + 1) + s->brownbr + 1 ) );
    int64_t *p = buf;
    b200_symbol_t sym;
    int rc;

    if ( buf == NULL ) {
        return PASTIX_ERR_OUTOFMEMORY;
    }
    sym.n       = pastix_data->bcsc->gN;
    sym.cblknbr = C;
    sym.bloknbr = B;
    sym.brownbr = s->brownbr;
    int64_t *fcol = p;  p += C + 1;
    int64_t *lcol = p;  p += C + 1;
    int64_t *fblk = p;  p += C + 1;
    int64_t *strd = p;  p += C + 1;
    int64_t *lidx = p;  p += C + 1;
    int64_t *brwn = p;  p += C + 1;
    int64_t *frow = p;  p += B + 1;
    int64_t *lrow = p;  p += B + 1;
    int64_t *lcbk = p;  p += B + 1;
    int64_t *fcbk = p;  p += B + 1;
    int64_t *brow = p;
    for ( k = 0; k <= C; k++ ) {
        const SolverCblk *c = s->cblktab + k;
        fcol[k] = c->fcolnum;
        lcol[k] = c->lcolnum;
        fblk[k] = c->fblokptr - s->bloktab;
        strd[k] = c->stride;
        lidx[k] = c->lcolidx;
        brwn[k] = c->brownum;
    }
    for ( b = 0; b <= B; b++ ) {
        const SolverBlok *bl = s->bloktab + b;
        frow[b] = bl->frownum;
        lrow[b] = bl->lrownum;
        lcbk[b] = bl->lcblknm;
        fcbk[b] = bl->fcblknm;
    }
    for ( b = 0; b < s->brownbr; b++ ) {
        brow[b] = s->browtab[b];
    }
    sym.cblk_fcolnum = fcol;
    sym.cblk_lcolnum = lcol;
    sym.cblk_fblok   = fblk;
    sym.cblk_stride  = strd;
    sym.cblk_lcolidx = lidx;
    sym.cblk_brownum = brwn;
    sym.blok_frownum = frow;
    sym.blok_lrownum = lrow;
    sym.blok_lcblknm = lcbk;
    sym.blok_fcblknm = fcbk;
    sym.browtab      = brow;
    sym.peritab      = pastix_data->ordemesh->peritab;
    rc = b200_solver_create_schur( &sym, facto, precision, NULL, s->cblkschur, out );
    free( buf );
    return rc;
}

int
pastix_b200_subtask_bcsc2ctab( pastix_data_t *pastix_data )
{
    pastix_bcsc_t *bcsc = pastix_data->bcsc;
    b200_entry_t  *e;
    int facto = b200_facto( pastix_data->iparm[IPARM_FACTORIZATION] );
    int prec, rc;
    pastix_int_t n = bcsc->gN, nnz, col = 0, k, j;
    int64_t *colptr;
    double  *Lv, *Uv = NULL;

    if ( (bcsc->flttype != PastixDouble) && (bcsc->flttype != PastixFloat) ) {
        errorPrint( "pastix_b200: complex arithmetic is not supported by the B200 backend" );
        return PASTIX_ERR_NOTIMPLEMENTED;
    }
    if ( facto < 0 ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    prec = b200_precision( pastix_data );
    e = b200_entry( pastix_data, 1 );
    if ( (e->solver != NULL) && ((e->facto != facto) || (e->precision != prec)) ) {
        b200_solver_destroy( e->solver );
        e->solver = NULL;
    }
    if ( e->solver == NULL ) {
        rc = b200_create( pastix_data, facto, prec, &e->solver );
        if ( rc != PASTIX_SUCCESS ) {
            return rc;
        }
        e->facto     = facto;
        e->precision = prec;
    }

    /* the bcsc (bcsc/bcsc.h:28-53) with one column pointer over the permuted columns */
    colptr = malloc( (n + 1) * sizeof(int64_t) );
    for ( k = 0; k < bcsc->cscfnbr; k++ ) {
        for ( j = 0; j < bcsc->cscftab[k].colnbr; j++ ) {
            colptr[col++] = bcsc->cscftab[k].coltab[j];
        }
    }
    nnz = bcsc->cscftab[bcsc->cscfnbr - 1].coltab[bcsc->cscftab[bcsc->cscfnbr - 1].colnbr];
    colptr[col] = nnz;
    if ( bcsc->flttype == PastixDouble ) {
        Lv = bcsc->Lvalues;
        Uv = bcsc->Uvalues;
    }
    else {
        const float *lf = bcsc->Lvalues, *uf = bcsc->Uvalues;
        Lv = malloc( nnz * sizeof(double) );
        for ( j = 0; j < nnz; j++ ) Lv[j] = lf[j];
        if ( uf != NULL ) {
            Uv = malloc( nnz * sizeof(double) );
            for ( j = 0; j < nnz; j++ ) Uv[j] = uf[j];
        }
    }
    rc = b200_bcsc_load( e->solver, nnz, colptr, bcsc->rowtab, Lv,
                         (facto == B200_FACTO_GETRF) ? Uv : NULL, pastix_data->dparm[DPARM_A_NORM] );
    if ( bcsc->flttype != PastixDouble ) {
        free( Lv );
        free( Uv );
    }
    free( colptr );
    if ( rc != PASTIX_SUCCESS ) {
        return rc;
    }
    pastix_data->solvmatr->factotype = pastix_data->iparm[IPARM_FACTORIZATION];
    pastix_data->steps &= ~STEP_NUMFACT;
    pastix_data->steps |= STEP_BCSC2CTAB;
    return PASTIX_SUCCESS;
}

int
pastix_b200_subtask_sopalin( pastix_data_t *pastix_data )
{
    b200_entry_t *e = b200_entry( pastix_data, 0 );
    int64_t npiv = 0;
    double  st[13], t0, t;
    int rc;

    if ( (e == NULL) || (e->solver == NULL) ) {
        errorPrint( "pastix_b200: pastix_subtask_bcsc2ctab has to be called before the factorization" );
        return PASTIX_ERR_BADPARAMETER;
    }
    t0 = b200_wtime();
    /* the threshold rule of sopalin/pastix_task_sopalin.c:401-425 on DPARM_A_NORM */
    rc = b200_numfact( e->solver, pastix_data->dparm[DPARM_EPSILON_MAGN_CTRL], &npiv );
    t  = b200_wtime() - t0;
    if ( rc != PASTIX_SUCCESS ) {
        return rc;
    }
    b200_stats( e->solver, st );
    pastix_data->solvmatr->diagthreshold      = st[4];
    pastix_data->solvmatr->nbpivots           = npiv;
    pastix_data->iparm[IPARM_STATIC_PIVOTING] = npiv;
    pastix_data->dparm[DPARM_FACT_TIME]       = t;
    pastix_data->dparm[DPARM_FACT_FLOPS]      = pastix_data->dparm[DPARM_FACT_THFLOPS] / t / 1073741824.;
    pastix_data->steps &= ~( STEP_BCSC2CTAB | STEP_SOLVE | STEP_REFINE );
    pastix_data->steps |= STEP_NUMFACT;
    return PASTIX_SUCCESS;
}

/* Vectors in the matrix's precision: double as is, float through a double copy */
static double *
b200_vec_in( const pastix_data_t *pastix_data, const void *v, pastix_int_t n, pastix_int_t nrhs,
             pastix_int_t ld, pastix_int_t *ldd )
{
    pastix_int_t i, j;
    double *d;
    if ( pastix_data->bcsc->flttype == PastixDouble ) {
        *ldd = ld;
        return (double *)v;
    }
    d = malloc( (size_t)n * nrhs * sizeof(double) );
    for ( j = 0; j < nrhs; j++ ) {
        for ( i = 0; i < n; i++ ) {
            d[i + j * n] = ((const float *)v)[i + j * ld];
        }
    }
    *ldd = n;
    return d;
}

static void
b200_vec_out( const pastix_data_t *pastix_data, double *d, void *v, pastix_int_t n, pastix_int_t nrhs,
              pastix_int_t ld, int copy )
{
    pastix_int_t i, j;
    if ( pastix_data->bcsc->flttype == PastixDouble ) {
        return;
    }
    if ( copy ) {
        for ( j = 0; j < nrhs; j++ ) {
            for ( i = 0; i < n; i++ ) {
                ((float *)v)[i + j * ld] = (float)d[i + j * n];
            }
        }
    }
    free( d );
}

static b200_entry_t *
b200_factored( pastix_data_t *pastix_data, const char *who )
{
    b200_entry_t *e = b200_entry( pastix_data, 0 );
    if ( !(pastix_data->steps & STEP_NUMFACT) || (e == NULL) || (e->solver == NULL) ) {
        errorPrint( "%s: pastix_task_numfact() has to be called before calling this function", who );
        return NULL;
    }
    return e;
}

int
pastix_b200_task_solve( pastix_data_t *pastix_data, pastix_int_t nrhs, void *b, pastix_int_t ldb )
{
    b200_entry_t *e = b200_factored( pastix_data, "pastix_task_solve" );
    pastix_int_t n = pastix_data->bcsc->gN, ldd;
    double *d, t0;
    int rc;

    if ( e == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    t0 = b200_wtime();
    if ( pastix_data->bcsc->flttype == PastixFloat ) {
        rc = b200_solve_float( e->solver, nrhs, b, ldb );
    }
    else {
        d  = b200_vec_in( pastix_data, b, n, nrhs, ldb, &ldd );
        rc = b200_solve( e->solver, nrhs, d, ldd );
        b200_vec_out( pastix_data, d, b, n, nrhs, ldb, rc == PASTIX_SUCCESS );
    }
    pastix_data->dparm[DPARM_SOLV_TIME] = b200_wtime() - t0;
    if ( rc == PASTIX_SUCCESS ) {
        pastix_data->steps |= STEP_SOLVE;
    }
    return rc;
}

/* one step of b200_trsm (0 forward, 1 backward, 2 D^-1) on a permuted b */
static int
b200_step( pastix_data_t *pastix_data, b200_entry_t *e, int step, pastix_int_t nrhs, void *b,
           pastix_int_t ldb )
{
    pastix_int_t n = pastix_data->bcsc->gN, ldd;
    double *d = b200_vec_in( pastix_data, b, n, nrhs, ldb, &ldd );
    int rc = b200_trsm( e->solver, step, nrhs, d, ldd );
    b200_vec_out( pastix_data, d, b, n, nrhs, ldb, rc == PASTIX_SUCCESS );
    return rc;
}

int
pastix_b200_subtask_trsm( pastix_data_t *pastix_data, pastix_coeftype_t flttype, pastix_side_t side,
                          pastix_uplo_t uplo, pastix_trans_t trans, pastix_diag_t diag,
                          pastix_int_t nrhs, void *b, pastix_int_t ldb )
{
    b200_entry_t *e = b200_factored( pastix_data, "pastix_subtask_trsm" );
    if ( e == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    if ( (flttype != pastix_data->bcsc->flttype) || (side != PastixLeft) ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    /* the two sweeps of pastix_subtask_solve (sopalin/pastix_task_solve.c:434-505):
     * L y = b forward; L^t x = y, or U x = y for LU, backward */
    if ( (uplo == PastixLower) && (trans == PastixNoTrans) ) {
        return b200_step( pastix_data, e, 0, nrhs, b, ldb );
    }
    if ( ((uplo == PastixLower) && (trans != PastixNoTrans)) ||
         ((uplo == PastixUpper) && (trans == PastixNoTrans) && (e->facto == B200_FACTO_GETRF)) ) {
        return b200_step( pastix_data, e, 1, nrhs, b, ldb );
    }
    (void)diag;
    return PASTIX_ERR_NOTIMPLEMENTED;
}

int
pastix_b200_subtask_diag( pastix_data_t *pastix_data, pastix_coeftype_t flttype, pastix_int_t nrhs,
                          void *b, pastix_int_t ldb )
{
    b200_entry_t *e = b200_factored( pastix_data, "pastix_subtask_diag" );
    if ( (e == NULL) || (flttype != pastix_data->bcsc->flttype) ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    return b200_step( pastix_data, e, 2, nrhs, b, ldb );
}

int
pastix_b200_subtask_solve( pastix_data_t *pastix_data, pastix_int_t nrhs, void *b, pastix_int_t ldb )
{
    b200_entry_t *e = b200_factored( pastix_data, "pastix_subtask_solve" );
    double t0 = b200_wtime();
    int rc;
    if ( e == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    rc = b200_step( pastix_data, e, 0, nrhs, b, ldb );
    if ( (rc == PASTIX_SUCCESS) && (e->facto == B200_FACTO_SYTRF) ) {
        rc = b200_step( pastix_data, e, 2, nrhs, b, ldb );
    }
    if ( rc == PASTIX_SUCCESS ) {
        rc = b200_step( pastix_data, e, 1, nrhs, b, ldb );
    }
    pastix_data->dparm[DPARM_SOLV_TIME] = b200_wtime() - t0;
    return rc;
}

int
pastix_b200_task_refine( pastix_data_t *pastix_data, pastix_int_t n, pastix_int_t nrhs, void *b,
                         pastix_int_t ldb, void *x, pastix_int_t ldx )
{
    b200_entry_t *e = b200_factored( pastix_data, "pastix_task_refine" );
    pastix_int_t  gN = pastix_data->bcsc->gN, ldbd, ldxd, j;
    pastix_int_t  method = pastix_data->iparm[IPARM_REFINEMENT];
    int64_t niter = 0;
    double *db, *dx, *berr, t0, emax = 0.;
    int rc;

    if ( e == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    if ( (method != PastixRefineGMRES) && (method != PastixRefineCG) && (method != PastixRefineSR) &&
         (method != PastixRefineBiCGSTAB) ) {
        errorPrint( "pastix_b200: unknown refinement method %ld", (long)method );
        return PASTIX_ERR_BADPARAMETER;
    }
    t0   = b200_wtime();
    berr = malloc( (nrhs > 0 ? nrhs : 1) * sizeof(double) );
    /* GMRES = 0, CG = 1, SR = 2, BiCGSTAB = 3 in both enums (include/pastix/api.h:241-246) */
    if ( pastix_data->bcsc->flttype == PastixFloat ) {
        rc = b200_refine_float( e->solver, nrhs, b, ldb, x, ldx, (int)method,
                                pastix_data->dparm[DPARM_EPSILON_REFINEMENT], pastix_data->iparm[IPARM_ITERMAX],
                                pastix_data->iparm[IPARM_GMRES_IM], &niter, berr );
    }
    else {
        db = b200_vec_in( pastix_data, b, gN, nrhs, ldb, &ldbd );
        dx = b200_vec_in( pastix_data, x, gN, nrhs, ldx, &ldxd );
        rc = b200_refine( e->solver, nrhs, db, ldbd, dx, ldxd, (int)method,
                          pastix_data->dparm[DPARM_EPSILON_REFINEMENT], pastix_data->iparm[IPARM_ITERMAX],
                          pastix_data->iparm[IPARM_GMRES_IM], &niter, berr );
        b200_vec_out( pastix_data, db, (void *)b, gN, nrhs, ldb, 0 );
        b200_vec_out( pastix_data, dx, x, gN, nrhs, ldx, rc == PASTIX_SUCCESS );
    }
    for ( j = 0; j < nrhs; j++ ) {
        emax = berr[j] > emax ? berr[j] : emax;
    }
    free( berr );
    pastix_data->dparm[DPARM_REFINE_TIME] = b200_wtime() - t0;
    if ( rc != PASTIX_SUCCESS ) {
        return rc;
    }
    pastix_data->iparm[IPARM_NBITER]        = niter;
    pastix_data->dparm[DPARM_RELATIVE_ERROR] = emax;
    pastix_data->steps |= STEP_REFINE;
    (void)n;
    return PASTIX_SUCCESS;
}

void
pastix_b200_finalize( pastix_data_t *pastix_data )
{
    b200_entry_t **pe, *e = NULL;
    pthread_mutex_lock( &b200_lock );
    for ( pe = &b200_entries; *pe != NULL; pe = &(*pe)->next ) {
        if ( (*pe)->pastix_data == pastix_data ) {
            e   = *pe;
            *pe = e->next;
            break;
        }
    }
    pthread_mutex_unlock( &b200_lock );
    if ( e != NULL ) {
        b200_solver_destroy( e->solver );
        free( e );
    }
}
