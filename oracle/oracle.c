/*
 * oracle.c -- TEST INFRASTRUCTURE.  A plain-C restatement of PaStiX's
 * full-rank supernodal numerical factorization and triangular solves, used only
 * as the checker of the GPU library (tests, the smoke check and the benchmark's
 * CPU-baseline leg).  It is never part of the product path.
 *
 * It works on the flattened SolverMatrix (blend/solver.h:83-213) in PaStiX's 2D
 * coefficient layout: every block of a cblk is a column-major tile with
 * ld = its row count, at offset coefind inside the cblk's array
 * (blend/solver_matrix_gen_utils.h:137-165); cblk arrays are concatenated in
 * cblk order.  For LU the U factor is stored transposed in a second array with
 * the same layout (kernels/cpucblk_zinit.c:130-134).
 *
 * Arithmetic follows the reference kernels step by step (same blocking of 64
 * in the diagonal factorizations, same static-pivot rule, same update
 * ordering), restated with plain loops instead of BLAS calls.  Compiled for
 * double (or_d_*) and float (or_s_*), and for x87 long double (or_q_*, 64-bit
 * mantissa), whose factor stands in for the exact one when the tests rate how far
 * two FP64 factorizations of an ill-conditioned matrix sit from it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL double
#define FN(x) or_d_##x
#define SQRT(x) sqrt(x)
#elif defined(ORACLE_LONG)
#define FN(x) or_q_##x
#define SQRT(x) sqrtl(x)
#else
#define FN(x) or_s_##x
#define SQRT(x) sqrt((double)(x))
#endif

#define MAXSIZEOFBLOCKS 64 /* kernels/core_zpotrfsp.c:25 */

typedef struct {
    int64_t cblknbr, bloknbr;
    const int64_t *fcolnum, *lcolnum, *fblok, *stride, *lcolidx, *brownum;
    const int64_t *frownum, *lrownum, *lcblknm, *fcblknm, *coefind, *browtab;
    const int64_t *cblkoff; /* offset of each cblk's array in the concatenated coeftab */
} or_struct_t;

static inline int64_t ncols_of( const or_struct_t *s, int64_t k ) { return s->lcolnum[k] - s->fcolnum[k] + 1; }
static inline int64_t rows_of( const or_struct_t *s, int64_t b ) { return s->lrownum[b] - s->frownum[b] + 1; }

/* ---------------------------------------------------------------- dense helpers */

/* C[m x n] += alpha * A[m x k] * op(B); op(B)=B^T with B[n x k] (ldb) */
static void
gemm_nt( int64_t m, int64_t n, int64_t k, REAL alpha, const REAL *A, int64_t lda,
         const REAL *B, int64_t ldb, REAL *C, int64_t ldc )
{
    for ( int64_t j = 0; j < n; j++ ) {
        for ( int64_t l = 0; l < k; l++ ) {
            REAL t = alpha * B[j + l * ldb];
            if ( t == 0 ) continue;
            const REAL *a = A + l * lda;
            REAL *c = C + j * ldc;
            for ( int64_t i = 0; i < m; i++ ) c[i] += t * a[i];
        }
    }
}

/* C[m x n] += alpha * A[m x k] * B[k x n] */
static void
gemm_nn( int64_t m, int64_t n, int64_t k, REAL alpha, const REAL *A, int64_t lda,
         const REAL *B, int64_t ldb, REAL *C, int64_t ldc )
{
    for ( int64_t j = 0; j < n; j++ ) {
        for ( int64_t l = 0; l < k; l++ ) {
            REAL t = alpha * B[l + j * ldb];
            if ( t == 0 ) continue;
            const REAL *a = A + l * lda;
            REAL *c = C + j * ldc;
            for ( int64_t i = 0; i < m; i++ ) c[i] += t * a[i];
        }
    }
}

/* X * op(T) = B on the right, B[m x n] overwritten.  T n x n (ldt).
 * lower_trans=1: op(T) = L^T with L lower  (Right, Lower, Trans)
 * lower_trans=0: op(T) = U   with U upper  (Right, Upper, NoTrans)  -- same access pattern
 * unit: unit diagonal. */
static void
trsm_right( int64_t m, int64_t n, const REAL *T, int64_t ldt, int lower_trans, int unit,
            REAL *B, int64_t ldb )
{
    /* column j of X: X[:,j] = (B[:,j] - sum_{l<j} X[:,l] * opT[l,j]) / opT[j,j]
     * opT[l,j] = L[j,l] (lower_trans) or U[l,j] (upper): both are T[l*?]. */
    for ( int64_t j = 0; j < n; j++ ) {
        REAL *bj = B + j * ldb;
        for ( int64_t l = 0; l < j; l++ ) {
            REAL t = lower_trans ? T[j + l * ldt] : T[l + j * ldt];
            if ( t == 0 ) continue;
            const REAL *bl = B + l * ldb;
            for ( int64_t i = 0; i < m; i++ ) bj[i] -= t * bl[i];
        }
        if ( !unit ) {
            REAL d = (REAL)1.0 / T[j + j * ldt];
            for ( int64_t i = 0; i < m; i++ ) bj[i] *= d;
        }
    }
}

/* op(T) * X = B on the left, B[n x nrhs].  T n x n (ldt).
 * trans=0: T lower, forward substitution.  trans=1: T^T with T lower (backward). */
static void
trsm_left_lower( int64_t n, int64_t nrhs, const REAL *T, int64_t ldt, int trans, int unit,
                 REAL *B, int64_t ldb )
{
    for ( int64_t r = 0; r < nrhs; r++ ) {
        REAL *b = B + r * ldb;
        if ( !trans ) {
            for ( int64_t j = 0; j < n; j++ ) {
                if ( !unit ) b[j] /= T[j + j * ldt];
                REAL x = b[j];
                for ( int64_t i = j + 1; i < n; i++ ) b[i] -= T[i + j * ldt] * x;
            }
        }
        else {
            for ( int64_t j = n - 1; j >= 0; j-- ) {
                REAL acc = b[j];
                for ( int64_t i = j + 1; i < n; i++ ) acc -= T[i + j * ldt] * b[i];
                b[j] = unit ? acc : acc / T[j + j * ldt];
            }
        }
    }
}

/* ------------------------------------------------ diagonal-block factorizations */

/* core_zpotf2sp (kernels/core_zpotrfsp.c:66-100); returns -1 on negative pivot */
static int
potf2( int64_t n, REAL *A, int64_t lda, int64_t *nbpivots, double criterion )
{
    for ( int64_t k = 0; k < n; k++ ) {
        REAL *akk = A + k * (lda + 1);
        if ( fabs( (double)*akk ) < criterion ) {
            *akk = (REAL)criterion;
            (*nbpivots)++;
        }
        if ( *akk < 0 ) return -1;
        *akk = (REAL)SQRT( *akk );
        REAL alpha = (REAL)1.0 / *akk;
        for ( int64_t i = k + 1; i < n; i++ ) A[i + k * lda] *= alpha;
        /* zher lower: A[k+1:,k+1:] -= a a^T */
        for ( int64_t j = k + 1; j < n; j++ ) {
            REAL t = A[j + k * lda];
            for ( int64_t i = j; i < n; i++ ) A[i + j * lda] -= A[i + k * lda] * t;
        }
    }
    return 0;
}

/* core_zpotrfsp (kernels/core_zpotrfsp.c:144-189) */
static int
potrfsp( int64_t n, REAL *A, int64_t lda, int64_t *nbpivots, double criterion )
{
    int64_t blocknbr = (n + MAXSIZEOFBLOCKS - 1) / MAXSIZEOFBLOCKS;
    for ( int64_t k = 0; k < blocknbr; k++ ) {
        int64_t bs = n - k * MAXSIZEOFBLOCKS < MAXSIZEOFBLOCKS ? n - k * MAXSIZEOFBLOCKS : MAXSIZEOFBLOCKS;
        REAL *tmp = A + (k * MAXSIZEOFBLOCKS) * (lda + 1);
        if ( potf2( bs, tmp, lda, nbpivots, criterion ) ) return -1;
        if ( k * MAXSIZEOFBLOCKS + bs < n ) {
            REAL *tmp1 = tmp + bs, *tmp2 = tmp1 + bs * lda;
            int64_t ms = n - (k * MAXSIZEOFBLOCKS + bs);
            trsm_right( ms, bs, tmp, lda, 1, 0, tmp1, lda );
            /* herk lower: tmp2 -= tmp1 tmp1^T (lower triangle only) */
            for ( int64_t j = 0; j < ms; j++ )
                for ( int64_t l = 0; l < bs; l++ ) {
                    REAL t = tmp1[j + l * lda];
                    for ( int64_t i = j; i < ms; i++ ) tmp2[i + j * lda] -= tmp1[i + l * lda] * t;
                }
        }
    }
    return 0;
}

/* core_zgetf2sp (kernels/core_zgetrfsp.c:64-110) */
static void
getf2( int64_t m, int64_t n, REAL *A, int64_t lda, int64_t *nbpivots, double criterion )
{
    int64_t mn = m < n ? m : n;
    for ( int64_t k = 0; k < mn; k++ ) {
        REAL *akk = A + k * (lda + 1);
        if ( fabs( (double)*akk ) < criterion ) {
            *akk = (*akk < 0) ? (REAL)(-criterion) : (REAL)criterion;
            (*nbpivots)++;
        }
        REAL alpha = (REAL)1.0 / *akk;
        for ( int64_t i = k + 1; i < m; i++ ) A[i + k * lda] *= alpha;
        if ( k + 1 < mn ) {
            for ( int64_t j = k + 1; j < n; j++ ) {
                REAL t = A[k + j * lda];
                for ( int64_t i = k + 1; i < m; i++ ) A[i + j * lda] -= A[i + k * lda] * t;
            }
        }
    }
}

/* core_zgetrfsp (kernels/core_zgetrfsp.c:137-183) */
static void
getrfsp( int64_t n, REAL *A, int64_t lda, int64_t *nbpivots, double criterion )
{
    int64_t blocknbr = (n + MAXSIZEOFBLOCKS - 1) / MAXSIZEOFBLOCKS;
    REAL *Akk = A;
    for ( int64_t k = 0; k < blocknbr; k++ ) {
        int64_t tempm = n - k * MAXSIZEOFBLOCKS;
        int64_t bs = tempm < MAXSIZEOFBLOCKS ? tempm : MAXSIZEOFBLOCKS;
        REAL *Lik = Akk + bs, *Ukj = Akk + bs * lda, *Aij = Ukj + bs;
        getf2( tempm, bs, Akk, lda, nbpivots, criterion );
        int64_t ms = tempm - bs;
        if ( ms > 0 ) {
            /* trsm Left Lower NoTrans Unit: Ukj = L^-1 Ukj */
            for ( int64_t j = 0; j < ms; j++ ) {
                REAL *u = Ukj + j * lda;
                for ( int64_t l = 0; l < bs; l++ ) {
                    REAL x = u[l];
                    for ( int64_t i = l + 1; i < bs; i++ ) u[i] -= Akk[i + l * lda] * x;
                }
            }
            gemm_nn( ms, ms, bs, (REAL)-1.0, Lik, lda, Ukj, lda, Aij, lda );
        }
        Akk += bs * (lda + 1);
    }
}

/* core_zsytf2sp (kernels/core_zsytrfsp.c:63-103) */
static void
sytf2( int64_t n, REAL *A, int64_t lda, int64_t *nbpivots, double criterion )
{
    for ( int64_t k = 0; k < n; k++ ) {
        int64_t m = n - k - 1;
        REAL *akk = A + k * (lda + 1);
        if ( fabs( (double)*akk ) < criterion ) {
            *akk = (*akk < 0) ? (REAL)(-criterion) : (REAL)criterion;
            (*nbpivots)++;
        }
        REAL alpha = (REAL)1.0 / *akk;
        REAL *amk = akk + 1, *akm = akk + lda;
        for ( int64_t i = 0; i < m; i++ ) akm[i * lda] = amk[i];
        for ( int64_t i = 0; i < m; i++ ) amk[i] *= alpha;
        REAL beta = -*akk;
        REAL *a2 = akk + lda + 1;
        /* syrk lower: a2 += beta * amk amk^T */
        for ( int64_t j = 0; j < m; j++ ) {
            REAL t = beta * amk[j];
            for ( int64_t i = j; i < m; i++ ) a2[i + j * lda] += amk[i] * t;
        }
    }
}

/* core_zsytrfsp (kernels/core_zsytrfsp.c:144-215) */
static void
sytrfsp( int64_t n, REAL *A, int64_t lda, int64_t *nbpivots, double criterion )
{
    int64_t blocknbr = (n + MAXSIZEOFBLOCKS - 1) / MAXSIZEOFBLOCKS;
    for ( int64_t k = 0; k < blocknbr; k++ ) {
        int64_t bs = n - k * MAXSIZEOFBLOCKS < MAXSIZEOFBLOCKS ? n - k * MAXSIZEOFBLOCKS : MAXSIZEOFBLOCKS;
        REAL *Akk = A + (k * MAXSIZEOFBLOCKS) * (lda + 1);
        REAL *Amk = Akk + bs, *Akm = Akk + bs * lda, *Amm = Amk + bs * lda;
        sytf2( bs, Akk, lda, nbpivots, criterion );
        if ( k * MAXSIZEOFBLOCKS + bs < n ) {
            int64_t ms = n - (k * MAXSIZEOFBLOCKS + bs);
            /* trsm Right Lower Trans Unit */
            trsm_right( ms, bs, Akk, lda, 1, 1, Amk, lda );
            for ( int64_t col = 0; col < bs; col++ ) {
                for ( int64_t i = 0; i < ms; i++ ) Akm[col + i * lda] = Amk[i + col * lda];
                REAL alpha = (REAL)1.0 / Akk[col * (lda + 1)];
                for ( int64_t i = 0; i < ms; i++ ) Amk[i + col * lda] *= alpha;
            }
            gemm_nn( ms, ms, bs, (REAL)-1.0, Amk, lda, Akm, lda, Amm, lda );
        }
    }
}

/* ----------------------------------------------------------- cblk-level steps */

/* cpucblk_zfillin_fr (kernels/cpucblk_zinit.c:229-309) on zeroed L/U */
void
FN(fillin)( const or_struct_t *s, const int64_t *colptr, const int64_t *rowtab,
            const REAL *Lvalues, const REAL *Uvalues, REAL *L, REAL *U )
{
    for ( int64_t k = 0; k < s->cblknbr; k++ ) {
        int64_t nc = ncols_of( s, k );
        for ( int64_t jc = 0; jc < nc; jc++ ) {
            int64_t col = s->fcolnum[k] + jc;
            int64_t b = s->fblok[k], lb = s->fblok[k + 1];
            for ( int64_t e = colptr[col]; e < colptr[col + 1]; e++ ) {
                int64_t r = rowtab[e];
                if ( r < col ) continue;
                while ( b < lb && (s->lrownum[b] < r || s->frownum[b] > r) ) b++;
                if ( b >= lb ) continue;
                int64_t idx = s->cblkoff[k] + s->coefind[b] + (r - s->frownum[b]) + jc * rows_of( s, b );
                L[idx] = Lvalues[e];
                if ( U && r > col ) U[idx] = Uvalues[e];
            }
        }
    }
}

/* core_ztrsmsp_2d (kernels/core_ztrsmsp.c:147-181): every off-diagonal block of
 * cblk k solved against the factored diagonal block. */
static void
panel_trsm( const or_struct_t *s, int64_t k, REAL *C, int lower_trans, int unit )
{
    int64_t nc = ncols_of( s, k );
    REAL *base = C + s->cblkoff[k];
    const REAL *D = base; /* diagonal block, ld = ncols */
    for ( int64_t b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++ ) {
        trsm_right( rows_of( s, b ), nc, D, nc, lower_trans, unit, base + s->coefind[b], rows_of( s, b ) );
    }
}

/* core_zgemmsp_2d2d (kernels/core_zgemmsp.c:396-465):
 * C[fcblk] -= A[iterblok] * B[blok]^T for iterblok >= blok (+shift). */
static void
gemm_2d2d( const or_struct_t *s, int64_t k, int64_t blok, int shift, const REAL *A, const REAL *B,
           REAL *C )
{
    int64_t f = s->fcblknm[blok];
    int64_t K = ncols_of( s, k ), N = rows_of( s, blok );
    const REAL *bB = B + s->cblkoff[k] + s->coefind[blok];
    int64_t fb = s->fblok[f];
    for ( int64_t it = blok + shift; it < s->fblok[k + 1]; it++ ) {
        while ( !(s->frownum[it] >= s->frownum[fb] && s->lrownum[it] <= s->lrownum[fb]) ) fb++;
        int64_t ldc = rows_of( s, fb ), M = rows_of( s, it );
        REAL *cC = C + s->cblkoff[f] + s->coefind[fb] + (s->frownum[it] - s->frownum[fb])
                   + (s->frownum[blok] - s->fcolnum[f]) * ldc;
        gemm_nt( M, N, K, (REAL)-1.0, A + s->cblkoff[k] + s->coefind[it], M, bB, N, cC, ldc );
    }
}

/* Sequential factorization, cblk by cblk in index order
 * (sopalin/sequential_zpotrf.c:34-65, sequential_zgetrf.c, sequential_zsytrf.c).
 * facto: 0 POTRF, 1 SYTRF, 2 GETRF.  DLt: workspace of coefnbr entries (SYTRF).
 * Returns 0, or -1 on a negative pivot in POTRF. */
int
FN(numfact)( const or_struct_t *s, int facto, REAL *L, REAL *U, REAL *DLt, double criterion,
             int64_t *nbpivots )
{
    *nbpivots = 0;
    for ( int64_t k = 0; k < s->cblknbr; k++ ) {
        int64_t nc = ncols_of( s, k );
        REAL *Lk = L + s->cblkoff[k];
        if ( facto == 0 ) {
            /* cpucblk_zpotrfsp1d (kernels/core_zpotrfsp.c:326-359) */
            if ( potrfsp( nc, Lk, nc, nbpivots, criterion ) ) return -1;
            panel_trsm( s, k, L, 1, 0 );
            for ( int64_t b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++ ) gemm_2d2d( s, k, b, 0, L, L, L );
        }
        else if ( facto == 2 ) {
            /* cpucblk_zgetrfsp1d (kernels/core_zgetrfsp.c:340-382) */
            REAL *Uk = U + s->cblkoff[k];
            for ( int64_t j = 0; j < nc; j++ )      /* geadd(Trans): L += U^T */
                for ( int64_t i = 0; i < nc; i++ ) Lk[i + j * nc] += Uk[j + i * nc];
            getrfsp( nc, Lk, nc, nbpivots, criterion );
            for ( int64_t j = 0; j < nc; j++ )      /* getmo: U = L^T */
                for ( int64_t i = 0; i < nc; i++ ) Uk[j + i * nc] = Lk[i + j * nc];
            panel_trsm( s, k, L, 0, 0 );            /* Right Upper NoTrans NonUnit */
            panel_trsm( s, k, U, 0, 1 );            /* Right Upper NoTrans Unit    */
            for ( int64_t b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++ ) {
                gemm_2d2d( s, k, b, 0, L, U, L );
                if ( b + 1 < s->fblok[k + 1] ) gemm_2d2d( s, k, b, 1, U, L, U );
            }
        }
        else {
            /* cpucblk_zsytrfsp1d (kernels/core_zsytrfsp.c:478-523) */
            sytrfsp( nc, Lk, nc, nbpivots, criterion );
            panel_trsm( s, k, L, 0, 0 );            /* Right Upper NoTrans NonUnit on D L^T */
            /* cpucblk_zscalo (kernels/core_zscalo.c:161): DLt = L * D per block */
            for ( int64_t b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++ ) {
                int64_t m = rows_of( s, b );
                const REAL *lb = L + s->cblkoff[k] + s->coefind[b];
                REAL *db = DLt + s->cblkoff[k] + s->coefind[b];
                for ( int64_t j = 0; j < nc; j++ ) {
                    REAL d = Lk[j * (nc + 1)];
                    for ( int64_t i = 0; i < m; i++ ) db[i + j * m] = lb[i + j * m] * d;
                }
            }
            for ( int64_t b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++ ) gemm_2d2d( s, k, b, 0, L, DLt, L );
        }
    }
    return 0;
}

/* solve_blok_zgemm forward (kernels/solve_ztrsmsp.c:275): b[f] -= A * b[k] */
static void
blok_gemm_fwd( const or_struct_t *s, int64_t blok, const REAL *A, int64_t nrhs, REAL *b, int64_t ldb )
{
    int64_t k = s->lcblknm[blok], f = s->fcblknm[blok];
    int64_t m = rows_of( s, blok ), n = ncols_of( s, k );
    const REAL *a = A + s->cblkoff[k] + s->coefind[blok];
    REAL *c = b + s->lcolidx[f] + (s->frownum[blok] - s->fcolnum[f]);
    const REAL *x = b + s->lcolidx[k];
    for ( int64_t r = 0; r < nrhs; r++ )
        for ( int64_t j = 0; j < n; j++ ) {
            REAL t = x[j + r * ldb];
            for ( int64_t i = 0; i < m; i++ ) c[i + r * ldb] -= a[i + j * m] * t;
        }
}

/* backward (trans): b[k] -= A^T * b[f] */
static void
blok_gemm_bwd( const or_struct_t *s, int64_t blok, const REAL *A, int64_t nrhs, REAL *b, int64_t ldb )
{
    int64_t k = s->lcblknm[blok], f = s->fcblknm[blok];
    int64_t m = rows_of( s, blok ), n = ncols_of( s, k );
    const REAL *a = A + s->cblkoff[k] + s->coefind[blok];
    const REAL *y = b + s->lcolidx[f] + (s->frownum[blok] - s->fcolnum[f]);
    REAL *c = b + s->lcolidx[k];
    for ( int64_t r = 0; r < nrhs; r++ )
        for ( int64_t j = 0; j < n; j++ ) {
            REAL acc = 0;
            for ( int64_t i = 0; i < m; i++ ) acc += a[i + j * m] * y[i + r * ldb];
            c[j + r * ldb] -= acc;
        }
}

/* pastix_subtask_solve in the permuted basis (sopalin/pastix_task_solve.c:408-516)
 * with the sequential sweeps of sopalin/sequential_ztrsm.c:34-120 and
 * solve_cblk_ztrsmsp_forward/backward (kernels/solve_ztrsmsp.c:332-557). */
void
FN(solve)( const or_struct_t *s, int facto, const REAL *L, const REAL *U, int64_t nrhs, REAL *b,
           int64_t ldb )
{
    int unit = (facto != 0);
    /* forward: L y = b */
    for ( int64_t k = 0; k < s->cblknbr; k++ ) {
        int64_t nc = ncols_of( s, k );
        trsm_left_lower( nc, nrhs, L + s->cblkoff[k], nc, 0, unit, b + s->lcolidx[k], ldb );
        for ( int64_t blk = s->fblok[k] + 1; blk < s->fblok[k + 1]; blk++ ) blok_gemm_fwd( s, blk, L, nrhs, b, ldb );
    }
    if ( facto == 1 ) {
        /* solve_cblk_zdiag (kernels/solve_ztrsmsp.c:584-633): b /= D */
        for ( int64_t k = 0; k < s->cblknbr; k++ ) {
            int64_t nc = ncols_of( s, k );
            const REAL *Lk = L + s->cblkoff[k];
            for ( int64_t r = 0; r < nrhs; r++ )
                for ( int64_t j = 0; j < nc; j++ ) b[s->lcolidx[k] + j + r * ldb] /= Lk[j * (nc + 1)];
        }
    }
    /* backward: L^T x = y (POTRF, SYTRF with unit L), U x = y (GETRF, U^T stored) */
    const REAL *T = (facto == 2) ? U : L;
    int bunit = (facto == 1);
    /* The reference's backward sweep scatters from cblk k into the cblks whose
     * blocks face k (browtab).  Gathering per cblk over its own off-diagonal
     * blocks is the same sum: x_k = T_kk^-T (b_k - sum_i A_i^T x[f(i)]). */
    for ( int64_t k = s->cblknbr - 1; k >= 0; k-- ) {
        int64_t nc = ncols_of( s, k );
        for ( int64_t blk = s->fblok[k + 1] - 1; blk > s->fblok[k]; blk-- ) blok_gemm_bwd( s, blk, T, nrhs, b, ldb );
        /* diagonal: T_kk^T x = b with T_kk lower (L, or U^T for LU) */
        trsm_left_lower( nc, nrhs, T + s->cblkoff[k], nc, 1, bunit, b + s->lcolidx[k], ldb );
    }
}
