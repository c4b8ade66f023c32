/*
 * pastix_b200.h -- C ABI of the B200 numerical factorization and solve backend
 * for PaStiX.
 *
 * PaStiX keeps its host analysis (ordering, symbolic factorization, blend); its
 * numerical factorization, triangular solves and iterative refinement run on one
 * B200 through these entry points.  Only plain C types cross this boundary: the
 * SolverMatrix integer tables are passed as int64 arrays, values and vectors as
 * host (or, for the *_device variants, device) pointers.
 *
 * Return values are PaStiX error codes (include/pastix/api.h:321-334):
 * 0 = PASTIX_SUCCESS, 2 = PASTIX_ERR_ALLOC, 3 = PASTIX_ERR_NOTIMPLEMENTED,
 * 4 = PASTIX_ERR_OUTOFMEMORY, 6 = PASTIX_ERR_INTERNAL, 7 = PASTIX_ERR_BADPARAMETER.
 *
 * Threading: the factorization, bcsc and structure calls of one solver instance are
 * not re-entrant (as a pastix_data_t) and must not overlap with its solves.  The
 * solve and refinement calls on DIFFERENT CUDA streams may run concurrently from
 * different host threads on the same factor: every stream gets its own workspaces,
 * tickets and status word on its first call (a device allocation then), so their
 * work overlaps on the GPU.  Calls on the same stream are serialized by the caller.
 * The host-pointer calls (b200_solve, b200_refine, b200_spmv, b200_trsm,
 * b200_applyorder) all use the solver's own stream.  Separate instances may be used
 * from separate host threads.
 */
#ifndef PASTIX_B200_H
#define PASTIX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Factorization kinds, numbered as PaStiX's pastix_factotype_t
 * (include/pastix/api.h:272-285). */
enum { B200_FACTO_POTRF = 0, B200_FACTO_SYTRF = 1, B200_FACTO_GETRF = 2 };

/* Arithmetic of the factor.
 *  FP64   : factor in double, FP64 updates (the drop-in path).
 *  FP32   : factor in float, FP32 CUDA-core updates.
 *  TF32   : factor in float, wide updates on tcgen05 tensor cores in TF32
 *           with FP32 accumulation.
 *  TF32X3 : as TF32 with split (big + small) operands, three TF32 products per
 *           update, for close-to-FP32 accuracy.
 *  BF16X3 : factor in float, wide updates on tcgen05 tensor cores with split BF16
 *           operands (x = hi + lo, both BF16; three BF16 products accumulated in
 *           FP32, about 2^-17 relative per product): half the operand bytes and
 *           twice the MMA rate of TF32, a less accurate factor for the refinement
 *           to correct.
 * The solve and refinement vectors are always double. */
enum { B200_PREC_FP64 = 0, B200_PREC_FP32 = 1, B200_PREC_TF32 = 2, B200_PREC_TF32X3 = 3, B200_PREC_BF16X3 = 4 };

/* Refinement methods, numbered as PaStiX's pastix_refine_t
 * (include/pastix/api.h:241-246, IPARM_REFINEMENT): GMRES, CG, simple refinement,
 * BiCGSTAB. */
enum { B200_REFINE_GMRES = 0, B200_REFINE_CG = 1, B200_REFINE_SR = 2, B200_REFINE_BICGSTAB = 3 };

/* The SolverMatrix integer structure (blend/solver.h:83-213), 0-based.
 * cblk arrays hold cblknbr+1 entries (the last is PaStiX's sentinel cblk, whose
 * fblok is bloknbr and brownum is brownbr); blok arrays hold bloknbr+1 entries
 * (SolverBlok fields); cblk_fblok[k] = cblktab[k].fblokptr - bloktab.
 * peritab is ordemesh->peritab (new -> original index). */
typedef struct b200_symbol_s {
    int64_t n, cblknbr, bloknbr, brownbr;
    const int64_t *cblk_fcolnum, *cblk_lcolnum, *cblk_fblok, *cblk_stride;
    const int64_t *cblk_lcolidx, *cblk_brownum;
    const int64_t *blok_frownum, *blok_lrownum, *blok_lcblknm, *blok_fcblknm;
    const int64_t *browtab;
    const int64_t *peritab;
} b200_symbol_t;

typedef struct b200_solver_s b200_solver_t;

/* Kernel choices of one solver instance, as an autotuner picks them (no
 * counterpart in PaStiX, whose GEMM kernels take fixed blockings,
 * kernels/gpus/kepler/gemm_config/dgemm_param_nt.h:35,64, with per-kernel cost models
 * in common/models.c).  update[w][h] selects the kernel of the GEMM-scatter updates
 * of an FP32 factor (precisions FP32, TF32, TF32X3) whose width K (the source cblk's
 * columns) falls in width class w and whose height M (rows of the source panel from
 * the facing block down) in height class h:
 *   width classes  K: [1,16) [16,32) [32,48) [48,64) [64,128) [128,inf)
 *   height classes M: [1,64) [64,128) [128,256) [256,512) [512,inf)
 * B200_UPD_DEFAULT keeps the built-in rule (tensor cores for K >= 32 and M >= 64,
 * 128-column tiles for updates wider than 64 columns), B200_UPD_SIMT the CUDA-core
 * kernels, B200_UPD_TC the tensor cores with the built-in tile width, B200_UPD_TC64
 * the tensor cores with 64-column tiles.  Updates the tensor-core kernel does not
 * handle (LDL^T's D-scaled operands, K not a multiple of 32 past the first K chunk)
 * stay on the CUDA cores whatever the table says.  flow_min: the solve sweeps take
 * one dataflow launch for the levels from the first one with fewer than flow_min
 * cblks (0: the default, 8).  panel_tiles: 1 forces the 64 x 64 tile-item form of
 * the wide-cblk panel launches. */
#define B200_TUNE_WCLASSES 6
#define B200_TUNE_HCLASSES 5
enum { B200_UPD_DEFAULT = 0, B200_UPD_SIMT = 1, B200_UPD_TC = 2, B200_UPD_TC64 = 3 };
typedef struct b200_tuning_s {
    int32_t update[B200_TUNE_WCLASSES][B200_TUNE_HCLASSES];
    int32_t flow_min;
    int32_t panel_tiles;
} b200_tuning_t;

/* Upload the structure and build the device-side schedules.  Replaces the
 * structure walk PaStiX does in coeftabInit / solverBackupInit
 * (sopalin/coeftab.c:70-140, blend/solver_backup.c:60-100) and selects the
 * kernels that the per-(facto, precision) table sopalinFacto
 * (sopalin/pastix_task_sopalin.c:41-48) would have picked.  stream may be NULL
 * (the library then creates its own CUDA stream). */
int b200_solver_create( const b200_symbol_t *symbol, int facto, int precision, void *stream,
                        b200_solver_t **solver );
int b200_solver_destroy( b200_solver_t *solver );

/* The same with a Schur complement (pastixSetSchurUnknownList, IPARM_SCHUR_SOLV_MODE =
 * PastixSolvModeInterface): the cblks from cblkschur on (PaStiX's
 * solvmtx->cblkschur, the CBLK_IN_SCHUR cblks) receive the updates of the others but
 * are not factored (sopalin/sequential_zpotrf.c:51); b200_get_schur returns that
 * block, b200_trsm solves around it.  b200_solve, b200_solve_device* and
 * b200_refine* refuse such an instance (PASTIX_ERR_BADPARAMETER). */
int b200_solver_create_schur( const b200_symbol_t *symbol, int facto, int precision, void *stream,
                              int64_t cblkschur, b200_solver_t **solver );

/* b200_solver_create_schur with a tuning table (NULL: the defaults); cblkschur =
 * symbol->cblknbr for no Schur complement. */
int b200_solver_create_tuned( const b200_symbol_t *symbol, int facto, int precision, void *stream,
                              int64_t cblkschur, const b200_tuning_t *tuning, b200_solver_t **solver );

/* Load the permuted blocked CSC (bcsc/bcsc.h:28-53; pastix_subtask_spm2bcsc,
 * sopalin/pastix_task_sopalin.c:82).  colptr has n+1 entries in the permuted
 * column numbering; Lvalues holds A (both triangles for a symmetric matrix),
 * Uvalues holds A^T (LU only, else NULL); anorm is ||A||_F (DPARM_A_NORM).
 * Host pointers.  The first call fixes the pattern; later calls with the same
 * colptr/rowtab only replace the values (same-pattern refactorization). */
int b200_bcsc_load( b200_solver_t *solver, int64_t nnz, const int64_t *colptr,
                    const int64_t *rowtab, const double *Lvalues, const double *Uvalues,
                    double anorm );

/* New values on the pattern of the last b200_bcsc_load (same colptr/rowtab, in the
 * same order), without re-checking or re-deriving the structure: the
 * refactorization path of PaStiX, where pastix_subtask_bcsc2ctab refills the
 * coeftab from the bcsc of an spm whose values changed
 * (sopalin/pastix_task_sopalin.c:196).  Host arrays of nnz doubles; pinned host
 * memory makes the copy a DMA at full PCIe / C2C speed.  PASTIX_ERR_BADPARAMETER
 * before a first b200_bcsc_load. */
int b200_bcsc_values( b200_solver_t *solver, const double *Lvalues, const double *Uvalues, double anorm );

/* The bcsc construction of a same-pattern refactorization on the device
 * (bcsc_zinit_centralized, bcsc/bcsc_zinit.c:52-541, after pastix_subtask_spm2bcsc,
 * sopalin/pastix_task_sopalin.c:82): b200_spm_map records, for every entry e of the
 * bcsc of the last b200_bcsc_load, the index lmap[e] (umap[e] for the A^T values of
 * LU) of the input matrix value it holds, in the matrix's own CSC order (nnz_spm
 * values; for symmetric matrices the stored triangle, both bcsc entries of an
 * off-diagonal value mapping to it).  b200_spm_values / b200_spm_values_device then
 * take new values in that order (host / device memory), permute and expand them on
 * the GPU, and set ||A||_F for the threshold (computed on the device when anorm < 0,
 * as spmNorm(SpmFrobeniusNorm)).  A new pattern in b200_bcsc_load drops the map. */
/* pastixGetSchur (sopalin/schur.c, coeftab_zgetschur, sopalin/coeftab_z.c:413-437):
 * the Schur complement after b200_numfact, nschur x nschur column-major in S
 * (lds >= nschur = n - first column of the Schur part), in the permuted order of
 * the Schur unknowns: the lower triangle for Cholesky and LDL^T, the full block for
 * LU. */
int b200_get_schur( b200_solver_t *solver, double *S, int64_t lds );

/* pastix_subtask_applyorder (sopalin/pastix_task_solve.c:118-170): b <- P b (dir 0,
 * to the permuted basis) or P^T b (dir 1, back). */
int b200_applyorder( b200_solver_t *solver, int dir, int64_t nrhs, double *b, int64_t ldb );

/* pastix_subtask_trsm / pastix_subtask_diag (sopalin/pastix_task_solve.c:194-407)
 * on a permuted b (host memory): step 0 the forward sweep (L y = b, unit L for LU and
 * LDL^T), 1 the backward sweep (L^T, U, or L^T for LDL^T with unit diagonal),
 * 2 b <- D^{-1} b (LDL^T; no-op otherwise).  With a Schur complement the sweeps cover
 * the unknowns before it: the forward sweep leaves b_S - A_S1 y_1 in the Schur rows,
 * the backward sweep reads the Schur rows as the caller's solution. */
int b200_trsm( b200_solver_t *solver, int step, int64_t nrhs, double *b, int64_t ldb );

/* pastixGetDiag (sopalin/diag.c:55, coeftab_zgetdiag, sopalin/coeftab_z.c:462): the
 * diagonal of the factor's diagonal blocks in the permuted numbering (Cholesky: the
 * diagonal of L; LDL^T: D; LU: the diagonal of U), n values D[i * incD] as double.
 * Requires a completed b200_numfact. */
int b200_get_diag( b200_solver_t *solver, double *D, int64_t incD );

/* Batch of independent systems.  The reference factors each system through its own
 * pastix_task_numfact / pastix_task_solve / pastix_task_refine
 * (sopalin/pastix_task_sopalin.c:563, sopalin/pastix_task_solve.c:550,
 * refinement/pastix_task_refine.c:226); here the systems' SolverMatrix structures
 * are concatenated into one elimination forest (cblks, blocks, columns and browtab
 * offset system by system) so that every level of all trees runs in the same
 * launches.  sys_cblk[0..nsys]: first cblk of each system (sys_cblk[0] = 0,
 * sys_cblk[nsys] = cblknbr); every block of a system's cblks must face a cblk of
 * the same system.  Call once, after b200_solver_create and before b200_numfact.
 * Then each system keeps its own static-pivoting threshold (the threshold rule with
 * its own ||A_i||_F, computed from its bcsc columns on the device; b200_stats
 * reports -1 as the threshold) and its own pivot count (b200_numfact returns their
 * sum), and b200_refine /
 * b200_refine_device run one refinement per (column, system), each with its own
 * stopping rule; their berr then holds per column the largest error of its systems. */
int b200_batch_set( b200_solver_t *solver, int64_t nsys, const int64_t *sys_cblk );
/* the nsys thresholds of the last b200_numfact of a batch */
int b200_batch_thresholds( b200_solver_t *solver, double *thr, int64_t nsys );
/* the pivots each system's last factorization replaced (its IPARM_STATIC_PIVOTING) */
int b200_batch_pivots( b200_solver_t *solver, int64_t *npiv, int64_t nsys );
/* the backward errors of the last refinement per problem, column-major
 * (problem r * nsys + system; count = nrhs * nsys, or nrhs outside a batch) */
int b200_batch_berr( b200_solver_t *solver, double *berr, int64_t count );

int b200_spm_map( b200_solver_t *solver, int64_t nnz_spm, const int64_t *lmap, const int64_t *umap );
int b200_spm_values( b200_solver_t *solver, const double *values, double anorm );
int b200_spm_values_device( b200_solver_t *solver, const double *d_values, double anorm, void *stream );

/* Numerical factorization: bcsc -> coeftab scatter (cpucblk_zfillin,
 * kernels/cpucblk_zinit.c:229) and the supernodal factorization
 * (sopalin/sequential_z{potrf,sytrf,getrf}.c).  epsilon_magn_ctrl has the
 * meaning of DPARM_EPSILON_MAGN_CTRL (sopalin/pastix_task_sopalin.c:401-425):
 * < 0: |value| is the threshold, 0: sqrt(eps)*||A||_F, > 0: value*||A||_F.
 * nbpivots (may be NULL) receives the static-pivot count (IPARM_STATIC_PIVOTING).
 * Returns 6 (PASTIX_ERR_INTERNAL) on a negative pivot in a Cholesky. */
int b200_numfact( b200_solver_t *solver, double epsilon_magn_ctrl, int64_t *nbpivots );

/* Per-kernel timing of one factorization, the counterpart of PaStiX's kernel
 * tracing and flop accounting (kernels/kernels_trace.h:206-300).  Runs
 * b200_numfact once through the CUDA graph, then once more kernel by kernel
 * with CUDA events.  ms[4] receives the device time of each kernel class
 * (0: arena clear + bcsc scatter, 1: diagonal blocks, 2: panel TRSM,
 * 3: GEMM-scatter updates); flops[4] (may be NULL) their algorithmic flops
 * (diagonal n^3/3, TRSM m n^2, updates 2 M N K; doubled for LU). */
int b200_numfact_trace( b200_solver_t *solver, double epsilon_magn_ctrl, double *ms, double *flops );

/* pastix_task_solve (sopalin/pastix_task_solve.c:550): b (n x nrhs, column
 * major, leading dimension ldb, original ordering, host memory) is overwritten
 * with x. */
int b200_solve( b200_solver_t *solver, int64_t nrhs, double *b, int64_t ldb );

/* Timing of the triangular sweeps of one solve of nrhs zero right-hand sides (in
 * the permuted basis, no permutation): ms[1] the forward sweep, ms[2] the
 * backward sweep (one dataflow launch each), ms[3] the D scaling of LDL^T
 * (ms[0] unused), with CUDA events around every launch; bytes[4] (may be NULL)
 * the algorithmic traffic of each sweep (factor entries read once, vectors read
 * and written once, in the factor's precision). */
int b200_solve_trace( b200_solver_t *solver, int64_t nrhs, double *ms, double *bytes );

/* Per-launch device times of the last b200_numfact_trace / b200_solve_trace:
 * ms[i] and cls[i] for the first min(cap, count) launches, grouped by kind in
 * launch order within a kind.  Kinds: 0-3 the classes of the trace, 4 panel
 * factorizations of the wide cblks (diagonal block, panel solve and the updates
 * inside the panel, one launch per level), 5 inverses of the diagonal blocks,
 * 6 GEMM-scatter updates on the tensor cores, 7 the row-major operand copies they
 * read, 8 the tree-bottom launch (every cblk of the bottom levels, at most 32
 * columns each: diagonal block, panel solve and updates, ordered by dependency
 * counters instead of level by level).  Returns the launch count (or a negative
 * error code).
 * Counterpart of PaStiX's kernel trace (kernels/kernels_trace.h). */
int64_t b200_trace_launches( b200_solver_t *solver, double *ms, int32_t *cls, int64_t cap );

/* Per-kind totals of the last b200_numfact_trace: ms[i] the device time and
 * flops[i] the algorithmic flops (useful products of the GEMM-scatter updates,
 * PaStiX's counting; panels: their diagonal and solve flops; 0 where not
 * counted; kind 8: its updates' useful products) of kind i < min(nkinds, 9), kinds as
 * in b200_trace_launches.  Returns the number of kinds filled.  Counterpart of
 * the per-kernel flop counters of kernels/kernels_trace.h. */
int b200_trace_kinds( b200_solver_t *solver, double *ms, double *flops, int nkinds );

/* Same on device memory, asynchronously on the solver's stream (or on stream if
 * not NULL).  Check b200_solve_status once the stream has been synchronized. */
int b200_solve_device( b200_solver_t *solver, int64_t nrhs, double *d_b, int64_t ldb, void *stream );

/* Status of the last solve or refinement of this instance on stream (NULL: the
 * solver's own stream), for the asynchronous device entry points
 * (b200_solve_device, b200_solve_device_noalloc, b200_refine_device): call it after
 * synchronizing that stream.  PASTIX_ERR_INTERNAL if a sweep gave up waiting for its
 * inputs (the result is not to be used), else PASTIX_SUCCESS.  Each solve or
 * refinement call clears the status of its stream when it starts; the host-pointer
 * calls check it themselves.  b200_solve_device_noalloc reports on the solver's own
 * stream's status, whatever stream it ran on.  Counterpart of the return code of
 * pastix_task_solve (sopalin/pastix_task_solve.c:550). */
int b200_solve_status( b200_solver_t *solver, void *stream );

/* Size of the fixed scratch of b200_solve_device_noalloc: 4,194,304 doubles
 * (32 MiB); a call needs 2 * n * nrhs of them. */
#define B200_NOALLOC_SCRATCH_DOUBLES 4194304

/* Solve on device memory without allocating anything.  It has no counterpart in
 * PaStiX: it exists for callers that cannot call cudaMalloc when they solve --
 * a request loop whose device memory is all reserved by a pool, code that must
 * not trigger the implicit device synchronization of cudaMalloc/cudaFree, or a
 * process that must keep a fixed footprint.  Same result as b200_solve_device.
 * The permuted right-hand sides live in one fixed scratch array compiled into
 * this library (B200_NOALLOC_SCRATCH_DOUBLES doubles).  The array is reserved on a
 * GPU when the first solver instance is created on it (b200_solver_create looks
 * up its device address with cudaGetSymbolAddress, which loads it there) and is
 * held until the process exits; this call itself only reads the address stored
 * in the instance.  Calls with 2 * n * nrhs > B200_NOALLOC_SCRATCH_DOUBLES are
 * rejected with PASTIX_ERR_BADPARAMETER.  All calls share the array: calls that
 * overlap on the GPU (other streams, other solver instances, other host threads)
 * race and must be serialized by the caller; each call writes every entry it
 * reads first, so what a previous call left there does not matter.  stream may be
 * NULL (the solver's own stream); check b200_solve_status after synchronizing. */
int b200_solve_device_noalloc( b200_solver_t *solver, int64_t nrhs, double *d_b, int64_t ldb,
                               void *stream );

/* pastix_task_refine (refinement/pastix_task_refine.c:226): iterative
 * refinement in double of x (initial guess, overwritten) for A x = b, with the
 * factor as preconditioner.  method: B200_REFINE_*; eps: stopping tolerance on
 * ||b - A x||_2 / ||b||_2 per right-hand side (DPARM_EPSILON_REFINEMENT);
 * itermax: IPARM_ITERMAX; gmres_im: IPARM_GMRES_IM.  Host pointers.
 * niter (may be NULL) receives the largest iteration count over the
 * right-hand sides, berr (may be NULL, nrhs entries) the final backward errors. */
int b200_refine( b200_solver_t *solver, int64_t nrhs, const double *b, int64_t ldb, double *x,
                 int64_t ldx, int method, double eps, int64_t itermax, int64_t gmres_im,
                 int64_t *niter, double *berr );

/* pastix_task_solve / pastix_task_refine with single-precision vectors, as PaStiX
 * takes them for a float matrix (the call dispatches on the bcsc's flttype,
 * sopalin/pastix_task_solve.c:550, refinement/pastix_task_refine.c:226): host
 * arrays of float, widened to double on the GPU for the solve and the refinement,
 * narrowed back into b (solve) or x (refinement). */
int b200_solve_float( b200_solver_t *solver, int64_t nrhs, float *b, int64_t ldb );
int b200_refine_float( b200_solver_t *solver, int64_t nrhs, const float *b, int64_t ldb, float *x,
                       int64_t ldx, int method, double eps, int64_t itermax, int64_t gmres_im,
                       int64_t *niter, double *berr );

/* Same on device memory (b and x on the device). */
int b200_refine_device( b200_solver_t *solver, int64_t nrhs, const double *d_b, int64_t ldb,
                        double *d_x, int64_t ldx, int method, double eps, int64_t itermax,
                        int64_t gmres_im, int64_t *niter, double *berr, void *stream );

/* y = alpha A x + beta y with the loaded matrix, in the original ordering, host
 * pointers (spmMatVec; used for backward errors).  nrhs columns. */
int b200_spmv( b200_solver_t *solver, int64_t nrhs, double alpha, const double *x, int64_t ldx,
               double beta, double *y, int64_t ldy );

/* The same product on device pointers, enqueued on stream (NULL: the solver's
 * stream) without a synchronization; its scratch is the solve workspace. */
int b200_spmv_device( b200_solver_t *solver, int64_t nrhs, double alpha, const double *d_x, int64_t ldx,
                      double beta, double *d_y, int64_t ldy, void *stream );

/* Copy the factor back in PaStiX's coeftab layout: every cblk's 2D block layout
 * (blend/solver_matrix_gen_utils.h:137-165), cblks concatenated in order, as
 * double.  U (LU only, else NULL) receives the transposed U factor.  Each array
 * holds coefnbr entries. */
int b200_factor_download( b200_solver_t *solver, double *L, double *U );

/* Statistics of the last calls: out[0] numfact ms, out[1] solve ms, out[2]
 * refine ms, out[3] static pivots, out[4] diag threshold used, out[5] device
 * bytes held by the factor, out[6] number of etree levels, out[7] kernel launches
 * of the last numfact, out[8] kernel launches of the last solve, out[9] coefnbr,
 * out[10] kernels run by this instance so far, out[11] bytes of the solve /
 * refinement workspace, out[12] bytes of the device copies of host vectors.
 * out holds 13 entries. */
int b200_stats( b200_solver_t *solver, double *out );

/* Short description of a return code. */
const char *b200_strerror( int code );

#ifdef __cplusplus
}
#endif

#endif /* PASTIX_B200_H */
