// Kernel launchers of the B200 factorization/solve library.
#pragma once

#include <cuda.h>

#include "b200_internal.h"

namespace b200 {

// factorization (factor_kernels.cu)
template <typename T>
void launch_scatter(int64_t nnz, const int64_t *dest, const double *Lv, const double *Uv, T *L, T *U,
                    cudaStream_t st);
// tinv: per cblk 32 x ncols (x2 for LU) tile inverses written by the diagonal kernel, read by the TRSM
template <typename T>
void launch_diag(int facto, const DevSym &s, const int *cblks, int ncblk, T *L, T *U, T *tinv,
                 const int64_t *tinv_off, const double *thr, unsigned long long *npiv, int *err, cudaStream_t st);
// the same for cblks of at most nb (8, 16 or 32) columns, one warp per cblk, with the
// panel solve of their rows below (no TRSM task for them)
template <typename T>
void launch_diag_small(int facto, const DevSym &s, const int *cblks, int ncblk, int nb, T *L, T *U, T *tinv,
                       const int64_t *tinv_off, const double *thr, unsigned long long *npiv, int *err,
                       cudaStream_t st);
// X op(T) = B: mode 0 upper / 1 lower-transposed for the left-looking part; which = 0 (inv L) or 1 (inv U^T)
// selects the tile inverse; scale_d divides by D (LDL^T)
template <typename T>
void launch_trsm(const DevSym &s, const RowTask *tasks, int ntasks, int TR, int nmax, T *P, const T *D, int mode,
                 const T *tinv, const int64_t *tinv_off, int which, int getrf, int scale_d, cudaStream_t st);
// every wide POTRF / LDL^T cblk of a level in one launch (panel_kernels.cu): items
// taken in order from *ticket, dependencies through the solved / updated counters
// (zeroed before the factorization, like *ticket and *abort_word)
template <typename T>
void launch_panel(int facto, const DevSym &s, const PanelCblk *pcb, const PanelItem *items, int nitems, int *ticket,
                  int *solved, int *updated, int *abort_word, T *L, const double *thr, unsigned long long *npiv,
                  int *err, cudaStream_t st);
// the row-block form (one item per row block, resident in shared memory for all
// steps): items = the diagonal blocks' 64-row blocks first, then the rb-row blocks
// below; nsmax = the most 64-column steps of a cblk of the launch;
// panel_rows_block gives the rb (128 or 64) whose blocks of such a cblk fit in
// shared memory, 0 if none does
template <typename T>
void launch_panel_rows(int facto, const DevSym &s, const PanelCblk *pcb, const PanelItem *items, int nitems,
                       int nsmax, int rb, int *ticket, int *solved, int *abort_word, T *L, const double *thr,
                       unsigned long long *npiv, int *err, cudaStream_t st);
int panel_rows_block(int nsmax, size_t esz);
int configure_panel_kernels();
// the diagonal of the factor's diagonal blocks, in the permuted numbering (n doubles)
template <typename T>
void launch_get_diag(const DevSym &s, const T *L, double *out, cudaStream_t st);
// updates with K <= 16 and N <= 32, one warp each
template <typename T>
void launch_update_small(const DevSym &s, const Upd *upds, int nupd, T *L, T *U, cudaStream_t st);
void launch_update_f64(const DevSym &s, const Upd *upds, int nupd, int ntiles, double *L, double *U,
                       cudaStream_t st);
void launch_update_f32(const DevSym &s, const Upd *upds, int nupd, int ntiles, float *L, float *U,
                       cudaStream_t st);
// the bottom levels of the tree in one launch (cblks of at most 32 columns): items
// (factor items, then update items, level by level) taken by warps from *ticket; a
// factor item starts when cnt[k] (the update items k receives from the launch's cblks)
// reaches 0 and sets it to -1 when k is factored, which its update items wait for;
// updates (upds, indexed by the items) accumulate with atomics.  cnt, *ticket and
// *abort_word are reset before every factorization; a wait that runs out sets bit 5
// of err.
template <typename T>
void launch_dag_bottom(int facto, const DevSym &s, int grid, const DagItem *items, int nitems, const Upd *upds,
                       int *cnt, int *ticket, int *abort_word, T *L, T *U, T *tinv, const int64_t *tinv_off,
                       const double *thr, unsigned long long *npiv, int *err, cudaStream_t st);
// its grid: the CTAs resident at once on this device, capped by the items (-1 on error)
int dag_bottom_grid(int facto, bool f32, int ncblk);
// returns the dynamic shared memory (bytes) the panel TRSM may use, or -1
int configure_factor_kernels();
// FP32 updates on the tensor cores (update_tc.cu).  Tiles of 128 rows x bn (64 or 128)
// columns listed by tmap ({update index, row tile | column tile << 16}); maps: 4 x cblknbr
// tensor maps of the operand arenas, [(side * 2 + part) * cblknbr + k] with side
// 0 L / 1 U and part 0 hi / 1 lo; split: 3xTF32.
// op: operand format of the copies, 0 FP32 read as TF32 (kind::tf32), 1 BF16 (kind::f16, always split)
void launch_update_tc(const DevSym &s, const Upd *upds, const int2 *tmap, int ntiles, const void *maps, float *L,
                      float *U, int split, int bn, int op, int *err, cudaStream_t st);
int configure_tc_kernels();
// copy panel tiles row-major into the operand arena (hi, and lo = x - hi when lo is given)
void launch_panel_split(const DevSym &s, const SplitTask *tasks, int ntasks, const float *P, const int64_t *toff,
                        void *hi, void *lo, int op, cudaStream_t st);
// tensor maps of the operand copies of the cblks with wanted[k] != 0 (maps: cblknbr entries)
int encode_operand_maps(const std::vector<int64_t> &toff, const std::vector<int> &stride,
                        const std::vector<int> &ncols, const std::vector<char> &wanted, void *arena, int op,
                        CUtensorMap *maps);

// solve (solve_kernels.cu); x is the permuted right-hand side block, n x nrhs, leading
// dimension ldx, in the vector precision V (double with an FP64 factor, float with FP32)
// off-diagonal solve on 64x64 tiles with tensor cores (atomic accumulation into b)
template <typename T, typename V>
void launch_solve_tiles(const DevSym &s, const SolveTile *tasks, int ntasks, const T *L, const V *x, V *b,
                        int64_t ldx, int nrhs, int backward, cudaStream_t st);
// both sweeps' work of cblks with at most 32 columns, one warp per cblk: forward
// aux_k = W_k x_k and x[rows below] -= P aux_k; backward x_k = W_k^T (aux_k - P^T x[rows below])
template <typename T, typename V>
void launch_solve_leaf(const DevSym &s, const int *cblks, int ncblk, const T *P, const T *W, const int64_t *woff,
                       V *x, V *aux, int64_t ldx, int nrhs, int backward, cudaStream_t st);
// W_k = inverse of the lower-triangular diagonal block of every listed cblk (W: n x n per cblk)
template <typename T>
void launch_diag_inverse(const DevSym &s, const int *cblks, int ncblk, const T *L, T *W, const int64_t *woff,
                         int unit, cudaStream_t st);
// W_k of cblks with at most 32 columns, copied from the diagonal kernel's tile inverses (which: 0 L, 1 U^T)
template <typename T>
void launch_copy_tile_inverse(const DevSym &s, const int *cblks, int ncblk, const T *tinv, const int64_t *toff, T *W,
                              const int64_t *woff, int which, cudaStream_t st);
// xout[k] += W_k xin[k] (forward) or W_k^T xin[k] (backward), one 64 x 64 tile of W_k per task
// {k, output row0, K chunk col0}, xout zeroed by the caller before the sweep
template <typename T, typename V>
void launch_solve_diag_inv(const DevSym &s, const SolveTile *tasks, int ntasks, const T *W, const int64_t *woff,
                           const V *xin, V *xout, int64_t ldx, int nrhs, int backward, cudaStream_t st);
template <typename T, typename V>
void launch_solve_scale_diag(const DevSym &s, const int *cblks, int ncblk, const T *L, V *x, int64_t ldx, int nrhs,
                             cudaStream_t st);
// one sweep as a dataflow launch (solve_kernels.cu): items in order from *ticket;
// forward: need[f] contributions complete x_f (cnt_a), nprev[k] diagonal items
// complete aux_k (cnt_b); backward: need[f] items finish x_f (cnt_a), nprev[k]
// off-diagonal items complete aux_k (cnt_b); counters zeroed before the launch
template <typename T, typename V>
void launch_solve_flow(const DevSym &s, const FlowItem *items, int nitems, const int *leaf, const int *flist,
                       const int *need, const int *nprev, const T *P, const T *W, const int64_t *woff, V *x, V *aux,
                       int64_t ldx, int nrhs, int backward, int *ticket, int *cnt_a, int *cnt_b, int *abort_word,
                       int *err, cudaStream_t st);
// dst = (D) src on an n x nrhs block
template <typename S, typename D>
void launch_convert(int n, int nrhs, const S *src, int64_t lds, D *dst, int64_t ldd, cudaStream_t st);
void launch_permute(int n, int nrhs, const int *peri, const double *src, int64_t lds, double *dst, int64_t ldd,
                    int forward, cudaStream_t st);
int configure_solve_kernels();
int configure_inverse_kernels();

// refinement vectors (refine_kernels.cu)
// xt (n x 16 doubles, may be null): row-major staging of 16 columns of x at a time
void launch_spmv(int n, int nrhs, const int64_t *colptr, const int *rowtab, const double *vals, const double *x,
                 int64_t ldx, double *y, int64_t ldy, double alpha, double beta, cudaStream_t st,
                 double *xt = nullptr);
// dst[e] = src[map[e]], e < nnz
void launch_gather_values(int64_t nnz, const int64_t *map, const double *src, double *dst, cudaStream_t st);
// out[r] = sum_i x[i,r] * y[i,r]  (nrhs columns), accumulated in double
void launch_dots(int n, int nrhs, const double *x, int64_t ldx, const double *y, int64_t ldy, double *out,
                 cudaStream_t st);
// Per-problem scalars: problem p(i, r) = r * nseg + segid[i] in a batch of nseg
// independent systems (segid: system of each row), r without one (nseg = 1).
// y[:,r] += a[p] * x[:,r]  (a on the device); sign: +1 or -1 applied to a
void launch_axpys(int n, int nrhs, const double *a, double sign, const double *x, int64_t ldx, double *y,
                  int64_t ldy, cudaStream_t st, int nseg = 1, const int *segid = nullptr);
// y[:,r] = x[:,r] + b[p] * y[:,r]
void launch_xpbys(int n, int nrhs, const double *x, int64_t ldx, const double *b, double *y, int64_t ldy,
                  cudaStream_t st, int nseg = 1, const int *segid = nullptr);
void launch_copy(int n, int nrhs, const double *x, int64_t ldx, double *y, int64_t ldy, cudaStream_t st);
// y[:,r] = alpha * x[:,r] + beta * y[:,r]
void launch_axpby(int n, int nrhs, double alpha, const double *x, int64_t ldx, double beta, double *y, int64_t ldy,
                  cudaStream_t st);
// y[:,r] = s[p] * x[:,r]
void launch_scal_cols(int n, int nrhs, const double *s, const double *x, int64_t ldx, double *y, int64_t ldy,
                      cudaStream_t st, int nseg = 1, const int *segid = nullptr);
// out[r * nseg + p] = sum over the rows [seg[p], seg[p+1]) of x[i,r] * y[i,r]
void launch_seg_dots(int nseg, const int *seg, int nrhs, const double *x, int64_t ldx, const double *y, int64_t ldy,
                     double *out, cudaStream_t st);
// thr[i] = use_norm ? c * ||columns [sys_col[i], sys_col[i+1]) of the bcsc||_F : c
void launch_batch_threshold(int nsys, const int *sys_col, const int64_t *colptr, const double *vals, double c,
                            int use_norm, double *thr, cudaStream_t st);

}  // namespace b200
