// Kernel launchers of the B200 factorization/solve library.
#pragma once

#include "b200_internal.h"

namespace b200 {

// factorization (factor_kernels.cu)
template <typename T>
void launch_scatter(int64_t nnz, const int64_t *dest, const double *Lv, const double *Uv, T *L, T *U,
                    cudaStream_t st);
template <typename T>
void launch_diag(int facto, const DevSym &s, const int *cblks, int ncblk, T *L, T *U, const double *thr,
                 unsigned long long *npiv, int *err, cudaStream_t st);
template <typename T>
void launch_trsm(const DevSym &s, const RowTask *tasks, int ntasks, int TR, int nmax, T *P, const T *D, int mode,
                 int unit, cudaStream_t st);
void launch_update_f64(const DevSym &s, const Upd *upds, int nupd, int ntiles, double *L, double *U,
                       cudaStream_t st);
void launch_update_f32(const DevSym &s, const Upd *upds, int nupd, int ntiles, float *L, float *U,
                       cudaStream_t st);
// returns the dynamic shared memory (bytes) the panel TRSM may use, or -1
int configure_factor_kernels();

// solve (solve_kernels.cu); x is the permuted right-hand side block, n x nrhs, leading dimension ldx
template <typename T>
void launch_solve_diag(const DevSym &s, const int *cblks, int ncblk, int nmax, const T *L, double *x, int64_t ldx,
                       int nrhs, int backward, int unit, cudaStream_t st);
template <typename T>
void launch_solve_offdiag(const DevSym &s, const RowTask *tasks, int ntasks, const T *L, double *x, int64_t ldx,
                          int nrhs, int backward, cudaStream_t st);
template <typename T>
void launch_solve_scale_diag(const DevSym &s, const int *cblks, int ncblk, const T *L, double *x, int64_t ldx,
                             int nrhs, cudaStream_t st);
void launch_permute(int n, int nrhs, const int *peri, const double *src, int64_t lds, double *dst, int64_t ldd,
                    int forward, cudaStream_t st);
int configure_solve_kernels();

// refinement vectors (refine_kernels.cu)
void launch_spmv(int n, int nrhs, const int64_t *colptr, const int *rowtab, const double *vals, const double *x,
                 int64_t ldx, double *y, int64_t ldy, double alpha, double beta, cudaStream_t st);
// out[r] = sum_i x[i,r] * y[i,r]  (nrhs columns), accumulated in double
void launch_dots(int n, int nrhs, const double *x, int64_t ldx, const double *y, int64_t ldy, double *out,
                 cudaStream_t st);
// y[:,r] += a[r] * x[:,r]  (a on the device); sign: +1 or -1 applied to a
void launch_axpys(int n, int nrhs, const double *a, double sign, const double *x, int64_t ldx, double *y,
                  int64_t ldy, cudaStream_t st);
// y[:,r] = x[:,r] + b[r] * y[:,r]
void launch_xpbys(int n, int nrhs, const double *x, int64_t ldx, const double *b, double *y, int64_t ldy,
                  cudaStream_t st);
void launch_copy(int n, int nrhs, const double *x, int64_t ldx, double *y, int64_t ldy, cudaStream_t st);
// y[:,r] = alpha * x[:,r] + beta * y[:,r]
void launch_axpby(int n, int nrhs, double alpha, const double *x, int64_t ldx, double beta, double *y, int64_t ldy,
                  cudaStream_t st);
// y[:,r] = s[r] * x[:,r]
void launch_scal_cols(int n, int nrhs, const double *s, const double *x, int64_t ldx, double *y, int64_t ldy,
                      cudaStream_t st);

}  // namespace b200
