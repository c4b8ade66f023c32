// FP64 vector kernels of the iterative refinement (sm_100a): bcsc SpMV and the
// BLAS-1 operations the refinement drivers need, all on n x nrhs column-major
// blocks with one scalar per column (bcsc/bcsc_zspmv.c, bcsc/bvec_zcompute.c).
#include "b200_internal.h"
#include "kernels.h"

namespace b200 {

// y = alpha * A x + beta * y.  The matrix is the bcsc in the permuted basis, read
// row-wise: for a symmetric matrix the bcsc columns hold both triangles so column
// i is row i; for a general matrix the values passed are A^T in the same pattern
// (Uvalues), whose column i is row i of A (bcsc/bcsc_zspmv.c:127-240).
// One warp per row.
__global__ void __launch_bounds__(256) spmv_kernel(int n, int nrhs, const int64_t *__restrict__ colptr,
                                                   const int *__restrict__ rowtab, const double *__restrict__ vals,
                                                   const double *__restrict__ x, int64_t ldx, double *y, int64_t ldy,
                                                   double alpha, double beta) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int64_t e0 = colptr[warp], e1 = colptr[warp + 1];
    for (int r = 0; r < nrhs; r++) {
        double acc = 0.0;
        for (int64_t e = e0 + lane; e < e1; e += 32) acc += vals[e] * x[rowtab[e] + r * ldx];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            double *yp = y + warp + r * ldy;
            *yp = (beta == 0.0) ? alpha * acc : alpha * acc + beta * *yp;
        }
    }
}

// Column dot products, one CTA per (column, chunk), atomically accumulated.
__global__ void dots_kernel(int n, const double *__restrict__ x, int64_t ldx, const double *__restrict__ y,
                            int64_t ldy, double *out) {
    const int r = blockIdx.y;
    __shared__ double red[32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += x[i + r * ldx] * y[i + r * ldy];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) atomicAdd(out + r, acc);
    }
}

// Refinement runs one independent problem per right-hand side column, or in a
// batch of independent systems one per (column, system): the problem of row i of
// column r is r * nseg + segid[i] (segid null: nseg = 1, the column).
__device__ __forceinline__ int problem_of(int i, int r, int nseg, const int *__restrict__ segid) {
    return r * nseg + (segid ? segid[i] : 0);
}

__global__ void axpys_kernel(int n, int nrhs, const double *__restrict__ a, double sign,
                             const double *__restrict__ x, int64_t ldx, double *y, int64_t ldy, int nseg,
                             const int *__restrict__ segid) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * nrhs) return;
    const int i = (int)(idx % n), r = (int)(idx / n);
    y[i + r * ldy] += sign * a[problem_of(i, r, nseg, segid)] * x[i + r * ldx];
}

__global__ void xpbys_kernel(int n, int nrhs, const double *__restrict__ x, int64_t ldx, const double *__restrict__ b,
                             double *y, int64_t ldy, int nseg, const int *__restrict__ segid) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * nrhs) return;
    const int i = (int)(idx % n), r = (int)(idx / n);
    y[i + r * ldy] = x[i + r * ldx] + b[problem_of(i, r, nseg, segid)] * y[i + r * ldy];
}

// Dot products of every (column, system) problem of a batch: one block per
// problem over its system's rows [seg[p], seg[p + 1]), in a fixed order.
__global__ void seg_dots_kernel(int nseg, const int *__restrict__ seg, const double *__restrict__ x, int64_t ldx,
                                const double *__restrict__ y, int64_t ldy, double *out) {
    const int p = blockIdx.x, r = blockIdx.y;
    __shared__ double red[32];
    double acc = 0.0;
    for (int i = seg[p] + threadIdx.x; i < seg[p + 1]; i += blockDim.x) acc += x[i + r * ldx] * y[i + r * ldy];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) out[r * nseg + p] = acc;
    }
}

// Static-pivoting threshold of every system of a batch from its own Frobenius
// norm, summed over its columns [sys_col[i], sys_col[i + 1]) of the bcsc (full
// pattern: both triangles of a symmetric matrix):
// thr_i = use_norm ? c * ||A_i||_F : c.
__global__ void batch_threshold_kernel(const int *__restrict__ sys_col, const int64_t *__restrict__ colptr,
                                       const double *__restrict__ vals, double c, int use_norm, double *thr) {
    const int p = blockIdx.x;
    __shared__ double red[32];
    double acc = 0.0;
    for (int64_t e = colptr[sys_col[p]] + threadIdx.x; e < colptr[sys_col[p + 1]]; e += blockDim.x)
        acc += vals[e] * vals[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) thr[p] = use_norm ? c * sqrt(acc) : c;
    }
}

__global__ void axpby_kernel(int n, int nrhs, double alpha, const double *__restrict__ x, int64_t ldx, double beta,
                             double *y, int64_t ldy) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * nrhs) return;
    const int i = (int)(idx % n), r = (int)(idx / n);
    const double yv = (beta == 0.0) ? 0.0 : beta * y[i + r * ldy];
    y[i + r * ldy] = alpha * x[i + r * ldx] + yv;
}

__global__ void scal_cols_kernel(int n, int nrhs, const double *__restrict__ s, const double *__restrict__ x,
                                 int64_t ldx, double *y, int64_t ldy, int nseg, const int *__restrict__ segid) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * nrhs) return;
    const int i = (int)(idx % n), r = (int)(idx / n);
    y[i + r * ldy] = s[problem_of(i, r, nseg, segid)] * x[i + r * ldx];
}

static inline unsigned nblk(int64_t tot, int bs) { return (unsigned)((tot + bs - 1) / bs); }

// Several right-hand sides: the columns r0 .. r0 + 15 of x first gathered
// row-major (16 doubles = 128 contiguous bytes per row), so that every matrix entry
// gathers one line instead of 16 scattered ones; then half a warp per row.
constexpr int SPMV_R = 16;

__global__ void gather_rows_kernel(int n, int R, const double *__restrict__ x, int64_t ldx, double *__restrict__ xt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v[SPMV_R];
#pragma unroll
    for (int r = 0; r < SPMV_R; r++) v[r] = r < R ? x[i + (int64_t)r * ldx] : 0.0;
    double2 *o = reinterpret_cast<double2 *>(xt + (int64_t)i * SPMV_R);
#pragma unroll
    for (int h = 0; h < SPMV_R / 2; h++) o[h] = make_double2(v[2 * h], v[2 * h + 1]);
}

// Half a warp per row, lane c of the half = right-hand side c: every entry is one
// broadcast load of its value and row index and one contiguous 128-byte load of the
// staged x row, accumulated in the row's order; no reduction across lanes.
__global__ void __launch_bounds__(256) spmv_rows_kernel(int n, int R, const int64_t *__restrict__ colptr,
                                                        const int *__restrict__ rowtab,
                                                        const double *__restrict__ vals,
                                                        const double *__restrict__ xt, double *y, int64_t ldy,
                                                        double alpha, double beta) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t row = t / SPMV_R;
    const int c = (int)(t % SPMV_R);
    if (row >= n) return;
    const int64_t e0 = colptr[row], e1 = colptr[row + 1];
    const double *xc = xt + c;
    double acc = 0.0;
    int64_t e = e0;
    for (; e + 4 <= e1; e += 4) {
        const int j0 = rowtab[e], j1 = rowtab[e + 1], j2 = rowtab[e + 2], j3 = rowtab[e + 3];
        const double v0 = vals[e], v1 = vals[e + 1], v2 = vals[e + 2], v3 = vals[e + 3];
        const double x0 = xc[(int64_t)j0 * SPMV_R], x1 = xc[(int64_t)j1 * SPMV_R];
        const double x2 = xc[(int64_t)j2 * SPMV_R], x3 = xc[(int64_t)j3 * SPMV_R];
        acc = fma(v0, x0, acc);
        acc = fma(v1, x1, acc);
        acc = fma(v2, x2, acc);
        acc = fma(v3, x3, acc);
    }
    for (; e < e1; e++) acc = fma(vals[e], xc[(int64_t)rowtab[e] * SPMV_R], acc);
    if (c < R) {
        double *yp = y + row + (int64_t)c * ldy;
        *yp = (beta == 0.0) ? alpha * acc : alpha * acc + beta * *yp;
    }
}

void launch_spmv(int n, int nrhs, const int64_t *colptr, const int *rowtab, const double *vals, const double *x,
                 int64_t ldx, double *y, int64_t ldy, double alpha, double beta, cudaStream_t st, double *xt) {
    if (n <= 0) return;
    if (nrhs > 1 && xt) {
        for (int r0 = 0; r0 < nrhs; r0 += SPMV_R) {
            const int R = nrhs - r0 < SPMV_R ? nrhs - r0 : SPMV_R;
            gather_rows_kernel<<<nblk(n, 256), 256, 0, st>>>(n, R, x + (int64_t)r0 * ldx, ldx, xt);
            spmv_rows_kernel<<<nblk((int64_t)n * SPMV_R, 256), 256, 0, st>>>(n, R, colptr, rowtab, vals, xt,
                                                                              y + (int64_t)r0 * ldy, ldy, alpha, beta);
        }
    } else {
        spmv_kernel<<<nblk((int64_t)n * 32, 256), 256, 0, st>>>(n, nrhs, colptr, rowtab, vals, x, ldx, y, ldy, alpha,
                                                                 beta);
    }
}

// dst[e] = src[map[e]] (values of the input matrix -> bcsc entries)
__global__ void gather_values_kernel(int64_t nnz, const int64_t *__restrict__ map, const double *__restrict__ src,
                                     double *__restrict__ dst) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < nnz) dst[e] = src[map[e]];
}

void launch_gather_values(int64_t nnz, const int64_t *map, const double *src, double *dst, cudaStream_t st) {
    if (nnz <= 0) return;
    gather_values_kernel<<<nblk(nnz, 256), 256, 0, st>>>(nnz, map, src, dst);
}

void launch_dots(int n, int nrhs, const double *x, int64_t ldx, const double *y, int64_t ldy, double *out,
                 cudaStream_t st) {
    if (nrhs <= 0) return;
    cudaMemsetAsync(out, 0, nrhs * sizeof(double), st);
    const int bs = 256;
    int gx = (int)std::min<int64_t>(296, ((int64_t)n + bs - 1) / bs);
    if (gx < 1) gx = 1;
    dots_kernel<<<dim3(gx, nrhs), bs, 0, st>>>(n, x, ldx, y, ldy, out);
}

void launch_axpys(int n, int nrhs, const double *a, double sign, const double *x, int64_t ldx, double *y,
                  int64_t ldy, cudaStream_t st, int nseg, const int *segid) {
    const int64_t tot = (int64_t)n * nrhs;
    if (tot <= 0) return;
    axpys_kernel<<<nblk(tot, 256), 256, 0, st>>>(n, nrhs, a, sign, x, ldx, y, ldy, nseg, segid);
}

void launch_xpbys(int n, int nrhs, const double *x, int64_t ldx, const double *b, double *y, int64_t ldy,
                  cudaStream_t st, int nseg, const int *segid) {
    const int64_t tot = (int64_t)n * nrhs;
    if (tot <= 0) return;
    xpbys_kernel<<<nblk(tot, 256), 256, 0, st>>>(n, nrhs, x, ldx, b, y, ldy, nseg, segid);
}

void launch_seg_dots(int nseg, const int *seg, int nrhs, const double *x, int64_t ldx, const double *y, int64_t ldy,
                     double *out, cudaStream_t st) {
    if (nseg <= 0 || nrhs <= 0) return;
    seg_dots_kernel<<<dim3(nseg, nrhs), 256, 0, st>>>(nseg, seg, x, ldx, y, ldy, out);
}

void launch_batch_threshold(int nsys, const int *sys_col, const int64_t *colptr, const double *vals, double c,
                            int use_norm, double *thr, cudaStream_t st) {
    if (nsys <= 0) return;
    batch_threshold_kernel<<<nsys, 256, 0, st>>>(sys_col, colptr, vals, c, use_norm, thr);
}

void launch_copy(int n, int nrhs, const double *x, int64_t ldx, double *y, int64_t ldy, cudaStream_t st) {
    launch_axpby(n, nrhs, 1.0, x, ldx, 0.0, y, ldy, st);
}

void launch_axpby(int n, int nrhs, double alpha, const double *x, int64_t ldx, double beta, double *y, int64_t ldy,
                  cudaStream_t st) {
    const int64_t tot = (int64_t)n * nrhs;
    if (tot <= 0) return;
    axpby_kernel<<<nblk(tot, 256), 256, 0, st>>>(n, nrhs, alpha, x, ldx, beta, y, ldy);
}

void launch_scal_cols(int n, int nrhs, const double *s, const double *x, int64_t ldx, double *y, int64_t ldy,
                      cudaStream_t st, int nseg, const int *segid) {
    const int64_t tot = (int64_t)n * nrhs;
    if (tot <= 0) return;
    scal_cols_kernel<<<nblk(tot, 256), 256, 0, st>>>(n, nrhs, s, x, ldx, y, ldy, nseg, segid);
}

}  // namespace b200
