// Supernodal triangular solve kernels (sm_100a).  Vectors are double; the factor
// is read in its own precision (double or float) and converted on load.
//
//  solve_diag_kernel        diagonal-block TRSM of one cblk, forward (L) or
//                           backward (L^T / U) -- solve_blok_ztrsm
//                           (kernels/solve_ztrsmsp.c:67-95)
//  solve_offdiag_fwd_kernel b[f] -= A_blk x[k] for a tile of off-diagonal rows,
//                           scattered to global rows (solve_blok_zgemm forward,
//                           kernels/solve_ztrsmsp.c:275-280)
//  solve_offdiag_bwd_kernel b[k] -= A_blk^T x[f] for a tile of rows (backward)
//  solve_scale_diag_kernel  b /= D (solve_cblk_zdiag, kernels/solve_ztrsmsp.c:584-633)
//  permute_kernel           bvec_zlapmr with peritab (bcsc/bvec_zcompute.c:875)
#include "b200_internal.h"
#include "kernels.h"

namespace b200 {

constexpr int SRB = 16;   // right-hand sides per pass
constexpr int STP = 33;

__device__ __forceinline__ int panel_row_to_global(const DevSym &s, int k, int prow) {
    int lo = s.fblok[k], hi = s.fblok[k + 1] - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s.rowoff[mid] <= prow) lo = mid; else hi = mid - 1;
    }
    return s.frow[lo] + (prow - s.rowoff[lo]);
}

template <typename T>
__global__ void __launch_bounds__(256) solve_diag_kernel(DevSym s, const int *__restrict__ cblks,
                                                         const T *__restrict__ L, double *x, int64_t ldx,
                                                         int nrhs, int backward, int unit) {
    extern __shared__ __align__(16) double bs[];  // n x SRB
    __shared__ double tile[32 * STP];
    const int k = cblks[blockIdx.x];
    const int n = s.ncols[k], ld = s.ld[k];
    const T *D = L + s.off[k];
    double *xk = x + s.fcol[k];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (int r0 = 0; r0 < nrhs; r0 += SRB) {
        const int R = min(SRB, nrhs - r0);
        for (int idx = tid; idx < n * R; idx += blockDim.x) {
            const int i = idx % n, r = idx / n;
            bs[i + r * n] = xk[i + (size_t)(r0 + r) * ldx];
        }
        __syncthreads();
        if (!backward) {
            for (int cb = 0; cb < n; cb += 32) {
                const int w = min(32, n - cb);
                for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
                    const int l = idx & 31, c = idx >> 5;
                    tile[l + c * STP] = (l < w && c < w && l >= c) ? (double)D[(cb + l) + (size_t)(cb + c) * ld] : 0.0;
                }
                __syncthreads();
                for (int r = warp; r < R; r += nw) {
                    double v = (lane < w) ? bs[cb + lane + r * n] : 0.0;
                    for (int c = 0; c < w; c++) {
                        double xc = __shfl_sync(0xffffffffu, v, c);
                        if (!unit) xc = xc / tile[c * (STP + 1)];
                        if (lane == c) v = xc;
                        else if (lane > c && lane < w) v -= tile[lane + c * STP] * xc;
                    }
                    if (lane < w) bs[cb + lane + r * n] = v;
                }
                __syncthreads();
                // rows below the tile: one thread per row, all right-hand sides
                for (int i = cb + w + tid; i < n; i += blockDim.x) {
                    double acc[SRB];
#pragma unroll
                    for (int j = 0; j < SRB; j++) acc[j] = 0.0;
#pragma unroll 8
                    for (int c = 0; c < w; c++) {
                        const double d = (double)D[i + (size_t)(cb + c) * ld];
#pragma unroll
                        for (int j = 0; j < SRB; j++)
                            if (j < R) acc[j] += d * bs[cb + c + j * n];
                    }
#pragma unroll
                    for (int j = 0; j < SRB; j++)
                        if (j < R) bs[i + j * n] -= acc[j];
                }
                __syncthreads();
            }
        } else {
            for (int cb = ((n - 1) / 32) * 32; cb >= 0; cb -= 32) {
                const int w = min(32, n - cb);
                // columns of the tile: one warp per column, lanes over the rows below
                for (int c = warp; c < w; c += nw) {
                    double acc[SRB];
#pragma unroll
                    for (int j = 0; j < SRB; j++) acc[j] = 0.0;
                    for (int i = cb + w + lane; i < n; i += 32) {
                        const double d = (double)D[i + (size_t)(cb + c) * ld];
#pragma unroll
                        for (int j = 0; j < SRB; j++)
                            if (j < R) acc[j] += d * bs[i + j * n];
                    }
#pragma unroll
                    for (int j = 0; j < SRB; j++) {
                        if (j < R) {
                            double v = acc[j];
#pragma unroll
                            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                            if (lane == 0) bs[cb + c + j * n] -= v;
                        }
                    }
                }
                for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
                    const int l = idx & 31, c = idx >> 5;
                    tile[l + c * STP] = (l < w && c < w && l >= c) ? (double)D[(cb + l) + (size_t)(cb + c) * ld] : 0.0;
                }
                __syncthreads();
                for (int r = warp; r < R; r += nw) {
                    double v = (lane < w) ? bs[cb + lane + r * n] : 0.0;
                    for (int c = w - 1; c >= 0; c--) {
                        double xc = __shfl_sync(0xffffffffu, v, c);
                        if (!unit) xc = xc / tile[c * (STP + 1)];
                        if (lane == c) v = xc;
                        else if (lane < c) v -= tile[c + lane * STP] * xc;
                    }
                    if (lane < w) bs[cb + lane + r * n] = v;
                }
                __syncthreads();
            }
        }
        for (int idx = tid; idx < n * R; idx += blockDim.x) {
            const int i = idx % n, r = idx / n;
            xk[i + (size_t)(r0 + r) * ldx] = bs[i + r * n];
        }
        __syncthreads();
    }
}

constexpr int SOL_TR = 128;

template <typename T>
__global__ void __launch_bounds__(SOL_TR) solve_offdiag_fwd_kernel(DevSym s, const RowTask *__restrict__ tasks,
                                                                   const T *__restrict__ L, double *x, int64_t ldx,
                                                                   int nrhs) {
    extern __shared__ __align__(16) double xs[];  // n x SRB
    const RowTask t = tasks[blockIdx.x];
    const int k = t.k, n = s.ncols[k], ld = s.ld[k];
    const int rows = min(SOL_TR, s.stride[k] - t.row0);
    const T *P = L + s.off[k] + t.row0;
    const int r = threadIdx.x;
    const int grow = (r < rows) ? panel_row_to_global(s, k, t.row0 + r) : -1;
    const double *xk = x + s.fcol[k];
    for (int r0 = 0; r0 < nrhs; r0 += SRB) {
        const int R = min(SRB, nrhs - r0);
        for (int idx = threadIdx.x; idx < n * R; idx += blockDim.x) {
            const int c = idx % n, j = idx / n;
            xs[c + j * n] = xk[c + (size_t)(r0 + j) * ldx];
        }
        __syncthreads();
        if (r < rows) {
            double acc[SRB];
#pragma unroll
            for (int j = 0; j < SRB; j++) acc[j] = 0.0;
            for (int c = 0; c < n; c++) {
                const double p = (double)P[r + (size_t)c * ld];
#pragma unroll
                for (int j = 0; j < SRB; j++)
                    if (j < R) acc[j] += p * xs[c + j * n];
            }
#pragma unroll
            for (int j = 0; j < SRB; j++)
                if (j < R) atomicAdd(&x[grow + (size_t)(r0 + j) * ldx], -acc[j]);
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(SOL_TR) solve_offdiag_bwd_kernel(DevSym s, const RowTask *__restrict__ tasks,
                                                                   const T *__restrict__ L, double *x, int64_t ldx,
                                                                   int nrhs) {
    __shared__ double xg[SOL_TR * SRB];
    const RowTask t = tasks[blockIdx.x];
    const int k = t.k, n = s.ncols[k], ld = s.ld[k];
    const int rows = min(SOL_TR, s.stride[k] - t.row0);
    const T *P = L + s.off[k] + t.row0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int grow = (tid < rows) ? panel_row_to_global(s, k, t.row0 + tid) : -1;
    double *xk = x + s.fcol[k];
    for (int r0 = 0; r0 < nrhs; r0 += SRB) {
        const int R = min(SRB, nrhs - r0);
        for (int j = 0; j < R; j++) xg[tid + j * SOL_TR] = (tid < rows) ? x[grow + (size_t)(r0 + j) * ldx] : 0.0;
        __syncthreads();
        for (int c = warp; c < n; c += nw) {
            double acc[SRB];
#pragma unroll
            for (int j = 0; j < SRB; j++) acc[j] = 0.0;
            for (int rr = lane; rr < rows; rr += 32) {
                const double p = (double)P[rr + (size_t)c * ld];
#pragma unroll
                for (int j = 0; j < SRB; j++)
                    if (j < R) acc[j] += p * xg[rr + j * SOL_TR];
            }
#pragma unroll
            for (int j = 0; j < SRB; j++) {
                if (j < R) {
                    double v = acc[j];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    if (lane == 0) atomicAdd(&xk[c + (size_t)(r0 + j) * ldx], -v);
                }
            }
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void solve_scale_diag_kernel(DevSym s, const int *__restrict__ cblks, const T *__restrict__ L, double *x,
                                        int64_t ldx, int nrhs) {
    const int k = cblks[blockIdx.x];
    const int n = s.ncols[k], ld = s.ld[k];
    const T *D = L + s.off[k];
    double *xk = x + s.fcol[k];
    for (int idx = threadIdx.x; idx < n * nrhs; idx += blockDim.x) {
        const int i = idx % n, r = idx / n;
        xk[i + (size_t)r * ldx] /= (double)D[(size_t)i * (ld + 1)];
    }
}

__global__ void permute_kernel(int n, int nrhs, const int *__restrict__ peri, const double *__restrict__ src,
                               int64_t lds, double *__restrict__ dst, int64_t ldd, int forward) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * nrhs) return;
    const int i = (int)(idx % n), r = (int)(idx / n);
    if (forward) dst[i + r * ldd] = src[peri[i] + r * lds];
    else dst[peri[i] + r * ldd] = src[i + r * lds];
}

template <typename T>
void launch_solve_diag(const DevSym &s, const int *cblks, int ncblk, int nmax, const T *L, double *x, int64_t ldx,
                       int nrhs, int backward, int unit, cudaStream_t st) {
    if (ncblk <= 0) return;
    const size_t smem = (size_t)nmax * SRB * sizeof(double);
    solve_diag_kernel<T><<<ncblk, 256, smem, st>>>(s, cblks, L, x, ldx, nrhs, backward, unit);
}

template <typename T>
void launch_solve_offdiag(const DevSym &s, const RowTask *tasks, int ntasks, const T *L, double *x, int64_t ldx,
                          int nrhs, int backward, cudaStream_t st) {
    if (ntasks <= 0) return;
    if (!backward) {
        // dynamic shared memory: widest cblk x SRB doubles; the caller guarantees ncols <= 1024
        solve_offdiag_fwd_kernel<T><<<ntasks, SOL_TR, 1024 * SRB * sizeof(double), st>>>(s, tasks, L, x, ldx, nrhs);
    } else {
        solve_offdiag_bwd_kernel<T><<<ntasks, SOL_TR, 0, st>>>(s, tasks, L, x, ldx, nrhs);
    }
}

template <typename T>
void launch_solve_scale_diag(const DevSym &s, const int *cblks, int ncblk, const T *L, double *x, int64_t ldx,
                             int nrhs, cudaStream_t st) {
    if (ncblk <= 0) return;
    solve_scale_diag_kernel<T><<<ncblk, 128, 0, st>>>(s, cblks, L, x, ldx, nrhs);
}

void launch_permute(int n, int nrhs, const int *peri, const double *src, int64_t lds, double *dst, int64_t ldd,
                    int forward, cudaStream_t st) {
    const int64_t tot = (int64_t)n * nrhs;
    if (tot <= 0) return;
    permute_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, nrhs, peri, src, lds, dst, ldd, forward);
}

int configure_solve_kernels() {
    const int big = 1024 * SRB * sizeof(double);
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int rc = 0;
    rc |= (int)cudaFuncSetAttribute(solve_offdiag_fwd_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    rc |= (int)cudaFuncSetAttribute(solve_offdiag_fwd_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    rc |= (int)cudaFuncSetAttribute(solve_diag_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    rc |= (int)cudaFuncSetAttribute(solve_diag_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    return (rc == 0 && optin >= big + 16 * 1024) ? 0 : -1;
}

template void launch_solve_diag<double>(const DevSym &, const int *, int, int, const double *, double *, int64_t, int,
                                        int, int, cudaStream_t);
template void launch_solve_diag<float>(const DevSym &, const int *, int, int, const float *, double *, int64_t, int,
                                       int, int, cudaStream_t);
template void launch_solve_offdiag<double>(const DevSym &, const RowTask *, int, const double *, double *, int64_t,
                                           int, int, cudaStream_t);
template void launch_solve_offdiag<float>(const DevSym &, const RowTask *, int, const float *, double *, int64_t, int,
                                          int, cudaStream_t);
template void launch_solve_scale_diag<double>(const DevSym &, const int *, int, const double *, double *, int64_t,
                                              int, cudaStream_t);
template void launch_solve_scale_diag<float>(const DevSym &, const int *, int, const float *, double *, int64_t, int,
                                             cudaStream_t);

}  // namespace b200

// ====================================================================== tensor-core solve tiles
//
// The off-diagonal part of the supernodal solves as small GEMMs on FP64 tensor
// cores (DMMA m16n8k4).  One CTA (4 warps) takes a 64-row x 64-column tile of a
// cblk's off-diagonal panel:
//   forward : b[grow(r)] -= sum_c P[r][c] x_k[c]        (warp = 16 rows)
//   backward: b_k[c]     -= sum_r P[r][c] x[grow(r)]    (warp = 16 columns)
// The panel is read straight into the MMA A fragments (for every lane group the
// 8 consecutive rows of one column, i.e. whole 32-byte sectors); the x operand is
// staged in shared memory; partial sums from the tiles of one cblk meet in
// global memory through atomics.  Up to 32 right-hand sides per pass.
namespace b200 {

constexpr int STT = 64;          // tile rows / columns
constexpr int SRHS = 32;         // right-hand sides per pass
constexpr int SXP = SRHS + 4;    // padded row of the staged x tile (conflict-free fragment reads)

__device__ __forceinline__ void dmma16x8x4(double (&c)[4], double a0, double a1, double b) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b));
}

template <typename T>
__global__ void __launch_bounds__(128) solve_tile_fwd_kernel(DevSym s, const SolveTile *__restrict__ tasks,
                                                             const T *__restrict__ L, const double *x,
                                                             double *b, int64_t ldx, int nrhs) {
    __shared__ double xs[STT * SXP];
    __shared__ int grows[STT];
    const SolveTile t = tasks[blockIdx.x];
    const int k = t.k, n = s.ncols[k], ld = s.ld[k];
    const int rows = min(STT, s.stride[k] - t.row0), cols = min(STT, n - t.col0);
    const T *P = L + s.off[k] + t.row0 + (size_t)t.col0 * ld;
    const double *xk = x + s.fcol[k] + t.col0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tg = lane & 3;
    if (tid < STT) grows[tid] = (tid < rows) ? panel_row_to_global(s, k, t.row0 + tid) : -1;
    const int r0w = warp * 16;
    const bool okA0 = (r0w + g) < rows, okA1 = (r0w + g + 8) < rows;
    for (int q0 = 0; q0 < nrhs; q0 += SRHS) {
        const int R = min(SRHS, nrhs - q0);
        __syncthreads();
        for (int idx = tid; idx < STT * SRHS; idx += blockDim.x) {
            const int c = idx % STT, j = idx / STT;
            xs[c * SXP + j] = (c < cols && j < R) ? xk[c + (size_t)(q0 + j) * ldx] : 0.0;
        }
        __syncthreads();
        const int ntn = (R + 7) >> 3;
        double acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[a][e] = 0.0;
        if (r0w < rows) {
#pragma unroll 4
            for (int kk = 0; kk < cols; kk += 4) {
                const int c = kk + tg;
                const bool okc = c < cols;
                const double a0 = (okA0 && okc) ? (double)P[(r0w + g) + (size_t)c * ld] : 0.0;
                const double a1 = (okA1 && okc) ? (double)P[(r0w + g + 8) + (size_t)c * ld] : 0.0;
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
                    if (nt < ntn) dmma16x8x4(acc[nt], a0, a1, xs[c * SXP + nt * 8 + g]);
            }
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                if (nt >= ntn) continue;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int r = r0w + g + (e >> 1) * 8;
                    const int j = nt * 8 + 2 * tg + (e & 1);
                    if (r < rows && j < R) atomicAdd(&b[grows[r] + (size_t)(q0 + j) * ldx], -acc[nt][e]);
                }
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(128) solve_tile_bwd_kernel(DevSym s, const SolveTile *__restrict__ tasks,
                                                             const T *__restrict__ L, const double *x,
                                                             double *b, int64_t ldx, int nrhs) {
    __shared__ double xg[STT * SXP];
    __shared__ int grows[STT];
    const SolveTile t = tasks[blockIdx.x];
    const int k = t.k, n = s.ncols[k], ld = s.ld[k];
    const int rows = min(STT, s.stride[k] - t.row0), cols = min(STT, n - t.col0);
    const T *P = L + s.off[k] + t.row0 + (size_t)t.col0 * ld;
    double *bk = b + s.fcol[k] + t.col0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tg = lane & 3;
    if (tid < STT) grows[tid] = (tid < rows) ? panel_row_to_global(s, k, t.row0 + tid) : -1;
    const int c0w = warp * 16;
    const bool okA0 = (c0w + g) < cols, okA1 = (c0w + g + 8) < cols;
    for (int q0 = 0; q0 < nrhs; q0 += SRHS) {
        const int R = min(SRHS, nrhs - q0);
        __syncthreads();
        for (int idx = tid; idx < STT * SRHS; idx += blockDim.x) {
            const int r = idx % STT, j = idx / STT;
            xg[r * SXP + j] = (r < rows && j < R) ? x[grows[r] + (size_t)(q0 + j) * ldx] : 0.0;
        }
        __syncthreads();
        const int ntn = (R + 7) >> 3;
        double acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[a][e] = 0.0;
        if (c0w < cols) {
#pragma unroll 4
            for (int kk = 0; kk < rows; kk += 4) {
                const int r = kk + tg;
                const bool okr = r < rows;
                const double a0 = (okA0 && okr) ? (double)P[r + (size_t)(c0w + g) * ld] : 0.0;
                const double a1 = (okA1 && okr) ? (double)P[r + (size_t)(c0w + g + 8) * ld] : 0.0;
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
                    if (nt < ntn) dmma16x8x4(acc[nt], a0, a1, xg[r * SXP + nt * 8 + g]);
            }
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                if (nt >= ntn) continue;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int c = c0w + g + (e >> 1) * 8;
                    const int j = nt * 8 + 2 * tg + (e & 1);
                    if (c < cols && j < R) atomicAdd(&bk[c + (size_t)(q0 + j) * ldx], -acc[nt][e]);
                }
            }
        }
    }
}

template <typename T>
void launch_solve_tiles(const DevSym &s, const SolveTile *tasks, int ntasks, const T *L, const double *x, double *b,
                        int64_t ldx, int nrhs, int backward, cudaStream_t st) {
    if (ntasks <= 0) return;
    if (!backward) solve_tile_fwd_kernel<T><<<ntasks, 128, 0, st>>>(s, tasks, L, x, b, ldx, nrhs);
    else solve_tile_bwd_kernel<T><<<ntasks, 128, 0, st>>>(s, tasks, L, x, b, ldx, nrhs);
}

template void launch_solve_tiles<double>(const DevSym &, const SolveTile *, int, const double *, const double *,
                                         double *, int64_t, int, int, cudaStream_t);
template void launch_solve_tiles<float>(const DevSym &, const SolveTile *, int, const float *, const double *,
                                        double *, int64_t, int, int, cudaStream_t);

}  // namespace b200

// ====================================================================== diagonal-block inverses
//
// W_k = T_k^{-1} for the lower-triangular diagonal block T_k of every cblk
// (L_kk, unit for LDL^T and LU; for the backward sweep of LU the stored U_kk^T).
// With W the diagonal solves of both sweeps are plain products, computed on
// tensor cores like the off-diagonal tiles, instead of a chain of dependent
// 32-column steps per cblk.  One CTA per cblk, 8 warps:
//   phase 1: every 32x32 diagonal tile inverted by one warp (row per lane);
//   phase 2: block column j of W by one warp: W_ij = -W_ii sum_{j<=m<i} T_im W_mj.
namespace b200 {

constexpr int IVP = 33;
constexpr int DIAG_INV_SMEM = 2 * 8 * 32 * IVP * sizeof(double);

template <typename T>
__global__ void __launch_bounds__(256) diag_inverse_kernel(DevSym s, const int *__restrict__ cblks,
                                                           const T *__restrict__ Lsrc, T *W,
                                                           const int64_t *__restrict__ woff, int unit) {
    extern __shared__ __align__(16) double inv_smem[];
    double *tl_all = inv_smem;                 // per warp: T tile, then W_mj tile
    double *wi_all = inv_smem + 8 * 32 * IVP;  // per warp: W_ii
    const int k = cblks[blockIdx.x];
    const int n = s.ncols[k], ld = s.ld[k];
    const T *Tk = Lsrc + s.off[k];
    T *Wk = W + woff[k];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = (n + 31) / 32;
    double *t = tl_all + warp * 32 * IVP;
    double *w = wi_all + warp * 32 * IVP;
    // phase 1: inverse of every diagonal 32x32 tile
    for (int b = warp; b < nb; b += 8) {
        const int b0 = b * 32, bw = min(32, n - b0);
        for (int idx = lane; idx < 32 * 32; idx += 32) {
            const int i = idx & 31, j = idx >> 5;
            t[i + j * IVP] = (i < bw && j < bw && i >= j) ? (double)Tk[(b0 + i) + (size_t)(b0 + j) * ld] : 0.0;
        }
        __syncwarp();
        // lane i computes row i of the inverse: W[i][i] = 1/T[i][i];
        // W[i][j] = -(1/T[i][i]) sum_{m=j}^{i-1} T[i][m] W[m][j]  (rows in order)
        for (int i = 0; i < bw; i++) {
            if (lane <= i) {
                const int j = lane;
                const double dii = unit ? 1.0 : t[i + i * IVP];
                double v;
                if (j == i) {
                    v = 1.0 / dii;
                } else {
                    double acc = 0.0;
                    for (int m = j; m < i; m++) acc += t[i + m * IVP] * w[m + j * IVP];
                    v = -acc / dii;
                }
                w[i + j * IVP] = v;
            }
            __syncwarp();
        }
        for (int idx = lane; idx < 32 * 32; idx += 32) {
            const int i = idx & 31, j = idx >> 5;
            if (i < bw && j < bw) Wk[(b0 + i) + (size_t)(b0 + j) * n] = (T)((i >= j) ? w[i + j * IVP] : 0.0);
        }
        __syncwarp();
    }
    __syncthreads();
    // phase 2: the blocks below the diagonal, one block column per warp
    for (int bj = warp; bj < nb; bj += 8) {
        const int j0 = bj * 32, jw = min(32, n - j0);
        // zero the strict upper blocks of this block column (W is lower triangular)
        for (int bi = 0; bi < bj; bi++) {
            const int i0 = bi * 32;
            for (int idx = lane; idx < 32 * jw; idx += 32) {
                const int i = idx & 31, j = idx >> 5;
                if (i0 + i < n) Wk[(i0 + i) + (size_t)(j0 + j) * n] = (T)0;
            }
        }
        for (int bi = bj + 1; bi < nb; bi++) {
            const int i0 = bi * 32, iw = min(32, n - i0);
            // acc (row = lane) = sum_{m = bj}^{bi-1} T[i0.., m0..] * W[m0.., j0..]
            double acc[32];
#pragma unroll
            for (int j = 0; j < 32; j++) acc[j] = 0.0;
            for (int bm = bj; bm < bi; bm++) {
                const int m0 = bm * 32, mw = min(32, n - m0);
                __syncwarp();
                for (int idx = lane; idx < 32 * 32; idx += 32) {
                    const int i = idx & 31, j = idx >> 5;
                    t[i + j * IVP] = (i < mw && j < jw) ? (double)Wk[(m0 + i) + (size_t)(j0 + j) * n] : 0.0;
                }
                __syncwarp();
                if (lane < iw) {
                    for (int m = 0; m < mw; m++) {
                        const double tv = (double)Tk[(i0 + lane) + (size_t)(m0 + m) * ld];
#pragma unroll
                        for (int j = 0; j < 32; j++) acc[j] += tv * t[m + j * IVP];
                    }
                }
            }
            __syncwarp();
            // W_ij = -W_ii acc : W_ii read back from the output (written in phase 1)
            for (int idx = lane; idx < 32 * 32; idx += 32) {
                const int i = idx & 31, j = idx >> 5;
                w[i + j * IVP] = (i < iw && j < iw) ? (double)Wk[(i0 + i) + (size_t)(i0 + j) * n] : 0.0;
            }
            // stage acc in t (row lane)
            __syncwarp();
#pragma unroll
            for (int j = 0; j < 32; j++) t[lane + j * IVP] = acc[j];
            __syncwarp();
            if (lane < iw) {
                double out[32];
#pragma unroll
                for (int j = 0; j < 32; j++) out[j] = 0.0;
                for (int m = 0; m <= lane; m++) {
                    const double wv = w[lane + m * IVP];
#pragma unroll
                    for (int j = 0; j < 32; j++) out[j] += wv * t[m + j * IVP];
                }
#pragma unroll
                for (int j = 0; j < 32; j++)
                    if (j < jw) Wk[(i0 + lane) + (size_t)(j0 + j) * n] = (T)(-out[j]);
            }
        }
    }
}

// x_out[k] = W_k x_in[k] (forward) or W_k^T x_in[k] (backward) for a 64-row tile
// of one cblk, on tensor cores; W is n x n column-major (ld = n), lower triangular.
template <typename T>
__global__ void __launch_bounds__(128) solve_diag_inv_kernel(DevSym s, const RowTask *__restrict__ tasks,
                                                             const T *__restrict__ W,
                                                             const int64_t *__restrict__ woff,
                                                             const double *__restrict__ xin, double *__restrict__ xout,
                                                             int64_t ldx, int nrhs, int backward) {
    __shared__ double xs[STT * SXP];
    const RowTask t = tasks[blockIdx.x];
    const int k = t.k, n = s.ncols[k];
    const int row0 = t.row0, rows = min(STT, n - row0);
    const T *Wk = W + woff[k];
    const double *in = xin + s.fcol[k];
    double *out = xout + s.fcol[k];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int r0w = warp * 16;
    const int ra = row0 + r0w + g, rb = ra + 8;
    const bool okA0 = (r0w + g) < rows, okA1 = (r0w + g + 8) < rows;
    // nonzero range of the product: forward columns [0, row0 + rows), backward [row0, n)
    const int cbeg = backward ? (row0 / STT) * STT : 0;
    const int cend = backward ? n : row0 + rows;
    for (int q0 = 0; q0 < nrhs; q0 += SRHS) {
        const int R = min(SRHS, nrhs - q0);
        const int ntn = (R + 7) >> 3;
        double acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[a][e] = 0.0;
        for (int c0 = cbeg; c0 < cend; c0 += STT) {
            const int cw = min(STT, cend - c0);
            __syncthreads();
            for (int idx = tid; idx < STT * SRHS; idx += blockDim.x) {
                const int c = idx % STT, j = idx / STT;
                xs[c * SXP + j] = (c < cw && j < R) ? in[c0 + c + (size_t)(q0 + j) * ldx] : 0.0;
            }
            __syncthreads();
            if (r0w < rows) {
#pragma unroll 4
                for (int kk = 0; kk < cw; kk += 4) {
                    const int c = c0 + kk + tg;
                    const bool okc = (kk + tg) < cw;
                    double a0 = 0.0, a1 = 0.0;
                    if (okc) {
                        if (!backward) {
                            if (okA0) a0 = (double)Wk[ra + (size_t)c * n];
                            if (okA1) a1 = (double)Wk[rb + (size_t)c * n];
                        } else {
                            if (okA0) a0 = (double)Wk[c + (size_t)ra * n];
                            if (okA1) a1 = (double)Wk[c + (size_t)rb * n];
                        }
                    }
#pragma unroll
                    for (int nt = 0; nt < 4; nt++)
                        if (nt < ntn) dmma16x8x4(acc[nt], a0, a1, xs[(kk + tg) * SXP + nt * 8 + g]);
                }
            }
        }
        if (r0w < rows) {
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                if (nt >= ntn) continue;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int r = r0w + g + (e >> 1) * 8;
                    const int j = nt * 8 + 2 * tg + (e & 1);
                    if (r < rows && j < R) out[row0 + r + (size_t)(q0 + j) * ldx] = acc[nt][e];
                }
            }
        }
    }
}

template <typename T>
void launch_diag_inverse(const DevSym &s, const int *cblks, int ncblk, const T *L, T *W, const int64_t *woff,
                         int unit, cudaStream_t st) {
    if (ncblk <= 0) return;
    diag_inverse_kernel<T><<<ncblk, 256, DIAG_INV_SMEM, st>>>(s, cblks, L, W, woff, unit);
}

template <typename T>
void launch_solve_diag_inv(const DevSym &s, const RowTask *tasks, int ntasks, const T *W, const int64_t *woff,
                           const double *xin, double *xout, int64_t ldx, int nrhs, int backward, cudaStream_t st) {
    if (ntasks <= 0) return;
    solve_diag_inv_kernel<T><<<ntasks, 128, 0, st>>>(s, tasks, W, woff, xin, xout, ldx, nrhs, backward);
}

int configure_inverse_kernels() {
    int rc = 0;
    rc |= (int)cudaFuncSetAttribute(diag_inverse_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    DIAG_INV_SMEM);
    rc |= (int)cudaFuncSetAttribute(diag_inverse_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    DIAG_INV_SMEM);
    return rc == 0 ? 0 : -1;
}

template void launch_diag_inverse<double>(const DevSym &, const int *, int, const double *, double *, const int64_t *,
                                          int, cudaStream_t);
template void launch_diag_inverse<float>(const DevSym &, const int *, int, const float *, float *, const int64_t *,
                                         int, cudaStream_t);
template void launch_solve_diag_inv<double>(const DevSym &, const RowTask *, int, const double *, const int64_t *,
                                            const double *, double *, int64_t, int, int, cudaStream_t);
template void launch_solve_diag_inv<float>(const DevSym &, const RowTask *, int, const float *, const int64_t *,
                                           const double *, double *, int64_t, int, int, cudaStream_t);

}  // namespace b200

// W_k for cblks of at most 32 columns: the diagonal kernel already stored the
// inverse of their single 32x32 tile (and, for LU, of the stored U^T) in the
// tile-inverse store; copy it to the n x n layout of the solves.
namespace b200 {

template <typename T>
__global__ void copy_tile_inverse_kernel(DevSym s, const int *__restrict__ cblks, const T *__restrict__ tinv,
                                         const int64_t *__restrict__ toff, T *W, const int64_t *__restrict__ woff,
                                         int which) {
    const int k = cblks[blockIdx.x];
    const int n = s.ncols[k];
    const T *src = tinv + toff[k] + (which ? 32 * n : 0);
    T *dst = W + woff[k];
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;
        dst[idx] = (i >= j) ? src[i + j * 32] : (T)0;
    }
}

template <typename T>
void launch_copy_tile_inverse(const DevSym &s, const int *cblks, int ncblk, const T *tinv, const int64_t *toff, T *W,
                              const int64_t *woff, int which, cudaStream_t st) {
    if (ncblk <= 0) return;
    copy_tile_inverse_kernel<T><<<ncblk, 128, 0, st>>>(s, cblks, tinv, toff, W, woff, which);
}

template void launch_copy_tile_inverse<double>(const DevSym &, const int *, int, const double *, const int64_t *,
                                               double *, const int64_t *, int, cudaStream_t);
template void launch_copy_tile_inverse<float>(const DevSym &, const int *, int, const float *, const int64_t *,
                                              float *, const int64_t *, int, cudaStream_t);

}  // namespace b200
