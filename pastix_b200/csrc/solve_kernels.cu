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
                const int rest = n - cb - w;
                for (int idx = tid; idx < rest * R; idx += blockDim.x) {
                    const int i = cb + w + idx % rest, r = idx / rest;
                    double acc = 0.0;
                    for (int c = 0; c < w; c++) acc += (double)D[i + (size_t)(cb + c) * ld] * bs[cb + c + r * n];
                    bs[i + r * n] -= acc;
                }
                __syncthreads();
            }
        } else {
            for (int cb = ((n - 1) / 32) * 32; cb >= 0; cb -= 32) {
                const int w = min(32, n - cb);
                for (int task = warp; task < w * R; task += nw) {
                    const int c = task % w, r = task / w;
                    double acc = 0.0;
                    for (int i = cb + w + lane; i < n; i += 32) acc += (double)D[i + (size_t)(cb + c) * ld] * bs[i + r * n];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                    if (lane == 0) bs[cb + c + r * n] -= acc;
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
