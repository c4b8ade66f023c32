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
#include "tile_ops.cuh"

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
// The off-diagonal and diagonal-inverse products of the supernodal solves as
// small GEMMs on FP64 tensor cores (DMMA m16n8k4), one CTA (4 warps) per 64 x 64
// tile of the factor (or of a diagonal-block inverse W) times up to 32 right-hand
// sides per pass:
//   OFF_FWD : b[grow(r)] -= sum_c P[r][c] x_k[c]     (solve_blok_zgemm forward,
//             kernels/solve_ztrsmsp.c:275-280; warp = 16 rows)
//   OFF_BWD : b_k[c]     -= sum_r P[r][c] x[grow(r)] (backward; warp = 16 columns)
//   DIAG_FWD: out_k[r]    = sum_c W[r][c] in_k[c]     (W = L_kk^{-1}, lower)
//   DIAG_BWD: out_k[c]    = sum_r W[r][c] in_k[r]     (W^T, upper)
// The factor tile is staged in shared memory with cp.async (every load of the tile
// in flight at once, zero fill outside the panel) and the diagonal products run a
// double-buffered pipeline over 64-column chunks, so a tile costs about one memory
// latency; partial sums of the off-diagonal tiles of one cblk meet in global
// memory through atomics.
namespace b200 {

constexpr int STT = 64;          // tile rows / columns
constexpr int SRHS = 32;         // right-hand sides per pass
constexpr int SXP = SRHS + 4;    // padded row of the staged x tile (conflict-free fragment reads)
constexpr int SM_FWD = 72;       // pitch of a staged tile read row-wise by the fragments
constexpr int SM_BWD = 68;       // pitch of a staged tile read column-wise
enum { OFF_FWD = 0, OFF_BWD = 1, DIAG_FWD = 2, DIAG_BWD = 3 };

__device__ __forceinline__ void dmma16x8x4(double (&c)[4], double a0, double a1, double b) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b));
}

__device__ __forceinline__ unsigned sm_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
template <typename T>
__device__ __forceinline__ void cp_async_el(T *dst, const T *src, bool ok) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sm_addr(dst)), "l"(src), "n"(sizeof(T)),
                 "r"(ok ? (int)sizeof(T) : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Stage M[gr0 + r][gc0 + c] (column-major, leading dimension ldm, nr x nc valid) as
// ms[c * PM + r] for r, c < 64; zeros outside.  Warp w takes columns w, w + 4, ...
// and its lanes rows lane and lane + 32: consecutive lanes read consecutive rows.
template <typename T, int PM>
__device__ __forceinline__ void stage_tile(T *ms, const T *M, int64_t ldm, int gr0, int gc0, int nr, int nc) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const bool r0ok = gr0 + lane < nr, r1ok = gr0 + lane + 32 < nr;
    const T *col = M + gr0 + lane + (size_t)(gc0 + w) * ldm;
    for (int c = w; c < STT; c += nw, col += (size_t)nw * ldm) {
        const bool cok = gc0 + c < nc;
        cp_async_el(ms + c * PM + lane, (cok && r0ok) ? col : M, cok && r0ok);
        cp_async_el(ms + c * PM + lane + 32, (cok && r1ok) ? col + 32 : M, cok && r1ok);
    }
}

// x tile: xs[i * SXP + j] = xv[i][q0 + j] for i < ni, j < R (zeros elsewhere); rows
// either contiguous from xv (rowmap null) or gathered through rowmap.
__device__ __forceinline__ void stage_x(double *xs, const double *xv, const int *rowmap, int ni, int64_t ldx, int q0,
                                        int R) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int i0 = lane, i1 = lane + 32;
    const bool ok0 = i0 < ni, ok1 = i1 < ni;
    const double *x0 = xv + (ok0 ? (rowmap ? rowmap[i0] : i0) : 0);
    const double *x1 = xv + (ok1 ? (rowmap ? rowmap[i1] : i1) : 0);
    for (int j = w; j < SRHS; j += nw) {
        const bool jok = j < R;
        cp_async_el(xs + i0 * SXP + j, x0 + (size_t)(q0 + j) * ldx, jok && ok0);
        cp_async_el(xs + i1 * SXP + j, x1 + (size_t)(q0 + j) * ldx, jok && ok1);
    }
}

// D += A B with A 16 x 16 (a[2j], a[2j+1] = rows g, g + 8 of column 4j + tg), B 16 x 8
// (b[j] = row 4j + tg, column g), the fragment layout of four m16n8k4 steps.
__device__ __forceinline__ void dmma16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
          "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// acc += M_tile(op) x_tile over 64 K values; ROW = 1: output index = tile row
// (a fragment reads ms[k * PM + out]), ROW = 0: output index = tile column
// (ms[out * PM + k]).
template <typename T, int PM, int ROW>
__device__ __forceinline__ void tile_mma(double (&acc)[4][4], const T *ms, const double *xs, int o0w, int ntn) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
#pragma unroll 2
    for (int kk = 0; kk < STT; kk += 16) {
        double a[8];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int kq = kk + 4 * j + tg;
            a[2 * j] = ROW ? (double)ms[kq * PM + o0w + g] : (double)ms[(o0w + g) * PM + kq];
            a[2 * j + 1] = ROW ? (double)ms[kq * PM + o0w + g + 8] : (double)ms[(o0w + g + 8) * PM + kq];
        }
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            if (nt < ntn) {
                double b[4];
#pragma unroll
                for (int j = 0; j < 4; j++) b[j] = xs[(kk + 4 * j + tg) * SXP + nt * 8 + g];
                dmma16x8x16(acc[nt], a, b);
            }
        }
    }
}

template <typename T, int MODE>
struct SolveSmem {
    static constexpr int PM = (MODE == OFF_FWD || MODE == DIAG_FWD) ? SM_FWD : SM_BWD;
    static constexpr int BYTES = STT * PM * (int)sizeof(T) + STT * SXP * 8;
};

// One 64 x 64 tile times up to 32 right-hand sides per pass.  Task {k, row0, col0}:
//   OFF_*  : panel rows [row0, row0 + 64) x columns [col0, col0 + 64) of cblk k
//   DIAG_* : output tile [row0, row0 + 64) of cblk k, K chunk [col0, col0 + 64) of
//            W_k (forward) or W_k^T (backward); the output (zeroed before the sweep)
//            accumulates the chunks through atomics.
template <typename T, int MODE>
__global__ void __launch_bounds__(128) solve_mm_kernel(DevSym s, const SolveTile *__restrict__ tasks,
                                                       const T *__restrict__ M, const int64_t *__restrict__ woff,
                                                       const double *xin, double *out, int64_t ldx, int nrhs) {
    using SS = SolveSmem<T, MODE>;
    constexpr int PM = SS::PM;
    constexpr bool ROW = (MODE == OFF_FWD || MODE == DIAG_FWD);
    extern __shared__ __align__(16) unsigned char sv_smem[];
    T *ms = reinterpret_cast<T *>(sv_smem);
    double *xs = reinterpret_cast<double *>(sv_smem + STT * PM * sizeof(T));
    __shared__ int rmap[STT];
    const SolveTile t = tasks[blockIdx.x];
    const int k = t.k, n = s.ncols[k];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int o0w = warp * 16;  // this warp's 16 outputs of the tile
    int nout;
    const double *xsrc;
    const int *xmap = nullptr;
    int nk;
    if (MODE == OFF_FWD || MODE == OFF_BWD) {
        const int rows = min(STT, s.stride[k] - t.row0), cols = min(STT, n - t.col0);
        if (tid < STT) rmap[tid] = (tid < rows) ? panel_row_to_global(s, k, t.row0 + tid) : 0;
        __syncthreads();
        stage_tile<T, PM>(ms, M + s.off[k], s.ld[k], t.row0, t.col0, s.stride[k], n);
        nout = ROW ? rows : cols;
        nk = ROW ? cols : rows;
        if (MODE == OFF_FWD) xsrc = xin + s.fcol[k] + t.col0;
        else { xsrc = xin; xmap = rmap; }
    } else {
        const T *Wk = M + woff[k];
        nout = min(STT, n - t.row0);
        nk = min(STT, n - t.col0);
        if (MODE == DIAG_FWD) stage_tile<T, PM>(ms, Wk, n, t.row0, t.col0, n, n);  // W[o][k]
        else stage_tile<T, PM>(ms, Wk, n, t.col0, t.row0, n, n);                   // W[k][o]
        xsrc = xin + s.fcol[k] + t.col0;
    }
    for (int q0 = 0; q0 < nrhs; q0 += SRHS) {
        const int R = min(SRHS, nrhs - q0), ntn = (R + 7) >> 3;
        if (q0 > 0) __syncthreads();
        stage_x(xs, xsrc, xmap, nk, ldx, q0, R);
        cp_commit();
        cp_wait<0>();
        __syncthreads();
        if (o0w < nout) {
            double acc[4][4] = {};
            tile_mma<T, PM, ROW>(acc, ms, xs, o0w, ntn);
            const double sg = (MODE == OFF_FWD || MODE == OFF_BWD) ? -1.0 : 1.0;
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                if (nt >= ntn) continue;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int o = o0w + g + (e >> 1) * 8;
                    const int j = nt * 8 + 2 * tg + (e & 1);
                    if (o < nout && j < R) {
                        double *dst = (MODE == OFF_FWD)   ? out + rmap[o]
                                      : (MODE == OFF_BWD) ? out + s.fcol[k] + t.col0 + o
                                                          : out + s.fcol[k] + t.row0 + o;
                        atomicAdd(dst + (size_t)(q0 + j) * ldx, sg * acc[nt][e]);
                    }
                }
            }
        }
    }
}

// Cblks of at most 32 columns, one warp each: the diagonal-block product and the
// off-diagonal rows of one sweep in a single pass (the bottom levels of the tree
// hold thousands of such cblks, far smaller than a 64 x 64 tile).
//   forward : aux_k = W_k x_k; x[grow(r)] -= P[r][:] aux_k  (lane = row)
//   backward: t = aux_k - P^T x[grow(rows)] (lane = column); x_k = W_k^T t
// W_k is the inverse of the diagonal block (n x n, column-major), P the cblk panel.
constexpr int LEAF_R = 16;  // right-hand sides per pass

template <typename T>
__global__ void __launch_bounds__(128) solve_leaf_kernel(DevSym s, const int *__restrict__ cblks, int ncblk,
                                                         const T *__restrict__ P, const T *__restrict__ W,
                                                         const int64_t *__restrict__ woff, double *x, double *aux,
                                                         int64_t ldx, int nrhs, int backward) {
    __shared__ double ys[4][32][LEAF_R + 1];
    __shared__ double xr[4][32][LEAF_R + 1];
    __shared__ int gr[4][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ci = blockIdx.x * 4 + w;
    if (ci >= ncblk) return;
    const int k = cblks[ci];
    const int n = s.ncols[k], ld = s.ld[k], stride = s.stride[k], f0 = s.fcol[k];
    const T *Pk = P + s.off[k];
    const T *Wk = W + woff[k];
    for (int q0 = 0; q0 < nrhs; q0 += LEAF_R) {
        const int R = min(LEAF_R, nrhs - q0);
        if (!backward) {
#pragma unroll
            for (int j = 0; j < LEAF_R; j++)
                ys[w][lane][j] = (lane < n && j < R) ? x[f0 + lane + (size_t)(q0 + j) * ldx] : 0.0;
            __syncwarp();
            double y[LEAF_R];
#pragma unroll
            for (int j = 0; j < LEAF_R; j++) y[j] = 0.0;
            if (lane < n) {
                for (int c = 0; c <= lane; c++) {
                    const double wv = (double)Wk[lane + (size_t)c * n];
#pragma unroll
                    for (int j = 0; j < LEAF_R; j++) y[j] += wv * ys[w][c][j];
                }
            }
            __syncwarp();
            if (lane < n) {
#pragma unroll
                for (int j = 0; j < LEAF_R; j++) {
                    ys[w][lane][j] = y[j];
                    if (j < R) aux[f0 + lane + (size_t)(q0 + j) * ldx] = y[j];
                }
            }
            __syncwarp();
            for (int r = n + lane; r < stride; r += 32) {
                const int g = panel_row_to_global(s, k, r);
                double acc[LEAF_R];
#pragma unroll
                for (int j = 0; j < LEAF_R; j++) acc[j] = 0.0;
                for (int c = 0; c < n; c++) {
                    const double pv = (double)Pk[r + (size_t)c * ld];
#pragma unroll
                    for (int j = 0; j < LEAF_R; j++) acc[j] += pv * ys[w][c][j];
                }
#pragma unroll
                for (int j = 0; j < LEAF_R; j++)
                    if (j < R) atomicAdd(&x[g + (size_t)(q0 + j) * ldx], -acc[j]);
            }
            __syncwarp();
        } else {
            double t[LEAF_R];
#pragma unroll
            for (int j = 0; j < LEAF_R; j++) t[j] = (lane < n && j < R) ? aux[f0 + lane + (size_t)(q0 + j) * ldx] : 0.0;
            for (int r0 = n; r0 < stride; r0 += 32) {
                const int nr = min(32, stride - r0);
                gr[w][lane] = (lane < nr) ? panel_row_to_global(s, k, r0 + lane) : 0;
                __syncwarp();
                // stage x of the 32 rows: xr[i][j] = x[grow(r0 + i)][q0 + j]
                for (int idx = lane; idx < 32 * LEAF_R; idx += 32) {
                    const int i = idx / LEAF_R, j = idx % LEAF_R;
                    xr[w][i][j] = (i < nr && j < R) ? x[gr[w][i] + (size_t)(q0 + j) * ldx] : 0.0;
                }
                __syncwarp();
                if (lane < n) {
                    for (int i = 0; i < nr; i++) {
                        const double pv = (double)Pk[r0 + i + (size_t)lane * ld];
#pragma unroll
                        for (int j = 0; j < LEAF_R; j++) t[j] -= pv * xr[w][i][j];
                    }
                }
                __syncwarp();
            }
            if (lane < n) {
#pragma unroll
                for (int j = 0; j < LEAF_R; j++) ys[w][lane][j] = t[j];
            }
            __syncwarp();
            if (lane < n) {
                double o[LEAF_R];
#pragma unroll
                for (int j = 0; j < LEAF_R; j++) o[j] = 0.0;
                for (int r = lane; r < n; r++) {
                    const double wv = (double)Wk[r + (size_t)lane * n];
#pragma unroll
                    for (int j = 0; j < LEAF_R; j++) o[j] += wv * ys[w][r][j];
                }
#pragma unroll
                for (int j = 0; j < LEAF_R; j++)
                    if (j < R) x[f0 + lane + (size_t)(q0 + j) * ldx] = o[j];
            }
            __syncwarp();
        }
    }
}

template <typename T>
void launch_solve_leaf(const DevSym &s, const int *cblks, int ncblk, const T *P, const T *W, const int64_t *woff,
                       double *x, double *aux, int64_t ldx, int nrhs, int backward, cudaStream_t st) {
    if (ncblk <= 0) return;
    solve_leaf_kernel<T><<<(ncblk + 3) / 4, 128, 0, st>>>(s, cblks, ncblk, P, W, woff, x, aux, ldx, nrhs, backward);
}
template void launch_solve_leaf<double>(const DevSym &, const int *, int, const double *, const double *,
                                        const int64_t *, double *, double *, int64_t, int, int, cudaStream_t);
template void launch_solve_leaf<float>(const DevSym &, const int *, int, const float *, const float *,
                                       const int64_t *, double *, double *, int64_t, int, int, cudaStream_t);

template <typename T>
void launch_solve_tiles(const DevSym &s, const SolveTile *tasks, int ntasks, const T *L, const double *x, double *b,
                        int64_t ldx, int nrhs, int backward, cudaStream_t st) {
    if (ntasks <= 0) return;
    if (!backward)
        solve_mm_kernel<T, OFF_FWD><<<ntasks, 128, SolveSmem<T, OFF_FWD>::BYTES, st>>>(s, tasks, L, nullptr, x, b, ldx,
                                                                                     nrhs);
    else
        solve_mm_kernel<T, OFF_BWD><<<ntasks, 128, SolveSmem<T, OFF_BWD>::BYTES, st>>>(s, tasks, L, nullptr, x, b, ldx,
                                                                                     nrhs);
}

template <typename T, int MODE>
void solve_diag_mm(const DevSym &s, const SolveTile *tasks, int ntasks, const T *W, const int64_t *woff,
                   const double *xin, double *xout, int64_t ldx, int nrhs, cudaStream_t st) {
    solve_mm_kernel<T, MODE><<<ntasks, 128, SolveSmem<T, MODE>::BYTES, st>>>(s, tasks, W, woff, xin, xout, ldx, nrhs);
}

// dynamic shared memory of the staged solve kernels (above the 48 KB default)
template <typename T>
int configure_solve_mm() {
    int rc = 0;
    rc |= (int)cudaFuncSetAttribute(solve_mm_kernel<T, OFF_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SolveSmem<T, OFF_FWD>::BYTES);
    rc |= (int)cudaFuncSetAttribute(solve_mm_kernel<T, OFF_BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SolveSmem<T, OFF_BWD>::BYTES);
    rc |= (int)cudaFuncSetAttribute(solve_mm_kernel<T, DIAG_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SolveSmem<T, DIAG_FWD>::BYTES);
    rc |= (int)cudaFuncSetAttribute(solve_mm_kernel<T, DIAG_BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SolveSmem<T, DIAG_BWD>::BYTES);
    return rc;
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

constexpr int INV_WARPS = 4;
constexpr int DIAG_INV_SMEM = INV_WARPS * 2 * 32 * TP * sizeof(double);

// W_k = T_k^{-1} for the lower-triangular diagonal block T_k of every listed cblk
// (L_kk, unit for LDL^T and LU; for the backward sweep of LU the stored U_kk^T).
// With W the diagonal solves of both sweeps are plain products on tensor cores.
// One CTA of 4 warps per cblk, 32 x 32 blocks:
//   phase 1: every diagonal block inverted by one warp (invert_lower_tile);
//   phase 2: block rows in order, the blocks of a row in parallel over the warps:
//            W_ij = -W_ii sum_{j <= m < i} T_im W_mj, each product from shared-memory
//            copies of T_im and W_mj staged with all loads in flight.
template <typename T>
__global__ void __launch_bounds__(128) diag_inverse_kernel(DevSym s, const int *__restrict__ cblks,
                                                           const T *__restrict__ Lsrc, T *W,
                                                           const int64_t *__restrict__ woff, int unit) {
    extern __shared__ __align__(16) double inv_smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *ta = inv_smem + warp * 2 * 32 * TP;
    double *tb = ta + 32 * TP;
    const int k = cblks[blockIdx.x];
    const int n = s.ncols[k], ld = s.ld[k];
    const T *Tk = Lsrc + s.off[k];
    T *Wk = W + woff[k];
    const int nb = (n + 31) / 32;
    // phase 1: diagonal blocks; the blocks above them are zero
    for (int b = warp; b < nb; b += INV_WARPS) {
        const int b0 = b * 32, bw = min(32, n - b0);
        for (int idx = lane; idx < 32 * 32; idx += 32) {
            const int i = idx & 31, j = idx >> 5;
            ta[i + j * TP] = (i < bw && j < bw && i >= j) ? (double)Tk[(b0 + i) + (size_t)(b0 + j) * ld] : 0.0;
        }
        __syncwarp();
        invert_lower_tile<double>(ta, tb, bw, lane, unit, 0);
        for (int idx = lane; idx < 32 * bw; idx += 32) {
            const int i = idx & 31, j = idx >> 5;
            if (i < bw) Wk[(b0 + i) + (size_t)(b0 + j) * n] = (T)tb[i + j * TP];
        }
        for (int idx = lane; idx < b0 * bw; idx += 32) {
            const int i = idx % b0, j = idx / b0;
            Wk[i + (size_t)(b0 + j) * n] = (T)0;
        }
        __syncwarp();
    }
    __syncthreads();
    // phase 2
    for (int bi = 1; bi < nb; bi++) {
        const int i0 = bi * 32, iw = min(32, n - i0);
        for (int bj = warp; bj < bi; bj += INV_WARPS) {
            const int j0 = bj * 32, jw = min(32, n - j0);
            double acc[32];
#pragma unroll
            for (int j = 0; j < 32; j++) acc[j] = 0.0;
            for (int bm = bj; bm < bi; bm++) {
                const int m0 = bm * 32, mw = min(32, n - m0);
                for (int idx = lane; idx < 32 * 32; idx += 32) {
                    const int i = idx & 31, j = idx >> 5;
                    ta[i + j * TP] = (i < iw && j < mw) ? (double)Tk[(i0 + i) + (size_t)(m0 + j) * ld] : 0.0;
                    tb[i + j * TP] = (i < mw && j < jw) ? (double)Wk[(m0 + i) + (size_t)(j0 + j) * n] : 0.0;
                }
                __syncwarp();
#pragma unroll 4
                for (int m = 0; m < 32; m++) {
                    const double tv = ta[lane + m * TP];
#pragma unroll
                    for (int j = 0; j < 32; j++) acc[j] += tv * tb[m + j * TP];
                }
                __syncwarp();
            }
            // W_ij = -W_ii acc (W_ii written in phase 1)
            for (int idx = lane; idx < 32 * 32; idx += 32) {
                const int i = idx & 31, j = idx >> 5;
                tb[i + j * TP] = (i < iw && j < iw && i >= j) ? (double)Wk[(i0 + i) + (size_t)(i0 + j) * n] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 32; j++) ta[lane + j * TP] = acc[j];
            __syncwarp();
            if (lane < iw) {
                double out[32];
#pragma unroll
                for (int j = 0; j < 32; j++) out[j] = 0.0;
                for (int l = 0; l <= lane; l++) {
                    const double wv = tb[lane + l * TP];
#pragma unroll
                    for (int j = 0; j < 32; j++) out[j] -= wv * ta[l + j * TP];
                }
#pragma unroll
                for (int j = 0; j < 32; j++)
                    if (j < jw) Wk[(i0 + lane) + (size_t)(j0 + j) * n] = (T)out[j];
            }
            __syncwarp();
        }
        __syncthreads();
    }
}

template <typename T>
void launch_diag_inverse(const DevSym &s, const int *cblks, int ncblk, const T *L, T *W, const int64_t *woff,
                         int unit, cudaStream_t st) {
    if (ncblk <= 0) return;
    diag_inverse_kernel<T><<<ncblk, 32 * INV_WARPS, DIAG_INV_SMEM, st>>>(s, cblks, L, W, woff, unit);
}

template <typename T>
void launch_solve_diag_inv(const DevSym &s, const SolveTile *tasks, int ntasks, const T *W, const int64_t *woff,
                           const double *xin, double *xout, int64_t ldx, int nrhs, int backward, cudaStream_t st) {
    if (ntasks <= 0) return;
    if (!backward) solve_diag_mm<T, DIAG_FWD>(s, tasks, ntasks, W, woff, xin, xout, ldx, nrhs, st);
    else solve_diag_mm<T, DIAG_BWD>(s, tasks, ntasks, W, woff, xin, xout, ldx, nrhs, st);
}

int configure_inverse_kernels() {
    int rc = configure_solve_mm<double>() | configure_solve_mm<float>();
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
template void launch_solve_diag_inv<double>(const DevSym &, const SolveTile *, int, const double *, const int64_t *,
                                            const double *, double *, int64_t, int, int, cudaStream_t);
template void launch_solve_diag_inv<float>(const DevSym &, const SolveTile *, int, const float *, const int64_t *,
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
