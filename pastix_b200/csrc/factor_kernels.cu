// Numerical factorization kernels (sm_100a).
//
//  scatter_kernel      bcsc -> panel arena (cpucblk_zfillin_fr, kernels/cpucblk_zinit.c:229-309)
//  diag_factor_kernel  per-cblk diagonal-block POTRF / GETRF / SYTRF with static pivoting
//                      (core_z{potrf,getrf,sytrf}sp, kernels/core_z*trfsp.c)
//  panel_trsm_kernel   off-diagonal panel solve (core_ztrsmsp_2d, kernels/core_ztrsmsp.c:147-181)
//  update_f64_kernel   GEMM + scatter-add into the facing cblk on FP64 tensor cores (DMMA)
//                      (core_zgemmsp_2d2d, kernels/core_zgemmsp.c:396-465)
//  update_simt_kernel  the same update for FP32 factors on CUDA cores
#include "b200_internal.h"
#include "kernels.h"
#include "tile_ops.cuh"

#include <algorithm>

namespace b200 {

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// 8-byte asynchronous global->shared copy; src_bytes = 0 fills zeros.
__device__ __forceinline__ void cp_async8(void *dst, const void *src, bool ok) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(ok ? 8 : 0));
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src, bool ok) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(ok ? 4 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ------------------------------------------------------------------ scatter

template <typename T>
__global__ void scatter_kernel(int64_t nnz, const int64_t *__restrict__ dest, const double *__restrict__ Lv,
                               const double *__restrict__ Uv, T *__restrict__ L, T *__restrict__ U) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    int64_t d = dest[e];
    if (d < 0) return;
    const bool strict = (d >> 62) & 1;
    d &= ((int64_t)1 << 62) - 1;
    L[d] = (T)Lv[e];
    if (U != nullptr && strict) U[d] = (T)Uv[e];
}

// ------------------------------------------------------------------ diagonal blocks


// Unblocked factorization of a pb x pb tile by one warp, held in registers: lane
// i owns row i (r[j] = t[i][j]), columns are broadcast with warp shuffles.
// POTRF: core_zpotf2sp (kernels/core_zpotrfsp.c:66-100)
// GETRF: core_zgetf2sp (kernels/core_zgetrfsp.c:64-110)
// SYTRF: core_zsytf2sp (kernels/core_zsytrfsp.c:63-103)
// The reciprocal of each pivot comes from rsqrt (POTRF) or one division computed
// beside the pivot, off the critical path of the trailing updates.  Every register
// index is a compile-time constant (static_for): a column loop left rolled by the
// compiler would move r[] to local memory (four times slower on a 32 x 32 tile).
// NB >= pb bounds the columns (8, 16 or 32): a narrow tile skips the padding.
template <typename T, int FACTO, int NB = 32>
__device__ void factor_tile(T *t, int pb, int lane, double thr, int *piv, int *err) {
    T r[NB];
    static_for<NB>([&](auto jj) {
        constexpr int j = decltype(jj)::value;
        r[j] = t[lane + j * TP];
    });
    const bool row_in = lane < pb;
    // Columns >= pb run too (no branch, so the compiler can overlap consecutive
    // columns): they only touch padding rows (lane >= pb) and count nothing.
    static_for<NB>([&](auto cc) {
        constexpr int c = decltype(cc)::value;
        const bool col_in = c < pb;
        T a = __shfl_sync(0xffffffffu, r[c], c);
        const bool rep = fabs((double)a) < thr;
        if (rep) a = (FACTO == FACTO_POTRF) ? (T)thr : ((a < (T)0) ? (T)(-thr) : (T)thr);
        bool neg = false;
        T d, inv;
        if (FACTO == FACTO_POTRF) {
            if (a < (T)0) { neg = true; a = -a; }
            d = sqrt(a);
            inv = rsqrt(a);
        } else {
            d = a;
            inv = (T)1 / a;
        }
        if (lane == 0 && col_in) {
            if (rep) (*piv)++;
            if (neg) *err = 1;
        }
        const bool below = lane > c && row_in;
        if (lane == c) r[c] = d;
        if (below) {
            if (FACTO == FACTO_SYTRF) t[c + lane * TP] = r[c];  // D L^T copy in the upper part
            r[c] *= inv;
        }
        const T li = r[c];
        if (FACTO == FACTO_GETRF) {
            static_for<NB>([&](auto jj) {
                constexpr int j = decltype(jj)::value;
                if constexpr (j > c) {
                    const T ucj = __shfl_sync(0xffffffffu, r[j], c);  // row c of U
                    if (below && j < pb) r[j] -= li * ucj;
                }
            });
        } else {
            const T m = (FACTO == FACTO_SYTRF) ? -d * li : li;
            static_for<NB>([&](auto jj) {
                constexpr int j = decltype(jj)::value;
                if constexpr (j > c) {
                    const T lj = __shfl_sync(0xffffffffu, r[c], j);  // l_j
                    if (below && j <= lane) {
                        if (FACTO == FACTO_SYTRF) r[j] += m * lj;
                        else r[j] -= m * lj;
                    }
                }
            });
        }
    });
    __syncwarp();
    static_for<NB>([&](auto jj) {
        constexpr int j = decltype(jj)::value;
        // LDL^T keeps the D L^T copies of the upper part written above
        if (FACTO != FACTO_SYTRF || j <= lane) t[lane + j * TP] = r[j];
    });
    __syncwarp();
}

// 32x32 output tile of a trailing update, computed by one warp:
// C[i][j] -= sum_c X[i][c] * B(j, c) for c < pb, where X(i, c) = A[(r0+i) + (p+c) ld]
// and B(j, c) = A[(c0+j) + (p+c) ld] (btrans = 0) or A[(p+c) + (c0+j) ld] (btrans = 1).
__device__ __forceinline__ void dmma_tile(double (&c)[4], double a0, double a1, double b) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b));
}

__device__ void warp_tile_update(double *A, int ld, int n, int p, int pb, int r0, int c0, int btrans, int lower_only,
                                 int lane, double *) {
    const int g = lane >> 2, tg = lane & 3;
    double acc[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[mi][ni][e] = 0.0;
    for (int kk = 0; kk < pb; kk += 4) {
        const int c = kk + tg;
        const bool okc = c < pb;
        double a[2][2], b[4];
#pragma unroll
        for (int mi = 0; mi < 2; mi++) {
            const int ra = r0 + mi * 16 + g, rb = ra + 8;
            a[mi][0] = (okc && ra < n) ? A[ra + (size_t)(p + c) * ld] : 0.0;
            a[mi][1] = (okc && rb < n) ? A[rb + (size_t)(p + c) * ld] : 0.0;
        }
#pragma unroll
        for (int ni = 0; ni < 4; ni++) {
            const int j = c0 + ni * 8 + g;
            b[ni] = (okc && j < n) ? (btrans ? A[(p + c) + (size_t)j * ld] : A[j + (size_t)(p + c) * ld]) : 0.0;
        }
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int ni = 0; ni < 4; ni++) dmma_tile(acc[mi][ni], a[mi][0], a[mi][1], b[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int i = r0 + mi * 16 + g + (e >> 1) * 8;
                const int j = c0 + ni * 8 + 2 * tg + (e & 1);
                if (i < n && j < n && (!lower_only || i >= j)) A[i + (size_t)j * ld] -= acc[mi][ni][e];
            }
}

// FP32 version: lane i owns row r0+i of the tile; B staged in per-warp shared memory.
__device__ void warp_tile_update(float *A, int ld, int n, int p, int pb, int r0, int c0, int btrans, int lower_only,
                                 int lane, float *bs) {
    for (int idx = lane; idx < 32 * 32; idx += 32) {
        const int j = idx & 31, c = idx >> 5;
        float v = 0.0f;
        if (c < pb && c0 + j < n) v = btrans ? A[(p + c) + (size_t)(c0 + j) * ld] : A[(c0 + j) + (size_t)(p + c) * ld];
        bs[c * 33 + j] = v;
    }
    __syncwarp();
    const int i = r0 + lane;
    float acc[32];
#pragma unroll
    for (int j = 0; j < 32; j++) acc[j] = 0.0f;
    if (i < n) {
        for (int c = 0; c < pb; c++) {
            const float x = A[i + (size_t)(p + c) * ld];
#pragma unroll
            for (int j = 0; j < 32; j++) acc[j] = fmaf(x, bs[c * 33 + j], acc[j]);
        }
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const int jj = c0 + j;
            if (jj < n && (!lower_only || i >= jj)) A[i + (size_t)jj * ld] -= acc[j];
        }
    }
    __syncwarp();
}

// One CTA (256 threads) factors the diagonal block of one cblk, blocked by 32
// columns.  Per panel: warp 0 factors the 32x32 diagonal tile in registers and then
// inverts it (warp 1 inverts the upper triangle for LU); the rows (and, for LU,
// columns) below the tile inside the diagonal block are solved as products with
// those inverses; every warp then updates its own 32x32 tiles of the trailing
// block (FP64 tensor cores for double).  The tile inverses are also stored in
// tinv for the panel TRSM.  For LU the diagonal block of the U arena is first
// added transposed into L (core_zgeadd) and afterwards receives the transposed
// factor (core_zgetmo).  At most 128 registers per thread, so that two CTAs share an
// SM: the levels of many 33-96 column cblks are latency-bound, and the second CTA's
// warps cover the first one's single-warp tile steps (the spills this costs are
// cheaper than the idle SMs).
template <typename T, int FACTO>
__global__ void __launch_bounds__(256, 2) diag_factor_kernel(DevSym s, const int *__restrict__ cblks, T *L,
                                                          T *U, T *tinv, const int64_t *__restrict__ tinv_off,
                                                          const double *__restrict__ thr_ptr,
                                                          unsigned long long *npiv, int *err) {
    __shared__ T tile[32 * TP];
    __shared__ T wl[32 * TP];
    __shared__ T wu[32 * TP];
    extern __shared__ __align__(16) float diag_wbuf[];  // FP32 only: per-warp 32x33 staging
    __shared__ int s_piv, s_err;
    const int k = cblks[blockIdx.x];
    const int n = s.ncols[k], ld = s.ld[k];
    const double thr = cblk_threshold(s, thr_ptr, k);
    T *A = L + s.off[k];
    T *ti = tinv + tinv_off[k];
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) { s_piv = 0; s_err = 0; }
    if (FACTO == FACTO_GETRF) {
        const T *Au = U + s.off[k];
        for (int idx = tid; idx < n * n; idx += nth) {
            const int i = idx % n, j = idx / n;
            A[i + (size_t)j * ld] += Au[j + (size_t)i * ld];
        }
    }
    __syncthreads();
    for (int p = 0, pi = 0; p < n; p += 32, pi++) {
        const int pb = min(32, n - p);
        T *Ap = A + p + (size_t)p * ld;
        for (int idx = tid; idx < 32 * 32; idx += nth) {
            const int i = idx & 31, j = idx >> 5;
            tile[i + j * TP] = (i < pb && j < pb) ? Ap[i + (size_t)j * ld] : (T)0;
        }
        __syncthreads();
        if (warp == 0) factor_tile<T, FACTO>(tile, pb, lane, thr, &s_piv, &s_err);
        __syncthreads();
        if (warp == 0) invert_lower_tile<T>(tile, wl, pb, lane, FACTO != FACTO_POTRF, 0);
        if (FACTO == FACTO_GETRF && warp == 1) invert_lower_tile<T>(tile, wu, pb, lane, 0, 1);  // inv(U^T)
        __syncthreads();
        // store the factored tile and its inverse(s)
        for (int idx = tid; idx < 32 * 32; idx += nth) {
            const int i = idx & 31, j = idx >> 5;
            if (i < pb && j < pb && (FACTO != FACTO_POTRF || i >= j)) Ap[i + (size_t)j * ld] = tile[i + j * TP];
            // panel pi of the tile-inverse store: 32 x pb, after pi full panels (two per panel for LU)
            if (j < pb) {
                T *tp = ti + (size_t)pi * 1024 * (FACTO == FACTO_GETRF ? 2 : 1);
                tp[i + j * 32] = wl[i + j * TP];
                if (FACTO == FACTO_GETRF) tp[32 * pb + i + j * 32] = wu[i + j * TP];
            }
        }
        const int rest = n - p - pb;
        if (rest > 0) {
            // rows below the tile: X = A op(T)^{-1}; Cholesky with the tile inverse,
            // LU / LDL^T by substitution in the reference's order (indefinite or
            // badly scaled tiles)
            for (int r = tid; r < rest; r += nth) {
                T *row = A + (p + pb + r) + (size_t)p * ld;
                T a[32];
#pragma unroll
                for (int c = 0; c < 32; c++) a[c] = (c < pb) ? row[(size_t)c * ld] : (T)0;
                if (FACTO == FACTO_POTRF) {
#pragma unroll
                    for (int c = 0; c < 32; c++) {
                        if (c < pb) {
                            // X = A L^{-T}: (L^{-T})[l][c] = inv(L)[c][l]
                            T v = 0;
#pragma unroll
                            for (int l = 0; l <= c; l++) v += a[l] * wl[c + l * TP];
                            row[(size_t)c * ld] = v;
                        }
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 32; c++) {
                        if (c < pb) {
                            T v = a[c];
#pragma unroll
                            for (int l = 0; l < c; l++) {
                                // GETRF: X U = A with U = the upper part; LDL^T: V L^T = A, unit L
                                const T u = (FACTO == FACTO_GETRF) ? tile[l + c * TP] : tile[c + l * TP];
                                v -= a[l] * u;
                            }
                            if (FACTO == FACTO_GETRF) v /= tile[c * (TP + 1)];
                            a[c] = v;
                            if (FACTO == FACTO_SYTRF) {
                                A[(p + c) + (size_t)(p + pb + r) * ld] = v;          // (L D)^T in the upper part
                                row[(size_t)c * ld] = v * ((T)1 / tile[c * (TP + 1)]);  // L
                            } else {
                                row[(size_t)c * ld] = v;
                            }
                        }
                    }
                }
            }
            if (FACTO == FACTO_GETRF) {
                // columns right of the tile: Y = L_tile^{-1} A (unit lower), by substitution
                for (int cc = tid; cc < rest; cc += nth) {
                    T *col = A + p + (size_t)(p + pb + cc) * ld;
                    T a[32];
#pragma unroll
                    for (int l = 0; l < 32; l++) a[l] = (l < pb) ? col[l] : (T)0;
#pragma unroll
                    for (int l = 0; l < 32; l++) {
                        if (l < pb) {
                            T v = a[l];
#pragma unroll
                            for (int m = 0; m < l; m++) v -= tile[l + m * TP] * a[m];
                            a[l] = v;
                            col[l] = v;
                        }
                    }
                }
            }
            __syncthreads();
            // trailing update, one 32x32 tile per warp at a time
            const int nt = (rest + 31) / 32;
            const int ntiles = (FACTO == FACTO_GETRF) ? nt * nt : nt * (nt + 1) / 2;
            for (int t = warp; t < ntiles; t += 8) {
                int ti_, tj_;
                if (FACTO == FACTO_GETRF) {
                    ti_ = t % nt;
                    tj_ = t / nt;
                } else {
                    tj_ = 0;
                    int rem = t;
                    while (rem >= nt - tj_) { rem -= nt - tj_; tj_++; }
                    ti_ = tj_ + rem;
                }
                warp_tile_update(A, ld, n, p, pb, p + pb + ti_ * 32, p + pb + tj_ * 32, FACTO != FACTO_POTRF,
                                 FACTO != FACTO_GETRF, lane, reinterpret_cast<T *>(diag_wbuf) + warp * 32 * 33);
            }
        }
        __syncthreads();
    }
    if (FACTO == FACTO_GETRF) {
        T *Au = U + s.off[k];
        for (int idx = tid; idx < n * n; idx += nth) {
            const int i = idx % n, j = idx / n;
            Au[j + (size_t)i * ld] = A[i + (size_t)j * ld];
        }
    }
    if (tid == 0) {
        if (s_piv) atomicAdd(cblk_pivot_counter(s, npiv, k), (unsigned long long)s_piv);
        if (s_err) atomicOr(err, 1);
    }
}

// ------------------------------------------------------------------ panel TRSM

// X op(T) = B for a tile of TR off-diagonal rows of cblk k, the whole tile held
// in shared memory.  op(T) is upper triangular:
//   mode 0: op(T)[l][c] = D[l + c*ld]  (upper part of the diagonal block)
//   mode 1: op(T)[l][c] = D[c + l*ld]  (lower part, transposed)
template <typename T>
__global__ void __launch_bounds__(256) panel_trsm_kernel(DevSym s, const RowTask *__restrict__ tasks, int TR,
                                                         T *P, const T *Dsrc, int mode, const T *__restrict__ tinv,
                                                         const int64_t *__restrict__ tinv_off, int which, int getrf,
                                                         int scale_d) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T *xs = reinterpret_cast<T *>(smraw);  // TR x n, column-major
    __shared__ T ts[64 * TP];
    __shared__ T tt[32 * TP];
    const RowTask t = tasks[blockIdx.x];
    const int k = t.k, n = s.ncols[k], ld = s.ld[k];
    const int rows = min(TR, s.stride[k] - t.row0);
    T *X = P + s.off[k] + t.row0;
    const T *D = Dsrc + s.off[k];
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int idx = tid; idx < TR * n; idx += nth) {
        const int r = idx % TR, c = idx / TR;
        xs[idx] = (r < rows) ? X[r + (size_t)c * ld] : (T)0;
    }
    __syncthreads();
    const int NG = nth / TR;      // column groups
    const int CPG = 32 / NG;      // columns per group (<= 8)
    const int r = tid % TR, cg = tid / TR;
    for (int cb = 0; cb < n; cb += 32) {
        const int w = min(32, n - cb);
        T acc[8];
#pragma unroll
        for (int q = 0; q < 8; q++) acc[q] = 0;
        for (int l0 = 0; l0 < cb; l0 += 64) {
            const int lw = min(64, cb - l0);
            for (int idx = tid; idx < 64 * 32; idx += nth) {
                const int l = idx >> 5, c = idx & 31;
                T v = 0;
                if (l < lw && c < w) v = mode == 0 ? D[(l0 + l) + (size_t)(cb + c) * ld] : D[(cb + c) + (size_t)(l0 + l) * ld];
                ts[l * TP + c] = v;
            }
            __syncthreads();
            for (int l = 0; l < lw; l++) {
                const T xv = xs[r + (l0 + l) * TR];
#pragma unroll
                for (int q = 0; q < 8; q++)
                    if (q < CPG) acc[q] += xv * ts[l * TP + cg * CPG + q];
            }
            __syncthreads();
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int c = cg * CPG + q;
            if (q < CPG && c < w) xs[r + (cb + c) * TR] -= acc[q];
        }
        if (!getrf && !scale_d) {
        // multiplier of this column block: M(l, c) = W[c][l] (W = the stored tile
        // inverse of the Cholesky factor)
        {
            const T *W = tinv + tinv_off[k] + (size_t)(cb >> 5) * 1024 * (getrf ? 2 : 1) + (which ? 32 * w : 0);
            for (int idx = tid; idx < 32 * 32; idx += nth) {
                const int l = idx >> 5, c = idx & 31;
                T v = 0;
                if (l < w && c < w && c >= l) {
                    v = W[c + l * 32];
                    if (scale_d) v = v / D[(size_t)(cb + c) * (ld + 1)];
                }
                tt[l * TP + c] = v;
            }
        }
        __syncthreads();
        {
            T out[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                out[q] = 0;
                const int c = cg * CPG + q;
                if (q < CPG && c < w)
                    for (int l = 0; l <= c; l++) out[q] += xs[r + (cb + l) * TR] * tt[l * TP + c];
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int c = cg * CPG + q;
                if (q < CPG && c < w) xs[r + (cb + c) * TR] = out[q];
            }
        }
        } else {
            // LU and LDL^T: substitution against the upper triangular block
            // U(l, c) = op(T)[cb + l][cb + c] (LDL^T: D L^T; the U-side LU panel has a
            // unit diagonal), the order of PaStiX's TRSM, which keeps indefinite or
            // badly scaled diagonal blocks as accurate as the reference
            for (int idx = tid; idx < 32 * 32; idx += nth) {
                const int l = idx >> 5, c = idx & 31;
                T v = 0;
                if (l < w && c < w && c >= l)
                    v = mode == 0 ? D[(cb + l) + (size_t)(cb + c) * ld] : D[(cb + c) + (size_t)(cb + l) * ld];
                tt[l * TP + c] = v;
            }
            __syncthreads();
            const bool unit = getrf && which == 0;
            if (tid < TR) {
                for (int c = 0; c < w; c++) {
                    T x = xs[tid + (cb + c) * TR];
                    for (int l = 0; l < c; l++) x -= xs[tid + (cb + l) * TR] * tt[l * TP + c];
                    xs[tid + (cb + c) * TR] = unit ? x : x / tt[c * TP + c];
                }
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < TR * n; idx += nth) {
        const int rr = idx % TR, c = idx / TR;
        if (rr < rows) X[rr + (size_t)c * ld] = xs[idx];
    }
}




// ------------------------------------------------------------------ updates

__device__ __forceinline__ int find_update(const Upd *__restrict__ upds, int nupd, int tile) {
    int lo = 0, hi = nupd - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (upds[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void tile_coords(const Upd &u, int lt, int &mt, int &nt) {
    if (u.flags & UPD_SYM) {
        nt = 0;
        while (lt >= u.tiles_m - nt) { lt -= u.tiles_m - nt; nt++; }
        mt = nt + lt;
    } else {
        mt = lt % u.tiles_m;
        nt = lt / u.tiles_m;
    }
}

__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], const double (&a)[2], double b) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(b));
}

constexpr int UT_M = 64, UT_N = 64, UT_K = 16, UT_STAGES = 3, UT_LDS = UT_M + 4;
constexpr int UPD_F64_SMEM = 2 * UT_STAGES * UT_K * UT_LDS * sizeof(double);

// 64x64 output tile per CTA, 4 warps (2x2) of 32x32, DMMA m16n8k4, 3-stage
// cp.async pipeline over K in chunks of 16 columns.
__global__ void __launch_bounds__(128) update_f64_kernel(DevSym s, const Upd *__restrict__ upds, int nupd,
                                                         double *L, double *U) {
    extern __shared__ __align__(16) unsigned char upd_smem[];
    double(*As)[UT_K][UT_LDS] = reinterpret_cast<double(*)[UT_K][UT_LDS]>(upd_smem);
    double(*Bs)[UT_K][UT_LDS] = reinterpret_cast<double(*)[UT_K][UT_LDS]>(upd_smem + sizeof(double) * UT_STAGES * UT_K * UT_LDS);
    __shared__ double Ds[UT_STAGES][UT_K];
    __shared__ int drow[UT_M];
    const int tile = blockIdx.x;
    const Upd u = upds[find_update(upds, nupd, tile)];
    int mt, nt;
    tile_coords(u, tile - u.tile0, mt, nt);
    const int m0 = mt * UT_M, n0 = nt * UT_N;
    const int k = u.k, ldk = s.ld[k];
    const double *Ap = ((u.flags & UPD_A_U) ? U : L) + s.off[k] + u.rowA0 + m0 + (size_t)u.colK0 * ldk;
    const double *Bp = ((u.flags & UPD_B_U) ? U : L) + s.off[k] + u.rowB0 + n0 + (size_t)u.colK0 * ldk;
    const double *Dp = L + s.off[k] + (size_t)u.colK0 * (ldk + 1);
    const bool scale = (u.flags & UPD_SCALE_D) != 0;
    const int mrem = u.M - m0, nrem = u.N - n0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int g = lane >> 2, tg = lane & 3;

    auto load_stage = [&](int st, int kc) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int idx = tid + i * 128;
            const int r = idx & 63, c = idx >> 6;
            const int kk = kc + c;
            const bool okA = (r < mrem) && (kk < u.K);
            const bool okB = (r < nrem) && (kk < u.K);
            cp_async8(&As[st][c][r], okA ? Ap + r + (size_t)kk * ldk : Ap, okA);
            cp_async8(&Bs[st][c][r], okB ? Bp + r + (size_t)kk * ldk : Bp, okB);
        }
        if (scale && tid < UT_K) {
            const int kk = kc + tid;
            Ds[st][tid] = (kk < u.K) ? Dp[(size_t)kk * (ldk + 1)] : 0.0;
        }
    };

    double acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[a][b][e] = 0.0;

    const int nk = (u.K + UT_K - 1) / UT_K;
#pragma unroll
    for (int st = 0; st < UT_STAGES - 1; st++) {
        if (st < nk) load_stage(st, st * UT_K);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; kt++) {
        cp_async_wait<UT_STAGES - 2>();
        __syncthreads();
        const int st = kt % UT_STAGES;
        const int nxt = kt + UT_STAGES - 1;
        if (nxt < nk) load_stage(nxt % UT_STAGES, nxt * UT_K);
        cp_async_commit();
#pragma unroll
        for (int k4 = 0; k4 < UT_K; k4 += 4) {
            double a[2][2], b[4];
            const double dsc = scale ? Ds[st][k4 + tg] : 1.0;
#pragma unroll
            for (int mi = 0; mi < 2; mi++) {
                const int row = wm * 32 + mi * 16 + g;
                a[mi][0] = As[st][k4 + tg][row] * dsc;
                a[mi][1] = As[st][k4 + tg][row + 8] * dsc;
            }
#pragma unroll
            for (int ni = 0; ni < 4; ni++) b[ni] = Bs[st][k4 + tg][wn * 32 + ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++) dmma_16x8x4(acc[mi][ni], a[mi], b[ni]);
        }
    }
    cp_async_wait<0>();
    if (tid < UT_M) drow[tid] = (m0 + tid < u.M) ? __ldg(s.rmap + u.rm0 + m0 + tid) : -1;
    __syncthreads();
    double *C = ((u.flags & UPD_C_U) ? U : L) + s.off[u.f];
    const int ldf = s.ld[u.f];
    const bool atomic = (u.flags & UPD_ATOMIC) != 0;
    const bool sym = (u.flags & UPD_SYM) != 0;
#pragma unroll
    for (int mi = 0; mi < 2; mi++) {
#pragma unroll
        for (int ni = 0; ni < 4; ni++) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int row = wm * 32 + mi * 16 + g + (e >> 1) * 8;
                const int col = wn * 32 + ni * 8 + 2 * tg + (e & 1);
                if (n0 + col >= u.N) continue;
                if (sym && m0 + row < n0 + col) continue;
                const int d = drow[row];
                if (d < 0) continue;
                double *p = C + d + (size_t)(u.colbase + n0 + col) * ldf;
                if (atomic) atomicAdd(p, -acc[mi][ni][e]);
                else *p -= acc[mi][ni][e];
            }
        }
    }
}

// FP32 factor update on CUDA cores: 64x64 tile, 256 threads (4x4 each), K chunks of 16.
__global__ void __launch_bounds__(256) update_simt_f32_kernel(DevSym s, const Upd *__restrict__ upds, int nupd,
                                                              float *L, float *U) {
    __shared__ __align__(16) float As[2][UT_K][UT_M + 4];
    __shared__ __align__(16) float Bs[2][UT_K][UT_N + 4];
    __shared__ int drow[UT_M];
    const int tile = blockIdx.x;
    const Upd u = upds[find_update(upds, nupd, tile)];
    int mt, nt;
    tile_coords(u, tile - u.tile0, mt, nt);
    const int m0 = mt * UT_M, n0 = nt * UT_N;
    const int k = u.k, ldk = s.ld[k];
    const float *Ap = ((u.flags & UPD_A_U) ? U : L) + s.off[k] + u.rowA0 + m0 + (size_t)u.colK0 * ldk;
    const float *Bp = ((u.flags & UPD_B_U) ? U : L) + s.off[k] + u.rowB0 + n0 + (size_t)u.colK0 * ldk;
    const float *Dp = L + s.off[k] + (size_t)u.colK0 * (ldk + 1);
    const bool scale = (u.flags & UPD_SCALE_D) != 0;
    const int mrem = u.M - m0, nrem = u.N - n0;
    const int tid = threadIdx.x;
    const int tr = tid & 15, tc = tid >> 4;
    float acc[4][4] = {};
    const int nk = (u.K + UT_K - 1) / UT_K;
    auto load_stage = [&](int st, int kc) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int idx = tid + i * 256;
            const int r = idx & 63, c = idx >> 6;
            const int kk = kc + c;
            const bool okA = (r < mrem) && (kk < u.K);
            const bool okB = (r < nrem) && (kk < u.K);
            cp_async4(&As[st][c][r], okA ? Ap + r + (size_t)kk * ldk : Ap, okA);
            cp_async4(&Bs[st][c][r], okB ? Bp + r + (size_t)kk * ldk : Bp, okB);
        }
    };
    load_stage(0, 0);
    cp_async_commit();
    for (int kt = 0; kt < nk; kt++) {
        const int st = kt & 1;
        if (kt + 1 < nk) load_stage(st ^ 1, (kt + 1) * UT_K);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
#pragma unroll
        for (int c = 0; c < UT_K; c++) {
            const int kk = kt * UT_K + c;
            const float dsc = (scale && kk < u.K) ? Dp[(size_t)kk * (ldk + 1)] : 1.0f;
            float av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; a++) av[a] = As[st][c][tr + 16 * a] * dsc;
#pragma unroll
            for (int b = 0; b < 4; b++) bv[b] = Bs[st][c][tc + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
        }
        __syncthreads();
    }
    if (tid < UT_M) drow[tid] = (m0 + tid < u.M) ? __ldg(s.rmap + u.rm0 + m0 + tid) : -1;
    __syncthreads();
    float *C = ((u.flags & UPD_C_U) ? U : L) + s.off[u.f];
    const int ldf = s.ld[u.f];
    const bool atomic = (u.flags & UPD_ATOMIC) != 0;
    const bool sym = (u.flags & UPD_SYM) != 0;
#pragma unroll
    for (int a = 0; a < 4; a++) {
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int row = tr + 16 * a, col = tc + 16 * b;
            if (n0 + col >= u.N) continue;
            if (sym && m0 + row < n0 + col) continue;
            const int d = drow[row];
            if (d < 0) continue;
            float *p = C + d + (size_t)(u.colbase + n0 + col) * ldf;
            if (atomic) atomicAdd(p, -acc[a][b]);
            else *p -= acc[a][b];
        }
    }
}

// ------------------------------------------------------------------ launchers

template <typename T>
void launch_scatter(int64_t nnz, const int64_t *dest, const double *Lv, const double *Uv, T *L, T *U,
                    cudaStream_t st) {
    if (nnz <= 0) return;
    const int bs = 256;
    scatter_kernel<T><<<(unsigned)((nnz + bs - 1) / bs), bs, 0, st>>>(nnz, dest, Lv, Uv, L, U);
}

constexpr int DS_WARPS = 4;  // warps (cblks) per CTA of diag_small_kernel

// Rows below the diagonal block of cblk k (at most 32 columns), lane = row: POTRF
// X = A L^{-T} with the tile inverse wl; LU (lower side) and LDL^T by substitution
// against the upper part of the factored tile (U; D L^T), dividing by its diagonal;
// LU upper side (the transposed U panel) against the unit lower part.  NB >= ncols
// (8, 16 or 32) bounds the columns.
template <typename T, int FACTO, int NB>
__device__ void small_trsm_warp(const DevSym &s, int k, T *L, T *U, const T *tile, const T *wl, int lane) {
    const int n = s.ncols[k], ld = s.ld[k], stride = s.stride[k];
    for (int side = 0; side < (FACTO == FACTO_GETRF ? 2 : 1); side++) {
        T *P = (side ? U : L) + s.off[k];
        for (int r0 = n; r0 < stride; r0 += 32) {
            const int row = r0 + lane;
            if (row >= stride) continue;
            T *rp = P + row;
            T a[NB];
#pragma unroll
            for (int c = 0; c < NB; c++) a[c] = (c < n) ? rp[(size_t)c * ld] : (T)0;
            if (FACTO == FACTO_POTRF) {
                // x_c = sum_{l <= c} a_l inv(L)[c][l], in place from the last column
#pragma unroll
                for (int c = NB - 1; c >= 0; c--) {
                    if (c < n) {
                        T v = 0;
#pragma unroll
                        for (int l = 0; l <= c; l++) v += a[l] * wl[c + l * TP];
                        a[c] = v;
                    }
                }
            } else {
#pragma unroll
                for (int c = 0; c < NB; c++) {
                    if (c < n) {
                        T v = a[c];
#pragma unroll
                        for (int l = 0; l < c; l++) v -= a[l] * (side ? tile[c + l * TP] : tile[l + c * TP]);
                        a[c] = side ? v : v / tile[c * (TP + 1)];
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < NB; c++)
                if (c < n) rp[(size_t)c * ld] = a[c];
        }
    }
}

// One warp factors the diagonal block of cblk k (at most NB <= 32 columns): tile,
// wl and (LU) wu are the warp's shared-memory tiles of NB columns (pitch TP), *piv /
// *ferr its counters in shared memory.  On return the factored tile is still in tile
// (the panel solve, small_trsm_warp, reads it from there).
template <typename T, int FACTO, int NB>
__device__ __forceinline__ void small_diag_warp(const DevSym &s, int k, T *L, T *U, T *tinv,
                                                const int64_t *__restrict__ tinv_off, const double *__restrict__ thr_ptr,
                                                unsigned long long *npiv, int *err, T *tile, T *wl, T *wu, int *piv,
                                                int *ferr, int lane) {
    const int n = s.ncols[k], ld = s.ld[k];
    const double thr = cblk_threshold(s, thr_ptr, k);
    T *A = L + s.off[k];
    if (lane == 0) { *piv = 0; *ferr = 0; }
    stage_n<NB, T>(
        [&](int j) {
            T v = 0;
            if (lane < n && j < n) {
                v = A[lane + (size_t)j * ld];
                if (FACTO == FACTO_GETRF) v += U[s.off[k] + j + (size_t)lane * ld];
            }
            return v;
        },
        [&](int j, T v) { tile[lane + j * TP] = v; });
    __syncwarp();
    factor_tile<T, FACTO, NB>(tile, n, lane, thr, piv, ferr);
    invert_lower_tile<T, NB>(tile, wl, n, lane, FACTO != FACTO_POTRF, 0);
    if (FACTO == FACTO_GETRF) invert_lower_tile<T, NB>(tile, wu, n, lane, 0, 1);  // inv(U^T)
    T *tp = tinv + tinv_off[k];
    for (int idx = lane; idx < 32 * NB; idx += 32) {
        const int i = idx & 31, j = idx >> 5;
        if (i < n && j < n && (FACTO != FACTO_POTRF || i >= j)) {
            A[i + (size_t)j * ld] = tile[i + j * TP];
            if (FACTO == FACTO_GETRF) U[s.off[k] + j + (size_t)i * ld] = tile[i + j * TP];
        }
        if (j < n) {
            tp[i + j * 32] = wl[i + j * TP];
            if (FACTO == FACTO_GETRF) tp[32 * n + i + j * 32] = wu[i + j * TP];
        }
    }
    __syncwarp();
    if (lane == 0) {
        if (*piv) atomicAdd(cblk_pivot_counter(s, npiv, k), (unsigned long long)*piv);
        if (*ferr) atomicOr(err, 1);
    }
}

// Cblks with at most 32 columns, one warp per cblk (the bottom levels of the tree
// hold tens of thousands): the single-panel case of diag_factor_kernel -- geadd of
// U^T for LU, factor_tile, the tile inverse(s), write-back (and U^T for LU) -- and
// the panel solve of the rows below (small_trsm_warp), so that these cblks need no
// TRSM launch.  One instance per width class NB (8, 16, 32 columns): the narrow
// classes, most of the cblks, need a fraction of the registers and shared memory, so
// more warps share an SM.
template <typename T, int FACTO, int NB>
__global__ void __launch_bounds__(32 * DS_WARPS) diag_small_kernel(DevSym s, const int *__restrict__ cblks, int ncblk,
                                                                   T *L, T *U, T *tinv,
                                                                   const int64_t *__restrict__ tinv_off,
                                                                   const double *__restrict__ thr_ptr,
                                                                   unsigned long long *npiv, int *err) {
    extern __shared__ __align__(16) unsigned char ds_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NT = (FACTO == FACTO_GETRF) ? 3 : 2;
    T *tile = reinterpret_cast<T *>(ds_smem) + (size_t)warp * NT * NB * TP;
    T *wl = tile + NB * TP;
    T *wu = wl + NB * TP;
    __shared__ int s_piv[DS_WARPS], s_err[DS_WARPS];
    const int ci = blockIdx.x * DS_WARPS + warp;
    if (ci >= ncblk) return;
    const int k = cblks[ci];
    small_diag_warp<T, FACTO, NB>(s, k, L, U, tinv, tinv_off, thr_ptr, npiv, err, tile, wl, wu, &s_piv[warp],
                                  &s_err[warp], lane);
    small_trsm_warp<T, FACTO, NB>(s, k, L, U, tile, wl, lane);
}

// Small GEMM-scatter updates (K <= 16, N <= 32: the bottom levels of the tree,
// far below a 64 x 64 tile), one warp each: lane = row of the M-range (32 rows per
// pass), C[d(i)][colbase + c] -= sum_k A[i][k] (D[k]) B[c][k] for c < N (c <= i when
// symmetric).  Same operation as the tile kernels (core_zgemmsp_2d2d,
// kernels/core_zgemmsp.c:396-465).  Each warp waits mostly on its loads, so the
// launch bounds ask for 4 (FP32) / 3 (FP64) CTAs per SM: 64 / 80 registers, a few
// bytes of spill, a third to a half more warps in flight.
constexpr int US_WARPS = 8;

template <typename T>
__global__ void __launch_bounds__(32 * US_WARPS, sizeof(T) == 4 ? 4 : 3) update_small_kernel(DevSym s, const Upd *__restrict__ upds, int nupd,
                                                                     T *L, T *U) {
    const int lane = threadIdx.x & 31;
    const int ui = blockIdx.x * US_WARPS + (threadIdx.x >> 5);
    if (ui >= nupd) return;
    const Upd u = upds[ui];
    const int k = u.k, ldk = s.ld[k];
    const T *Ap = ((u.flags & UPD_A_U) ? U : L) + s.off[k] + u.rowA0 + (size_t)u.colK0 * ldk;
    const T *Bp = ((u.flags & UPD_B_U) ? U : L) + s.off[k] + u.rowB0 + (size_t)u.colK0 * ldk;
    const T *Dp = L + s.off[k] + (size_t)u.colK0 * (ldk + 1);
    const bool scale = (u.flags & UPD_SCALE_D) != 0;
    const bool atomic = (u.flags & UPD_ATOMIC) != 0;
    const bool sym = (u.flags & UPD_SYM) != 0;
    T *C = ((u.flags & UPD_C_U) ? U : L) + s.off[u.f];
    const int ldf = s.ld[u.f];
    // B (N x K, N <= 32, K <= 16) with D folded into A: bs[c][q] = B[c][q] in shared
    // memory, read by every lane as 128-bit broadcasts
    __shared__ __align__(16) T bsm[US_WARPS][32][16];
    T(*bs)[16] = bsm[threadIdx.x >> 5];
#pragma unroll
    for (int q = 0; q < 16; q++) bs[lane][q] = (lane < u.N && q < u.K) ? Bp[lane + (size_t)q * ldk] : (T)0;
    T dk = (scale && lane < u.K) ? Dp[(size_t)lane * (ldk + 1)] : (T)1;
    __syncwarp();
    for (int r0 = 0; r0 < u.M; r0 += 32) {
        const int i = r0 + lane;
        const bool in = i < u.M;
        T a[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const T dq = __shfl_sync(0xffffffffu, dk, q);
            a[q] = (in && q < u.K) ? Ap[i + (size_t)q * ldk] * dq : (T)0;
        }
        const int d = in ? __ldg(s.rmap + u.rm0 + i) : -1;
        T *crow = C + d + (size_t)u.colbase * ldf;
        for (int c = 0; c < u.N; c++) {
            T acc = 0;
            if constexpr (sizeof(T) == 4) {
                const float4 *b4 = reinterpret_cast<const float4 *>(bs[c]);
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const float4 bq = b4[h];
                    acc += a[4 * h] * bq.x;
                    acc += a[4 * h + 1] * bq.y;
                    acc += a[4 * h + 2] * bq.z;
                    acc += a[4 * h + 3] * bq.w;
                }
            } else {
                const double2 *b2 = reinterpret_cast<const double2 *>(bs[c]);
#pragma unroll
                for (int h = 0; h < 8; h++) {
                    const double2 bq = b2[h];
                    acc += a[2 * h] * bq.x;
                    acc += a[2 * h + 1] * bq.y;
                }
            }
            if (d >= 0 && !(sym && i < c)) {
                if (atomic) atomicAdd(crow + (size_t)c * ldf, -acc);
                else crow[(size_t)c * ldf] -= acc;
            }
        }
    }
}

// ------------------------------------------------------------------ tree-bottom launch

// The bottom levels of the elimination tree (every cblk of at most 32 columns, no
// update on the tensor cores) in one launch, as PaStiX's dynamic scheduler runs
// them: a cblk starts as soon as the cblks that update it are done, without level
// barriers (cpucblk_zincoming_deps / cpucblk_zrelease_deps,
// kernels/cpucblk_zmpi_coeftab.c:482-562; sequential_zpotrf.c's dynamic driver,
// sopalin/sequential_zpotrf.c:129-234).  Items (DagItem) are taken by warps from an
// atomic ticket, level by level: the level's factor items, then its update items.  A
// factor item waits until its cblk's counter (the update items it receives from the
// launch's cblks, ctrbcnt) is 0, factors the diagonal block (small_diag_warp), solves
// the rows below it against the factored tile still in shared memory (core_ztrsmsp,
// kernels/core_ztrsmsp.c:147-181), runs the cblk's updates itself when they are few,
// and marks the cblk factored (counter -1).  An update item waits for that mark and
// applies its updates (or rows of one) with atomics, the facing cblk receiving
// others at the same time (core_zgemmsp_2d2d, kernels/core_zgemmsp.c:396-465); every
// item then decrements the facing cblks' counters, once per update.  An item only
// waits for earlier items, which running warps hold, so the launch completes whatever
// the number of resident warps.  Every wait is bounded: on expiry the warp sets bit 5
// of err and an abort word that ends the other warps' waits.
constexpr int DG_WARPS = 4;
constexpr long long DAG_WAIT_CYCLES = 1000000000LL;  // about 0.5 s at the maximum SM clock

__device__ __forceinline__ int dag_ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait (one lane) until *cnt <= target; false on expiry or abort.
__device__ bool dag_wait(const int *cnt, int target, const int *abort_word) {
    const long long t0 = clock64();
    for (int it = 0;; it++) {
        if (dag_ld_acquire(cnt) <= target) return true;
        if ((it & 15) == 15) {
            if (dag_ld_acquire(abort_word)) return false;
            if (clock64() - t0 > DAG_WAIT_CYCLES) return false;
        }
        __nanosleep(64);
    }
}

// One update with K <= KB columns by one warp on the rows [rb, re) of its M-range
// (rb a multiple of 32), every sum accumulated with atomics:
// C[d(i)][colbase + c] -= sum_q A[i][q] (D_q) B[c][q] (c <= i when symmetric), B in
// chunks of 32 rows staged in bs (32 x TP).
template <typename T, int KB>
__device__ void warp_update(const DevSym &s, const Upd &u, T *L, T *U, T *bs, int lane, int rb, int re) {
    const int k = u.k, ldk = s.ld[k];
    const T *Ap = ((u.flags & UPD_A_U) ? U : L) + s.off[k] + u.rowA0 + (size_t)u.colK0 * ldk;
    const T *Bp = ((u.flags & UPD_B_U) ? U : L) + s.off[k] + u.rowB0 + (size_t)u.colK0 * ldk;
    const T *Dp = L + s.off[k] + (size_t)u.colK0 * (ldk + 1);
    const bool scale = (u.flags & UPD_SCALE_D) != 0, sym = (u.flags & UPD_SYM) != 0;
    T *C = ((u.flags & UPD_C_U) ? U : L) + s.off[u.f];
    const int ldf = s.ld[u.f];
    const T dk = (scale && lane < u.K) ? Dp[(size_t)lane * (ldk + 1)] : (T)1;
    for (int n0 = 0; n0 < u.N; n0 += 32) {
        const int nw = min(32, u.N - n0);
        __syncwarp();
#pragma unroll
        for (int q = 0; q < KB; q++)
            bs[lane * TP + q] = (lane < nw && q < u.K) ? Bp[(n0 + lane) + (size_t)q * ldk] : (T)0;
        __syncwarp();
        // symmetric: rows above n0 lie above the diagonal for every column of the chunk
        const int rend = min(u.M, re);
        for (int r0 = sym ? max(n0, rb) : rb; r0 < rend; r0 += 32) {
            const int i = r0 + lane;
            const bool in = i < rend;
            T a[KB];
#pragma unroll
            for (int q = 0; q < KB; q++) {
                const T dq = __shfl_sync(0xffffffffu, dk, q);
                a[q] = (in && q < u.K) ? Ap[i + (size_t)q * ldk] * dq : (T)0;
            }
            const int d = in ? __ldg(s.rmap + u.rm0 + i) : -1;
            if (d < 0) continue;
            T *crow = C + d + (size_t)(u.colbase + n0) * ldf;
            for (int c = 0; c < nw; c++) {
                T acc = 0;
#pragma unroll
                for (int q = 0; q < KB; q++) acc += a[q] * bs[c * TP + q];
                if (!(sym && i < n0 + c)) atomicAdd(crow + (size_t)c * ldf, -acc);
            }
        }
    }
    __syncwarp();
}

template <typename T, int FACTO>
__global__ void __launch_bounds__(32 * DG_WARPS) dag_bottom_kernel(DevSym s, const DagItem *__restrict__ items,
                                                                   int nitems, const Upd *__restrict__ upds, int *cnt,
                                                                   int *ticket, int *abort_word, T *L, T *U,
                                                                   T *tinv, const int64_t *__restrict__ tinv_off,
                                                                   const double *__restrict__ thr_ptr,
                                                                   unsigned long long *npiv, int *err) {
    extern __shared__ __align__(16) unsigned char dg_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NT = (FACTO == FACTO_GETRF) ? 3 : 2;
    T *tile = reinterpret_cast<T *>(dg_smem) + (size_t)warp * NT * 32 * TP;
    T *wl = tile + 32 * TP;
    T *wu = wl + 32 * TP;
    __shared__ int s_piv[DG_WARPS], s_err[DG_WARPS];
    for (;;) {
        __syncwarp();
        int t = 0;
        if (lane == 0) t = atomicAdd(ticket, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= nitems) return;
        const DagItem it = items[t];
        const int k = it.k;
        int ok = 1;
        if (lane == 0) ok = dag_wait(cnt + k, it.fact ? 0 : -1, abort_word);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
            if (lane == 0) {
                atomicOr(err, 32);
                atomicExch(abort_word, 1);
            }
            return;
        }
        __syncwarp();  // the other lanes' reads of k's panel come after lane 0's acquire
        const int n = s.ncols[k];
        if (it.fact) {
            if (n <= 8) {
                small_diag_warp<T, FACTO, 8>(s, k, L, U, tinv, tinv_off, thr_ptr, npiv, err, tile, wl, wu,
                                             &s_piv[warp], &s_err[warp], lane);
                small_trsm_warp<T, FACTO, 8>(s, k, L, U, tile, wl, lane);
            } else if (n <= 16) {
                small_diag_warp<T, FACTO, 16>(s, k, L, U, tinv, tinv_off, thr_ptr, npiv, err, tile, wl, wu,
                                              &s_piv[warp], &s_err[warp], lane);
                small_trsm_warp<T, FACTO, 16>(s, k, L, U, tile, wl, lane);
            } else {
                small_diag_warp<T, FACTO, 32>(s, k, L, U, tinv, tinv_off, thr_ptr, npiv, err, tile, wl, wu,
                                              &s_piv[warp], &s_err[warp], lane);
                small_trsm_warp<T, FACTO, 32>(s, k, L, U, tile, wl, lane);
            }
            __syncwarp();  // the panel is final before any lane reads it for the updates
        }
        for (int q = it.q0; q < it.q1; q++) {
            const Upd u = upds[q];
            if (n <= 8) warp_update<T, 8>(s, u, L, U, wl, lane, it.r0, it.r1);
            else if (n <= 16) warp_update<T, 16>(s, u, L, U, wl, lane, it.r0, it.r1);
            else warp_update<T, 32>(s, u, L, U, wl, lane, it.r0, it.r1);
        }
        if (it.q1 > it.q0 || it.fact) {
            __threadfence();  // this lane's writes before the releases below
            __syncwarp();
            if (lane == 0) {
                __threadfence();
                for (int q = it.q0; q < it.q1; q++) atomicSub(cnt + upds[q].f, 1);
                if (it.fact) atomicExch(cnt + k, -1);  // factored: its update items may start
            }
        }
    }
}

// pastixGetDiag / coeftab_zgetdiag (sopalin/diag.c:55, sopalin/coeftab_z.c:462-492):
// the diagonal of every cblk's diagonal block in cblk order (the permuted
// numbering): L_kk's diagonal for Cholesky, D for LDL^T, U_kk's for LU.
template <typename T>
__global__ void get_diag_kernel(DevSym s, const T *__restrict__ L, double *out) {
    const int k = blockIdx.x;
    const int nc = s.ncols[k], ld = s.ld[k];
    const T *Lk = L + s.off[k];
    for (int i = threadIdx.x; i < nc; i += blockDim.x) out[s.fcol[k] + i] = (double)Lk[(size_t)i * (ld + 1)];
}

template <typename T>
void launch_get_diag(const DevSym &s, const T *L, double *out, cudaStream_t st) {
    if (s.cblknbr > 0) get_diag_kernel<T><<<s.cblknbr, 64, 0, st>>>(s, L, out);
}
template void launch_get_diag<double>(const DevSym &, const double *, double *, cudaStream_t);
template void launch_get_diag<float>(const DevSym &, const float *, double *, cudaStream_t);

template <typename T>
void launch_update_small(const DevSym &s, const Upd *upds, int nupd, T *L, T *U, cudaStream_t st) {
    if (nupd <= 0) return;
    update_small_kernel<T><<<(nupd + US_WARPS - 1) / US_WARPS, 32 * US_WARPS, 0, st>>>(s, upds, nupd, L, U);
}
template void launch_update_small<double>(const DevSym &, const Upd *, int, double *, double *, cudaStream_t);
template void launch_update_small<float>(const DevSym &, const Upd *, int, float *, float *, cudaStream_t);

template <typename T, int NB>
static void launch_diag_small_nb(int facto, const DevSym &s, const int *cblks, int ncblk, T *L, T *U, T *tinv,
                                 const int64_t *tinv_off, const double *thr, unsigned long long *npiv, int *err,
                                 cudaStream_t st) {
    const int grid = (ncblk + DS_WARPS - 1) / DS_WARPS;
    const size_t smem = (size_t)DS_WARPS * (facto == FACTO_GETRF ? 3 : 2) * NB * TP * sizeof(T);
    if (facto == FACTO_POTRF)
        diag_small_kernel<T, FACTO_POTRF, NB><<<grid, 32 * DS_WARPS, smem, st>>>(s, cblks, ncblk, L, U, tinv, tinv_off,
                                                                               thr, npiv, err);
    else if (facto == FACTO_GETRF)
        diag_small_kernel<T, FACTO_GETRF, NB><<<grid, 32 * DS_WARPS, smem, st>>>(s, cblks, ncblk, L, U, tinv, tinv_off,
                                                                               thr, npiv, err);
    else
        diag_small_kernel<T, FACTO_SYTRF, NB><<<grid, 32 * DS_WARPS, smem, st>>>(s, cblks, ncblk, L, U, tinv, tinv_off,
                                                                               thr, npiv, err);
}

template <typename T>
void launch_diag_small(int facto, const DevSym &s, const int *cblks, int ncblk, int nb, T *L, T *U, T *tinv,
                       const int64_t *tinv_off, const double *thr, unsigned long long *npiv, int *err,
                       cudaStream_t st) {
    if (ncblk <= 0) return;
    if (nb <= 8)
        launch_diag_small_nb<T, 8>(facto, s, cblks, ncblk, L, U, tinv, tinv_off, thr, npiv, err, st);
    else if (nb <= 16)
        launch_diag_small_nb<T, 16>(facto, s, cblks, ncblk, L, U, tinv, tinv_off, thr, npiv, err, st);
    else
        launch_diag_small_nb<T, 32>(facto, s, cblks, ncblk, L, U, tinv, tinv_off, thr, npiv, err, st);
}
template void launch_diag_small<double>(int, const DevSym &, const int *, int, int, double *, double *, double *,
                                        const int64_t *, const double *, unsigned long long *, int *, cudaStream_t);
template void launch_diag_small<float>(int, const DevSym &, const int *, int, int, float *, float *, float *,
                                       const int64_t *, const double *, unsigned long long *, int *, cudaStream_t);

static size_t dag_bottom_smem(int facto, size_t esz) {
    return (size_t)DG_WARPS * (facto == FACTO_GETRF ? 3 : 2) * 32 * TP * esz;
}

template <typename T>
void launch_dag_bottom(int facto, const DevSym &s, int grid, const DagItem *items, int nitems, const Upd *upds,
                       int *cnt, int *ticket, int *abort_word, T *L, T *U, T *tinv, const int64_t *tinv_off,
                       const double *thr, unsigned long long *npiv, int *err, cudaStream_t st) {
    if (nitems <= 0 || grid <= 0) return;
    const size_t smem = dag_bottom_smem(facto, sizeof(T));
    if (facto == FACTO_POTRF)
        dag_bottom_kernel<T, FACTO_POTRF><<<grid, 32 * DG_WARPS, smem, st>>>(
            s, items, nitems, upds, cnt, ticket, abort_word, L, U, tinv, tinv_off, thr, npiv, err);
    else if (facto == FACTO_GETRF)
        dag_bottom_kernel<T, FACTO_GETRF><<<grid, 32 * DG_WARPS, smem, st>>>(
            s, items, nitems, upds, cnt, ticket, abort_word, L, U, tinv, tinv_off, thr, npiv, err);
    else
        dag_bottom_kernel<T, FACTO_SYTRF><<<grid, 32 * DG_WARPS, smem, st>>>(
            s, items, nitems, upds, cnt, ticket, abort_word, L, U, tinv, tinv_off, thr, npiv, err);
}
template void launch_dag_bottom<double>(int, const DevSym &, int, const DagItem *, int, const Upd *, int *, int *,
                                        int *, double *, double *, double *, const int64_t *, const double *,
                                        unsigned long long *, int *, cudaStream_t);
template void launch_dag_bottom<float>(int, const DevSym &, int, const DagItem *, int, const Upd *, int *, int *,
                                       int *, float *, float *, float *, const int64_t *, const double *,
                                       unsigned long long *, int *, cudaStream_t);

// Grid of the tree-bottom launch: the CTAs resident at once (more would only queue
// behind them), at most one warp per item.
int dag_bottom_grid(int facto, bool f32, int ncblk) {
    if (ncblk <= 0) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = dag_bottom_smem(facto, f32 ? 4 : 8);
    cudaError_t e;
    if (f32)
        e = facto == FACTO_POTRF   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dag_bottom_kernel<float, FACTO_POTRF>, 32 * DG_WARPS, smem)
            : facto == FACTO_GETRF ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dag_bottom_kernel<float, FACTO_GETRF>, 32 * DG_WARPS, smem)
                                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dag_bottom_kernel<float, FACTO_SYTRF>, 32 * DG_WARPS, smem);
    else
        e = facto == FACTO_POTRF   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dag_bottom_kernel<double, FACTO_POTRF>, 32 * DG_WARPS, smem)
            : facto == FACTO_GETRF ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dag_bottom_kernel<double, FACTO_GETRF>, 32 * DG_WARPS, smem)
                                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dag_bottom_kernel<double, FACTO_SYTRF>, 32 * DG_WARPS, smem);
    if (e != cudaSuccess || per_sm <= 0 || sms <= 0) return -1;
    return std::min(per_sm * sms, (ncblk + DG_WARPS - 1) / DG_WARPS);
}

template <typename T>
void launch_diag(int facto, const DevSym &s, const int *cblks, int ncblk, T *L, T *U, T *tinv,
                 const int64_t *tinv_off, const double *thr, unsigned long long *npiv, int *err, cudaStream_t st) {
    if (ncblk <= 0) return;
    const size_t smem = (sizeof(T) == 4) ? 8 * 32 * 33 * sizeof(float) : 0;
    if (facto == FACTO_POTRF)
        diag_factor_kernel<T, FACTO_POTRF><<<ncblk, 256, smem, st>>>(s, cblks, L, U, tinv, tinv_off, thr, npiv, err);
    else if (facto == FACTO_GETRF)
        diag_factor_kernel<T, FACTO_GETRF><<<ncblk, 256, smem, st>>>(s, cblks, L, U, tinv, tinv_off, thr, npiv, err);
    else
        diag_factor_kernel<T, FACTO_SYTRF><<<ncblk, 256, smem, st>>>(s, cblks, L, U, tinv, tinv_off, thr, npiv, err);
}

template <typename T>
void launch_trsm(const DevSym &s, const RowTask *tasks, int ntasks, int TR, int nmax, T *P, const T *D, int mode,
                 const T *tinv, const int64_t *tinv_off, int which, int getrf, int scale_d, cudaStream_t st) {
    if (ntasks <= 0) return;
    const size_t smem = (size_t)TR * nmax * sizeof(T);
    panel_trsm_kernel<T><<<ntasks, 256, smem, st>>>(s, tasks, TR, P, D, mode, tinv, tinv_off, which, getrf, scale_d);
}

void launch_update_f64(const DevSym &s, const Upd *upds, int nupd, int ntiles, double *L, double *U,
                       cudaStream_t st) {
    if (ntiles <= 0) return;
    update_f64_kernel<<<ntiles, 128, UPD_F64_SMEM, st>>>(s, upds, nupd, L, U);
}

void launch_update_f32(const DevSym &s, const Upd *upds, int nupd, int ntiles, float *L, float *U,
                       cudaStream_t st) {
    if (ntiles <= 0) return;
    update_simt_f32_kernel<<<ntiles, 256, 0, st>>>(s, upds, nupd, L, U);
}

// Raise the dynamic shared-memory limit of a kernel to what the device allows
// beyond its static shared memory; returns that limit (bytes) or -1.
template <typename K>
static int raise_smem(K kernel) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return -1;
    const int dyn = optin - (int)fa.sharedSizeBytes;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess) return -1;
    return dyn;
}

// every instance of one width class (GETRF in FP64 needs more than the default 48 KB
// from 16 columns on)
template <int NB>
static int raise_diag_small_smem() {
    if (raise_smem(diag_small_kernel<double, FACTO_POTRF, NB>) < 0 ||
        raise_smem(diag_small_kernel<double, FACTO_SYTRF, NB>) < 0 ||
        raise_smem(diag_small_kernel<double, FACTO_GETRF, NB>) < 0 ||
        raise_smem(diag_small_kernel<float, FACTO_POTRF, NB>) < 0 ||
        raise_smem(diag_small_kernel<float, FACTO_SYTRF, NB>) < 0 ||
        raise_smem(diag_small_kernel<float, FACTO_GETRF, NB>) < 0)
        return -1;
    return 0;
}

int configure_factor_kernels() {
    int lim = 1 << 30;
    int v;
    if ((v = raise_smem(update_f64_kernel)) < UPD_F64_SMEM) return -1;
    if (raise_diag_small_smem<8>() < 0 || raise_diag_small_smem<16>() < 0 || raise_diag_small_smem<32>() < 0)
        return -1;
    if (raise_smem(dag_bottom_kernel<double, FACTO_POTRF>) < 0 || raise_smem(dag_bottom_kernel<double, FACTO_SYTRF>) < 0 ||
        raise_smem(dag_bottom_kernel<double, FACTO_GETRF>) < 0 || raise_smem(dag_bottom_kernel<float, FACTO_POTRF>) < 0 ||
        raise_smem(dag_bottom_kernel<float, FACTO_SYTRF>) < 0 || raise_smem(dag_bottom_kernel<float, FACTO_GETRF>) < 0)
        return -1;
    if ((v = raise_smem(panel_trsm_kernel<double>)) < 0) return -1;
    lim = std::min(lim, v);
    if ((v = raise_smem(panel_trsm_kernel<float>)) < 0) return -1;
    lim = std::min(lim, v);
    return lim;
}

template void launch_scatter<double>(int64_t, const int64_t *, const double *, const double *, double *, double *,
                                     cudaStream_t);
template void launch_scatter<float>(int64_t, const int64_t *, const double *, const double *, float *, float *,
                                    cudaStream_t);
template void launch_diag<double>(int, const DevSym &, const int *, int, double *, double *, double *,
                                  const int64_t *, const double *, unsigned long long *, int *, cudaStream_t);
template void launch_diag<float>(int, const DevSym &, const int *, int, float *, float *, float *, const int64_t *,
                                 const double *, unsigned long long *, int *, cudaStream_t);
template void launch_trsm<double>(const DevSym &, const RowTask *, int, int, int, double *, const double *, int,
                                  const double *, const int64_t *, int, int, int, cudaStream_t);
template void launch_trsm<float>(const DevSym &, const RowTask *, int, int, int, float *, const float *, int,
                                 const float *, const int64_t *, int, int, int, cudaStream_t);

}  // namespace b200
