// Supernodal triangular solve kernels (sm_100a).  The vectors of the sweeps are
// in the factor's precision V (double for the FP64 factor; float for the FP32
// factor, whose solves precondition an FP64 refinement); permutation and the
// conversions at the ends of a solve stay in double.
//
//  solve_mm_kernel          64 x 64 tiles of the panels (b[f] -= A_blk x[k],
//                           solve_blok_zgemm, kernels/solve_ztrsmsp.c:275-280, and
//                           its transpose) and of the diagonal-block inverses
//  solve_leaf_kernel        cblks of <= 32 columns, one warp each
//  solve_scale_diag_kernel  b /= D (solve_cblk_zdiag, kernels/solve_ztrsmsp.c:584-633)
//  permute_kernel           bvec_zlapmr with peritab (bcsc/bvec_zcompute.c:875)
//  convert_kernel           double <-> float copies of a vector block
#include <atomic>
#include "b200_internal.h"
#include "kernels.h"
#include "tile_ops.cuh"

namespace b200 {

__device__ __forceinline__ int panel_row_to_global(const DevSym &s, int k, int prow) {
    return s.prow[s.rbase[k] + prow];
}

template <typename T, typename V>
__global__ void solve_scale_diag_kernel(DevSym s, const int *__restrict__ cblks, const T *__restrict__ L, V *x,
                                        int64_t ldx, int nrhs) {
    const int k = cblks[blockIdx.x];
    const int n = s.ncols[k], ld = s.ld[k];
    const T *D = L + s.off[k];
    V *xk = x + s.fcol[k];
    for (int idx = threadIdx.x; idx < n * nrhs; idx += blockDim.x) {
        const int i = idx % n, r = idx / n;
        xk[i + (size_t)r * ldx] /= (V)D[(size_t)i * (ld + 1)];
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

template <typename S, typename D>
__global__ void convert_kernel(int n, int nrhs, const S *__restrict__ src, int64_t lds, D *__restrict__ dst,
                               int64_t ldd) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * nrhs) return;
    const int i = (int)(idx % n), r = (int)(idx / n);
    dst[i + r * ldd] = (D)src[i + r * lds];
}

template <typename T, typename V>
void launch_solve_scale_diag(const DevSym &s, const int *cblks, int ncblk, const T *L, V *x, int64_t ldx, int nrhs,
                             cudaStream_t st) {
    if (ncblk <= 0) return;
    solve_scale_diag_kernel<T, V><<<ncblk, 128, 0, st>>>(s, cblks, L, x, ldx, nrhs);
}

void launch_permute(int n, int nrhs, const int *peri, const double *src, int64_t lds, double *dst, int64_t ldd,
                    int forward, cudaStream_t st) {
    const int64_t tot = (int64_t)n * nrhs;
    if (tot <= 0) return;
    permute_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, nrhs, peri, src, lds, dst, ldd, forward);
}

template <typename S, typename D>
void launch_convert(int n, int nrhs, const S *src, int64_t lds, D *dst, int64_t ldd, cudaStream_t st) {
    const int64_t tot = (int64_t)n * nrhs;
    if (tot <= 0) return;
    convert_kernel<S, D><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, nrhs, src, lds, dst, ldd);
}

int configure_solve_kernels() { return 0; }

template void launch_solve_scale_diag<double, double>(const DevSym &, const int *, int, const double *, double *,
                                                      int64_t, int, cudaStream_t);
template void launch_solve_scale_diag<float, float>(const DevSym &, const int *, int, const float *, float *, int64_t,
                                                    int, cudaStream_t);
template void launch_convert<double, float>(int, int, const double *, int64_t, float *, int64_t, cudaStream_t);
template void launch_convert<float, double>(int, int, const float *, int64_t, double *, int64_t, cudaStream_t);

}  // namespace b200

// ====================================================================== tensor-core solve tiles
//
// The off-diagonal and diagonal-inverse products of the supernodal solves as
// small GEMMs on tensor cores, one CTA (4 warps) per 64 x 64 tile of the factor
// (or of a diagonal-block inverse W) times 16 (FP32) or 32 (FP64) right-hand sides
// per pass:
//   OFF_FWD : b[grow(r)] -= sum_c P[r][c] x_k[c]     (solve_blok_zgemm forward,
//             kernels/solve_ztrsmsp.c:275-280; warp = 16 rows)
//   OFF_BWD : b_k[c]     -= sum_r P[r][c] x[grow(r)] (backward; warp = 16 columns)
//   DIAG_FWD: out_k[r]   += sum_c W[r][c] in_k[c]     (W = L_kk^{-1}, lower)
//   DIAG_BWD: out_k[c]   += sum_r W[r][c] in_k[r]     (W^T, upper)
// FP64 vectors: DMMA m16n8k16.  FP32 vectors (FP32 factor): 3xTF32 mma.sync
// m16n8k8 (x = hi + lo, hi the TF32 part; hi*hi + hi*lo + lo*hi), FP32-accurate.
// The factor tile is staged in shared memory with cp.async (every load of the tile
// in flight at once, zero fill outside the panel), so a tile costs about one memory
// latency; partial sums meet in global memory through atomics.
namespace b200 {

constexpr int STT = 64;          // tile rows / columns
constexpr int SM_FWD = 72;       // pitch of a staged tile read row-wise by the fragments
constexpr int SM_BWD = 68;       // pitch of a staged tile read column-wise
enum { OFF_FWD = 0, OFF_BWD = 1, DIAG_FWD = 2, DIAG_BWD = 3 };

// Right-hand sides per pass (R) and the padded row of the staged x tile (P,
// conflict-free fragment reads): 16 for FP32 vectors, so that a CTA's shared
// memory stays at 24 KB (9 CTAs per SM), 32 for FP64.
template <typename V>
struct XPitch {
    static constexpr int R = sizeof(V) == 8 ? 32 : 16;
    static constexpr int P = sizeof(V) == 8 ? R + 4 : R + 8;
};

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

// The same tile in 16-byte chunks when every column of M starts on a 16-byte
// boundary (ldm a multiple of 16 / sizeof(T) and M aligned): the rows from gr0
// rounded down to a chunk boundary are copied as they are (chunks past nr zero
// filled), so the tile starts at ms + shift with shift = gr0 % (16 / sizeof(T)) < 4;
// a column takes at most 68 entries of its PM >= 68.  Returns shift.
template <typename T, int PM>
__device__ __forceinline__ int stage_tile16(T *ms, const T *M, int64_t ldm, int gr0, int gc0, int nr, int nc) {
    constexpr int EPV = 16 / sizeof(T);
    const int shift = gr0 % EPV, gr0a = gr0 - shift;
    const int cpc = (STT + shift + EPV - 1) / EPV;  // chunks per column
    for (int idx = threadIdx.x; idx < STT * cpc; idx += blockDim.x) {
        const int c = idx / cpc, i = idx % cpc;
        const int row = gr0a + i * EPV;
        int bytes = 0;
        if (gc0 + c < nc && row < nr) bytes = (nr - row >= EPV ? EPV : nr - row) * (int)sizeof(T);
        const T *src = bytes ? M + row + (size_t)(gc0 + c) * ldm : M;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sm_addr(ms + c * PM + i * EPV)), "l"(src),
                     "r"(bytes));
    }
    return shift;
}

// x tile: xs[i * XP + j] = xv[i][q0 + j] for i < ni, j < R (zeros elsewhere); rows
// either contiguous from xv (rowmap null) or gathered through rowmap.
template <typename V>
__device__ __forceinline__ void stage_x(V *xs, const V *xv, const int *rowmap, int ni, int64_t ldx, int q0, int R) {
    constexpr int XP = XPitch<V>::P;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int i0 = lane, i1 = lane + 32;
    const bool ok0 = i0 < ni, ok1 = i1 < ni;
    const V *x0 = xv + (ok0 ? (rowmap ? rowmap[i0] : i0) : 0);
    const V *x1 = xv + (ok1 ? (rowmap ? rowmap[i1] : i1) : 0);
    // columns j >= R are not staged: an output column of the products reads only its
    // own x column, and those outputs are discarded
    for (int j = w; j < R; j += nw) {
        cp_async_el(xs + i0 * XP + j, x0 + (size_t)(q0 + j) * ldx, ok0);
        cp_async_el(xs + i1 * XP + j, x1 + (size_t)(q0 + j) * ldx, ok1);
    }
}

// D += A B, A 16 x 16 (a[2j], a[2j+1] = rows g, g + 8 of column 4j + tg), B 16 x 8
// (b[j] = row 4j + tg, column g), the fragment layout of four m16n8k4 steps.
__device__ __forceinline__ void dmma16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
          "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// D += A B on TF32 operands, A 16 x 8 (a0..a3 = (g, tg), (g + 8, tg), (g, tg + 4),
// (g + 8, tg + 4)), B 8 x 8 (b0, b1 = (tg, g), (tg + 4, g)), FP32 accumulation.
__device__ __forceinline__ void mma_tf32_16x8x8(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// x = hi + lo with hi = x with its 13 low mantissa bits cleared (exact in TF32)
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo) {
    hi = __float_as_uint(x) & 0xFFFFE000u;
    lo = __float_as_uint(x - __uint_as_float(hi));
}

// acc += M_tile(op) x_tile over 64 K values; ROW = 1: output index = tile row
// (a fragment reads ms[k * PM + out]), ROW = 0: output index = tile column
// (ms[out * PM + k]).
template <typename T, int PM, int ROW>
__device__ __forceinline__ void tile_mma(double (&acc)[4][4], const T *ms, const double *xs, int o0w, int ntn) {
    constexpr int XP = XPitch<double>::P;
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
                for (int j = 0; j < 4; j++) b[j] = xs[(kk + 4 * j + tg) * XP + nt * 8 + g];
                dmma16x8x16(acc[nt], a, b);
            }
        }
    }
}

template <typename T, int PM, int ROW>
__device__ __forceinline__ void tile_mma(float (&acc)[4][4], const T *ms, const float *xs, int o0w, int ntn) {
    constexpr int XP = XPitch<float>::P;
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
    // the hi*hi products and the two correction terms in separate accumulators: two
    // shorter dependency chains per output tile instead of one of three MMAs
    float cor[4][4] = {};
#pragma unroll 2
    for (int kk = 0; kk < STT; kk += 8) {
        uint32_t ah[4], al[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int kq = kk + tg + 4 * (j >> 1), o = o0w + g + 8 * (j & 1);
            tf32_split((float)(ROW ? ms[kq * PM + o] : ms[o * PM + kq]), ah[j], al[j]);
        }
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            if (nt < ntn) {
                uint32_t bh[2], bl[2];
                tf32_split(xs[(kk + tg) * XP + nt * 8 + g], bh[0], bl[0]);
                tf32_split(xs[(kk + tg + 4) * XP + nt * 8 + g], bh[1], bl[1]);
                mma_tf32_16x8x8(acc[nt], ah, bh);
                mma_tf32_16x8x8(cor[nt], ah, bl);
                mma_tf32_16x8x8(cor[nt], al, bh);
            }
        }
    }
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[nt][e] += cor[nt][e];
}

template <typename T, typename V, int MODE>
struct SolveSmem {
    static constexpr int PM = (MODE == OFF_FWD || MODE == DIAG_FWD) ? SM_FWD : SM_BWD;
    static constexpr int BYTES = STT * PM * (int)sizeof(T) + STT * XPitch<V>::P * (int)sizeof(V);
};

// One 64 x 64 tile times 16 (FP32) or 32 (FP64) right-hand sides per pass.  Task {k, row0, col0}:
//   OFF_*  : panel rows [row0, row0 + 64) x columns [col0, col0 + 64) of cblk k
//   DIAG_* : output tile [row0, row0 + 64) of cblk k, K chunk [col0, col0 + 64) of
//            W_k (forward) or W_k^T (backward); the output (zeroed before the sweep)
//            accumulates the chunks through atomics.
template <typename T, typename V, int MODE>
__global__ void __launch_bounds__(128) solve_mm_kernel(DevSym s, const SolveTile *__restrict__ tasks,
                                                       const T *__restrict__ M, const int64_t *__restrict__ woff,
                                                       const V *xin, V *out, int64_t ldx, int nrhs) {
    using SS = SolveSmem<T, V, MODE>;
    constexpr int PM = SS::PM;
    constexpr bool ROW = (MODE == OFF_FWD || MODE == DIAG_FWD);
    extern __shared__ __align__(16) unsigned char sv_smem[];
    T *ms = reinterpret_cast<T *>(sv_smem);
    V *xs = reinterpret_cast<V *>(sv_smem + STT * PM * sizeof(T));
    __shared__ int rmap[STT];
    const SolveTile t = tasks[blockIdx.x];
    const int k = t.k, n = s.ncols[k];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int o0w = warp * 16;  // this warp's 16 outputs of the tile
    int nout;
    const V *xsrc;
    const int *xmap = nullptr;
    int nk;
    int shift = 0;  // the staged tile starts at ms + shift
    if (MODE == OFF_FWD || MODE == OFF_BWD) {
        const int rows = min(STT, s.stride[k] - t.row0), cols = min(STT, n - t.col0);
        // the tile's copies first: the row map's loads then overlap them
        shift = stage_tile16<T, PM>(ms, M + s.off[k], s.ld[k], t.row0, t.col0, s.stride[k], n);
        if (tid < STT) rmap[tid] = (tid < rows) ? panel_row_to_global(s, k, t.row0 + tid) : 0;
        __syncthreads();
        nout = ROW ? rows : cols;
        nk = ROW ? cols : rows;
        if (MODE == OFF_FWD) xsrc = xin + s.fcol[k] + t.col0;
        else { xsrc = xin; xmap = rmap; }
    } else {
        const T *Wk = M + woff[k];
        nout = min(STT, n - t.row0);
        nk = min(STT, n - t.col0);
        if (n % (16 / (int)sizeof(T)) == 0) {
            if (MODE == DIAG_FWD) shift = stage_tile16<T, PM>(ms, Wk, n, t.row0, t.col0, n, n);  // W[o][k]
            else shift = stage_tile16<T, PM>(ms, Wk, n, t.col0, t.row0, n, n);                   // W[k][o]
        } else {
            if (MODE == DIAG_FWD) stage_tile<T, PM>(ms, Wk, n, t.row0, t.col0, n, n);
            else stage_tile<T, PM>(ms, Wk, n, t.col0, t.row0, n, n);
        }
        xsrc = xin + s.fcol[k] + t.col0;
    }
    for (int q0 = 0; q0 < nrhs; q0 += XPitch<V>::R) {
        const int R = min(XPitch<V>::R, nrhs - q0), ntn = (R + 7) >> 3;
        if (q0 > 0) __syncthreads();
        stage_x<V>(xs, xsrc, xmap, nk, ldx, q0, R);
        cp_commit();
        cp_wait<0>();
        __syncthreads();
        if (o0w < nout) {
            V acc[4][4] = {};
            tile_mma<T, PM, ROW>(acc, ms + shift, xs, o0w, ntn);
            const V sg = (MODE == OFF_FWD || MODE == OFF_BWD) ? (V)-1 : (V)1;
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                if (nt >= ntn) continue;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int o = o0w + g + (e >> 1) * 8;
                    const int j = nt * 8 + 2 * tg + (e & 1);
                    if (o < nout && j < R) {
                        V *dst = (MODE == OFF_FWD)   ? out + rmap[o]
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

template <typename T, typename V>
__global__ void __launch_bounds__(128) solve_leaf_kernel(DevSym s, const int *__restrict__ cblks, int ncblk,
                                                         const T *__restrict__ P, const T *__restrict__ W,
                                                         const int64_t *__restrict__ woff, V *x, V *aux,
                                                         int64_t ldx, int nrhs, int backward) {
    __shared__ V ys[4][32][LEAF_R + 1];
    __shared__ V xr[4][32][LEAF_R + 1];
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
                ys[w][lane][j] = (lane < n && j < R) ? x[f0 + lane + (size_t)(q0 + j) * ldx] : (V)0;
            __syncwarp();
            V y[LEAF_R];
#pragma unroll
            for (int j = 0; j < LEAF_R; j++) y[j] = 0;
            if (lane < n) {
#pragma unroll 4
                for (int c = 0; c <= lane; c++) {
                    const V wv = (V)Wk[lane + (size_t)c * n];
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
                V acc[LEAF_R];
#pragma unroll
                for (int j = 0; j < LEAF_R; j++) acc[j] = 0;
#pragma unroll 4
                for (int c = 0; c < n; c++) {
                    const V pv = (V)Pk[r + (size_t)c * ld];
#pragma unroll
                    for (int j = 0; j < LEAF_R; j++) acc[j] += pv * ys[w][c][j];
                }
#pragma unroll
                for (int j = 0; j < LEAF_R; j++)
                    if (j < R) atomicAdd(&x[g + (size_t)(q0 + j) * ldx], -acc[j]);
            }
            __syncwarp();
        } else {
            V t[LEAF_R];
#pragma unroll
            for (int j = 0; j < LEAF_R; j++) t[j] = (lane < n && j < R) ? aux[f0 + lane + (size_t)(q0 + j) * ldx] : (V)0;
            for (int r0 = n; r0 < stride; r0 += 32) {
                const int nr = min(32, stride - r0);
                gr[w][lane] = (lane < nr) ? panel_row_to_global(s, k, r0 + lane) : 0;
                __syncwarp();
                // stage x of the 32 rows: xr[i][j] = x[grow(r0 + i)][q0 + j]
                for (int idx = lane; idx < 32 * LEAF_R; idx += 32) {
                    const int i = idx / LEAF_R, j = idx % LEAF_R;
                    xr[w][i][j] = (i < nr && j < R) ? x[gr[w][i] + (size_t)(q0 + j) * ldx] : (V)0;
                }
                __syncwarp();
                if (lane < n) {
#pragma unroll 4
                    for (int i = 0; i < nr; i++) {
                        const V pv = (V)Pk[r0 + i + (size_t)lane * ld];
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
                V o[LEAF_R];
#pragma unroll
                for (int j = 0; j < LEAF_R; j++) o[j] = 0;
                for (int r = lane; r < n; r++) {
                    const V wv = (V)Wk[r + (size_t)lane * n];
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

template <typename T, typename V>
void launch_solve_leaf(const DevSym &s, const int *cblks, int ncblk, const T *P, const T *W, const int64_t *woff,
                       V *x, V *aux, int64_t ldx, int nrhs, int backward, cudaStream_t st) {
    if (ncblk <= 0) return;
    solve_leaf_kernel<T, V><<<(ncblk + 3) / 4, 128, 0, st>>>(s, cblks, ncblk, P, W, woff, x, aux, ldx, nrhs, backward);
}
template void launch_solve_leaf<double, double>(const DevSym &, const int *, int, const double *, const double *,
                                                const int64_t *, double *, double *, int64_t, int, int, cudaStream_t);
template void launch_solve_leaf<float, float>(const DevSym &, const int *, int, const float *, const float *,
                                              const int64_t *, float *, float *, int64_t, int, int, cudaStream_t);

template <typename T, typename V>
void launch_solve_tiles(const DevSym &s, const SolveTile *tasks, int ntasks, const T *L, const V *x, V *b,
                        int64_t ldx, int nrhs, int backward, cudaStream_t st) {
    if (ntasks <= 0) return;
    if (!backward)
        solve_mm_kernel<T, V, OFF_FWD><<<ntasks, 128, SolveSmem<T, V, OFF_FWD>::BYTES, st>>>(s, tasks, L, nullptr, x, b,
                                                                                          ldx, nrhs);
    else
        solve_mm_kernel<T, V, OFF_BWD><<<ntasks, 128, SolveSmem<T, V, OFF_BWD>::BYTES, st>>>(s, tasks, L, nullptr, x, b,
                                                                                          ldx, nrhs);
}

template <typename T, typename V, int MODE>
void solve_diag_mm(const DevSym &s, const SolveTile *tasks, int ntasks, const T *W, const int64_t *woff, const V *xin,
                   V *xout, int64_t ldx, int nrhs, cudaStream_t st) {
    solve_mm_kernel<T, V, MODE><<<ntasks, 128, SolveSmem<T, V, MODE>::BYTES, st>>>(s, tasks, W, woff, xin, xout, ldx,
                                                                                  nrhs);
}

// dynamic shared memory of the staged solve kernels (above the 48 KB default)
template <typename T, typename V>
int configure_solve_mm() {
    int rc = 0;
    rc |= (int)cudaFuncSetAttribute(solve_mm_kernel<T, V, OFF_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SolveSmem<T, V, OFF_FWD>::BYTES);
    rc |= (int)cudaFuncSetAttribute(solve_mm_kernel<T, V, OFF_BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SolveSmem<T, V, OFF_BWD>::BYTES);
    rc |= (int)cudaFuncSetAttribute(solve_mm_kernel<T, V, DIAG_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SolveSmem<T, V, DIAG_FWD>::BYTES);
    rc |= (int)cudaFuncSetAttribute(solve_mm_kernel<T, V, DIAG_BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SolveSmem<T, V, DIAG_BWD>::BYTES);
    return rc;
}

template void launch_solve_tiles<double, double>(const DevSym &, const SolveTile *, int, const double *,
                                                 const double *, double *, int64_t, int, int, cudaStream_t);
template void launch_solve_tiles<float, float>(const DevSym &, const SolveTile *, int, const float *, const float *,
                                               float *, int64_t, int, int, cudaStream_t);

// ---------------------------------------------------------------- dataflow sweeps
//
// One sweep in one launch: the products above as items taken in a fixed order
// (level by level; the forward sweep bottom-up, the backward sweep top-down) from
// an atomic ticket by persistent CTAs, each item waiting only for the inputs it
// reads instead of for the whole previous level (solve_cblk_ztrsmsp_forward /
// _backward, kernels/solve_ztrsmsp.c, scheduled by the cblks' contributions as
// PaStiX's dynamic solve does).  Counters in global memory, per cblk:
//   forward : cnt_a[f] items that have subtracted into x_f (complete at need[f]);
//             cnt_b[k] diagonal items of k done (aux_k complete at ndiag[k]);
//   backward: cnt_a[f] items that have written x_f (final at need[f]);
//             cnt_b[k] off-diagonal items of k done (aux_k complete at noff[k]).
// Items:
//   FI_LEAF up to 16 cblks of <= 32 columns of one level, a warp at a time (the
//           leaf products above); forward: raises cnt_a of the facing cblks in its
//           list; backward: waits for them, then raises cnt_a of its own cblks;
//   FI_DIAG output rows [r0, r0 + 64), K chunk [c0, c0 + 64) of W_k x_k into aux_k
//           (forward) / W_k^T aux_k into x_k (backward), both zeroed before the sweep;
//   FI_OFF  panel rows [r0, r0 + 64), columns [c0, c0 + 64) of cblk k: forward
//           x[rows] -= P aux_k, raising the facing cblks' cnt_a; backward
//           aux_k -= P^T x[rows] after the facing cblks are final.
// Partial products meet through atomics, as in the level-synchronous tiles.
// Values other items write are read through L2 (ld.cg): an L1 line could hold a
// neighbouring cblk's entries from before they were final.  Every wait is bounded;
// on expiry the CTA sets bit 4 of err and an abort word that ends the others'
// waits.
constexpr int FLOW_THREADS = 128;

namespace {

constexpr long long FLOW_WAIT_CYCLES = 1000000000LL;  // about 0.5 s at the maximum SM clock

__device__ __forceinline__ int flow_ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool flow_wait(const int *c, int target, const int *abort_word) {
    const long long t0 = clock64();
    for (int it = 0;; it++) {
        if (flow_ld_acquire(c) >= target) return true;
        if ((it & 15) == 15) {
            if (flow_ld_acquire(abort_word)) return false;
            if (clock64() - t0 > FLOW_WAIT_CYCLES) return false;
        }
        __nanosleep(64);
    }
}

// x tile through L2: xs[i * XP + j] = xv[row(i)][q0 + j], zeros outside
template <typename V, int NT>
__device__ __forceinline__ void stage_x_cg(V *xs, const V *xv, const int *rowmap, int ni, int64_t ldx, int q0, int R) {
    constexpr int XP = XPitch<V>::P;
    stage_n<STT * XPitch<V>::R / NT, V>(
        [&](int u) {
            const int idx = threadIdx.x + NT * u, i = idx % STT, j = idx / STT;
            return (i < ni && j < R) ? __ldcg(xv + (rowmap ? rowmap[i] : i) + (size_t)(q0 + j) * ldx) : (V)0;
        },
        [&](int u, V v) {
            const int idx = threadIdx.x + NT * u;
            xs[(idx % STT) * XP + idx / STT] = v;
        });
}

}  // namespace

template <typename T, typename V>
struct FlowSmem {
    static constexpr int TILE = STT * SM_FWD * (int)sizeof(T) + STT * XPitch<V>::P * (int)sizeof(V);
    static constexpr int LEAF = 2 * 4 * 32 * (LEAF_R + 1) * (int)sizeof(V);
    static constexpr int BYTES = TILE > LEAF ? TILE : LEAF;
};

template <typename T, typename V, int BWD>
__global__ void __launch_bounds__(FLOW_THREADS) solve_flow_kernel(DevSym s, const FlowItem *__restrict__ items,
                                                                  int nitems, const int *__restrict__ leaf,
                                                                  const int *__restrict__ flist,
                                                                  const int *__restrict__ need,
                                                                  const int *__restrict__ nprev, const T *P,
                                                                  const T *W, const int64_t *__restrict__ woff, V *x,
                                                                  V *aux, int64_t ldx, int nrhs, int *ticket,
                                                                  int *cnt_a, int *cnt_b, int *abort_word, int *err) {
    extern __shared__ __align__(16) unsigned char fl_smem[];
    __shared__ int rmap[STT];
    __shared__ int s_item, s_ok;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int o0w = warp * 16;
    bool aborted = false;
    for (;;) {
        if (tid == 0) {
            s_item = atomicAdd(ticket, 1);
            s_ok = 1;
        }
        __syncthreads();
        const int t = s_item;
        if (t >= nitems) break;
        const FlowItem it = items[t];
        // ------------------------------------------------------------ inputs complete
        if (tid == 0) {
            if (it.type == FI_LEAF) {
                if (!BWD) {
                    for (int i = 0; i < it.n && s_ok; i++) {
                        const int kk = leaf[it.k + i];
                        if (!flow_wait(cnt_a + kk, need[kk], abort_word)) s_ok = 0;
                    }
                } else {
                    for (int i = 0; i < it.nf && s_ok; i++) {
                        const int f = flist[it.f0 + i];
                        if (!flow_wait(cnt_a + f, need[f], abort_word)) s_ok = 0;
                    }
                }
            } else if (it.type == FI_DIAG) {
                if (!flow_wait(BWD ? cnt_b + it.k : cnt_a + it.k, BWD ? nprev[it.k] : need[it.k], abort_word)) s_ok = 0;
            } else {
                if (!BWD) {
                    if (!flow_wait(cnt_b + it.k, nprev[it.k], abort_word)) s_ok = 0;
                } else {
                    for (int i = 0; i < it.nf && s_ok; i++) {
                        const int f = flist[it.f0 + i];
                        if (!flow_wait(cnt_a + f, need[f], abort_word)) s_ok = 0;
                    }
                }
            }
        }
        __syncthreads();
        if (!s_ok) {
            aborted = true;
            break;
        }
        if (it.type == FI_LEAF) {
            // ------------------------------------------------------------ leaf cblks
            V (*ys)[LEAF_R + 1] = reinterpret_cast<V (*)[LEAF_R + 1]>(fl_smem) + warp * 32;
            V (*xr)[LEAF_R + 1] = reinterpret_cast<V (*)[LEAF_R + 1]>(fl_smem) + 4 * 32 + warp * 32;
            for (int wi = warp; wi < it.n; wi += 4) {
                const int k = leaf[it.k + wi];
                const int n = s.ncols[k], ld = s.ld[k], stride = s.stride[k], f0 = s.fcol[k];
                const T *Pk = P + s.off[k];
                const T *Wk = W + woff[k];
                for (int q0 = 0; q0 < nrhs; q0 += LEAF_R) {
                    const int R = min(LEAF_R, nrhs - q0);
                    if (!BWD) {
#pragma unroll
                        for (int j = 0; j < LEAF_R; j++)
                            ys[lane][j] = (lane < n && j < R) ? __ldcg(x + f0 + lane + (size_t)(q0 + j) * ldx) : (V)0;
                        __syncwarp();
                        V y[LEAF_R];
#pragma unroll
                        for (int j = 0; j < LEAF_R; j++) y[j] = 0;
                        if (lane < n) {
                            for (int c = 0; c <= lane; c++) {
                                const V wv = (V)Wk[lane + (size_t)c * n];
#pragma unroll
                                for (int j = 0; j < LEAF_R; j++) y[j] += wv * ys[c][j];
                            }
                        }
                        __syncwarp();
                        if (lane < n) {
#pragma unroll
                            for (int j = 0; j < LEAF_R; j++) {
                                ys[lane][j] = y[j];
                                if (j < R) aux[f0 + lane + (size_t)(q0 + j) * ldx] = y[j];
                            }
                        }
                        __syncwarp();
                        for (int r = n + lane; r < stride; r += 32) {
                            const int gg = panel_row_to_global(s, k, r);
                            V acc[LEAF_R];
#pragma unroll
                            for (int j = 0; j < LEAF_R; j++) acc[j] = 0;
                            for (int c = 0; c < n; c++) {
                                const V pv = (V)Pk[r + (size_t)c * ld];
#pragma unroll
                                for (int j = 0; j < LEAF_R; j++) acc[j] += pv * ys[c][j];
                            }
#pragma unroll
                            for (int j = 0; j < LEAF_R; j++)
                                if (j < R) atomicAdd(&x[gg + (size_t)(q0 + j) * ldx], -acc[j]);
                        }
                        __syncwarp();
                    } else {
                        V tt[LEAF_R];
#pragma unroll
                        for (int j = 0; j < LEAF_R; j++)
                            tt[j] = (lane < n && j < R) ? __ldcg(aux + f0 + lane + (size_t)(q0 + j) * ldx) : (V)0;
                        for (int r0 = n; r0 < stride; r0 += 32) {
                            const int nr = min(32, stride - r0);
                            const int myg = (lane < nr) ? panel_row_to_global(s, k, r0 + lane) : 0;
                            for (int idx = lane; idx < 32 * LEAF_R; idx += 32) {
                                const int i = idx / LEAF_R, j = idx % LEAF_R;
                                const int gi = __shfl_sync(0xffffffffu, myg, i);
                                xr[i][j] = (i < nr && j < R) ? __ldcg(x + gi + (size_t)(q0 + j) * ldx) : (V)0;
                            }
                            __syncwarp();
                            if (lane < n) {
                                for (int i = 0; i < nr; i++) {
                                    const V pv = (V)Pk[r0 + i + (size_t)lane * ld];
#pragma unroll
                                    for (int j = 0; j < LEAF_R; j++) tt[j] -= pv * xr[i][j];
                                }
                            }
                            __syncwarp();
                        }
                        if (lane < n) {
#pragma unroll
                            for (int j = 0; j < LEAF_R; j++) ys[lane][j] = tt[j];
                        }
                        __syncwarp();
                        if (lane < n) {
                            V o[LEAF_R];
#pragma unroll
                            for (int j = 0; j < LEAF_R; j++) o[j] = 0;
                            for (int r = lane; r < n; r++) {
                                const V wv = (V)Wk[r + (size_t)lane * n];
#pragma unroll
                                for (int j = 0; j < LEAF_R; j++) o[j] += wv * ys[r][j];
                            }
#pragma unroll
                            for (int j = 0; j < LEAF_R; j++)
                                if (j < R) x[f0 + lane + (size_t)(q0 + j) * ldx] = o[j];
                        }
                        __syncwarp();
                    }
                }
            }
        } else {
            // ------------------------------------------------------------ one 64 x 64 tile
            T *ms = reinterpret_cast<T *>(fl_smem);
            V *xs = reinterpret_cast<V *>(fl_smem + STT * SM_FWD * sizeof(T));
            const int k = it.k, n = s.ncols[k], c0 = it.n;
            int nout, nk, shift = 0;
            const V *xsrc;
            const int *xmap = nullptr;
            if (it.type == FI_DIAG) {
                const T *Wk = W + woff[k];
                nout = min(STT, n - it.r0);
                nk = min(STT, n - c0);
                // forward W[o][kk] (row form); backward W[kk][o] (W^T, column form)
                if (n % (16 / (int)sizeof(T)) == 0) {
                    if (!BWD) shift = stage_tile16<T, SM_FWD>(ms, Wk, n, it.r0, c0, n, n);
                    else shift = stage_tile16<T, SM_BWD>(ms, Wk, n, c0, it.r0, n, n);
                } else {
                    if (!BWD) stage_tile<T, SM_FWD>(ms, Wk, n, it.r0, c0, n, n);
                    else stage_tile<T, SM_BWD>(ms, Wk, n, c0, it.r0, n, n);
                }
                xsrc = (BWD ? aux : x) + s.fcol[k] + c0;
            } else {
                const int rows = min(STT, s.stride[k] - it.r0), cols = min(STT, n - c0);
                if (tid < STT) rmap[tid] = (tid < rows) ? panel_row_to_global(s, k, it.r0 + tid) : 0;
                if (!BWD) shift = stage_tile16<T, SM_FWD>(ms, P + s.off[k], s.ld[k], it.r0, c0, s.stride[k], n);
                else shift = stage_tile16<T, SM_BWD>(ms, P + s.off[k], s.ld[k], it.r0, c0, s.stride[k], n);
                nout = BWD ? cols : rows;
                nk = BWD ? rows : cols;
                if (!BWD) xsrc = aux + s.fcol[k] + c0;
                else { xsrc = x; xmap = rmap; }
                __syncthreads();
            }
            cp_commit();
            for (int q0 = 0; q0 < nrhs; q0 += XPitch<V>::R) {
                const int R = min(XPitch<V>::R, nrhs - q0), ntn = (R + 7) >> 3;
                if (q0 > 0) __syncthreads();
                stage_x_cg<V, FLOW_THREADS>(xs, xsrc, xmap, nk, ldx, q0, R);
                cp_wait<0>();
                __syncthreads();
                if (o0w < nout) {
                    V acc[4][4] = {};
                    const bool row = !BWD;  // forward: outputs are tile rows; backward: tile columns
                    if (row) tile_mma<T, SM_FWD, 1>(acc, ms + shift, xs, o0w, ntn);
                    else tile_mma<T, SM_BWD, 0>(acc, ms + shift, xs, o0w, ntn);
                    // DIAG: + into aux_k (forward) / x_k (backward); OFF: - into x[rows] / aux_k
                    const V sg = it.type == FI_DIAG ? (V)1 : (V)-1;
                    V *dst;
                    if (it.type == FI_DIAG) dst = (BWD ? x : aux) + s.fcol[k] + it.r0;
                    else dst = BWD ? aux + s.fcol[k] + c0 : x;
#pragma unroll
                    for (int nt = 0; nt < 4; nt++) {
                        if (nt >= ntn) continue;
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const int o = o0w + g + (e >> 1) * 8;
                            const int j = nt * 8 + 2 * tg + (e & 1);
                            if (o < nout && j < R) {
                                const int row_o = (it.type == FI_OFF && !BWD) ? rmap[o] : o;
                                atomicAdd(dst + row_o + (size_t)(q0 + j) * ldx, sg * acc[nt][e]);
                            }
                        }
                    }
                }
            }
        }
        // ------------------------------------------------------------ announce
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            if (it.type == FI_LEAF) {
                if (!BWD)
                    for (int i = 0; i < it.nf; i++) atomicAdd(cnt_a + flist[it.f0 + i], 1);
                else
                    for (int i = 0; i < it.n; i++) atomicAdd(cnt_a + leaf[it.k + i], 1);
            } else if (it.type == FI_DIAG) {
                atomicAdd(BWD ? cnt_a + it.k : cnt_b + it.k, 1);
            } else {
                if (!BWD)
                    for (int i = 0; i < it.nf; i++) atomicAdd(cnt_a + flist[it.f0 + i], 1);
                else
                    atomicAdd(cnt_b + it.k, 1);
            }
        }
    }
    if (aborted && tid == 0) {
        atomicOr(err, 16);
        atomicExch(abort_word, 1);
    }
}

template <typename T, typename V>
void launch_solve_flow(const DevSym &s, const FlowItem *items, int nitems, const int *leaf, const int *flist,
                       const int *need, const int *nprev, const T *P, const T *W, const int64_t *woff, V *x, V *aux,
                       int64_t ldx, int nrhs, int backward, int *ticket, int *cnt_a, int *cnt_b, int *abort_word,
                       int *err, cudaStream_t st) {
    if (nitems <= 0) return;
    // resident CTAs of the launch, computed once (calls on several streams may race
    // to compute it; they store the same value)
    static std::atomic<int> ctas[2] = {{0}, {0}};
    const int bi = backward ? 1 : 0;
    const int smem = FlowSmem<T, V>::BYTES;
    if (!ctas[bi].load()) {
        int dev = 0, sms = 0, occ = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (backward) {
            cudaFuncSetAttribute(solve_flow_kernel<T, V, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, solve_flow_kernel<T, V, 1>, FLOW_THREADS, smem);
        } else {
            cudaFuncSetAttribute(solve_flow_kernel<T, V, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, solve_flow_kernel<T, V, 0>, FLOW_THREADS, smem);
        }
        ctas[bi].store(std::max(occ, 1) * std::max(sms, 1));
    }
    const int grid = std::min(nitems, ctas[bi].load());
    if (backward)
        solve_flow_kernel<T, V, 1><<<grid, FLOW_THREADS, smem, st>>>(s, items, nitems, leaf, flist, need, nprev, P, W,
                                                                    woff, x, aux, ldx, nrhs, ticket, cnt_a, cnt_b,
                                                                    abort_word, err);
    else
        solve_flow_kernel<T, V, 0><<<grid, FLOW_THREADS, smem, st>>>(s, items, nitems, leaf, flist, need, nprev, P, W,
                                                                    woff, x, aux, ldx, nrhs, ticket, cnt_a, cnt_b,
                                                                    abort_word, err);
}

template void launch_solve_flow<double, double>(const DevSym &, const FlowItem *, int, const int *, const int *,
                                                const int *, const int *, const double *, const double *,
                                                const int64_t *, double *, double *, int64_t, int, int, int *, int *,
                                                int *, int *, int *, cudaStream_t);
template void launch_solve_flow<float, float>(const DevSym &, const FlowItem *, int, const int *, const int *,
                                              const int *, const int *, const float *, const float *, const int64_t *,
                                              float *, float *, int64_t, int, int, int *, int *, int *, int *, int *,
                                              cudaStream_t);

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
__global__ void __launch_bounds__(128, 3) diag_inverse_kernel(DevSym s, const int *__restrict__ cblks,
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
        stage_n<32, double>(
            [&](int j) {
                return (lane < bw && j < bw && lane >= j) ? (double)Tk[(b0 + lane) + (size_t)(b0 + j) * ld] : 0.0;
            },
            [&](int j, double v) { ta[lane + j * TP] = v; });
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
                stage_n<32, double>(
                    [&](int j) {
                        return (lane < iw && j < mw) ? (double)Tk[(i0 + lane) + (size_t)(m0 + j) * ld] : 0.0;
                    },
                    [&](int j, double v) { ta[lane + j * TP] = v; });
                stage_n<32, double>(
                    [&](int j) { return (lane < mw && j < jw) ? (double)Wk[(m0 + lane) + (size_t)(j0 + j) * n] : 0.0; },
                    [&](int j, double v) { tb[lane + j * TP] = v; });
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
            stage_n<32, double>(
                [&](int j) {
                    return (lane < iw && j < iw && lane >= j) ? (double)Wk[(i0 + lane) + (size_t)(i0 + j) * n] : 0.0;
                },
                [&](int j, double v) { tb[lane + j * TP] = v; });
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

template <typename T, typename V>
void launch_solve_diag_inv(const DevSym &s, const SolveTile *tasks, int ntasks, const T *W, const int64_t *woff,
                           const V *xin, V *xout, int64_t ldx, int nrhs, int backward, cudaStream_t st) {
    if (ntasks <= 0) return;
    if (!backward) solve_diag_mm<T, V, DIAG_FWD>(s, tasks, ntasks, W, woff, xin, xout, ldx, nrhs, st);
    else solve_diag_mm<T, V, DIAG_BWD>(s, tasks, ntasks, W, woff, xin, xout, ldx, nrhs, st);
}

int configure_inverse_kernels() {
    int rc = configure_solve_mm<double, double>() | configure_solve_mm<float, float>();
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
template void launch_solve_diag_inv<double, double>(const DevSym &, const SolveTile *, int, const double *,
                                                    const int64_t *, const double *, double *, int64_t, int, int,
                                                    cudaStream_t);
template void launch_solve_diag_inv<float, float>(const DevSym &, const SolveTile *, int, const float *,
                                                  const int64_t *, const float *, float *, int64_t, int, int,
                                                  cudaStream_t);

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
