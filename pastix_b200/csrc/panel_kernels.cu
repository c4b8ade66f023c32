// Panel factorization of the wide POTRF / LDL^T cblks of one level, in one launch.
//
// PaStiX factors a cblk's diagonal block with its blocked kernel and then solves
// the whole panel below it (cpucblk_zpotrfsp1d_panel, kernels/core_zpotrfsp.c:284-295:
// core_zpotrfsp, kernels/core_zpotrfsp.c:66-100, then cpucblk_ztrsmsp;
// cpucblk_zsytrfsp1d_panel, kernels/core_zsytrfsp.c:424-446: core_zsytrfsp,
// kernels/core_zsytrfsp.c:63-103, then the solve against D L^T).  Here the same
// factorization runs right-looking over 64-column steps j, with the panel's rows
// cut into row blocks b of 64 rows: blocks 0 .. ns-1 are the rows of the diagonal
// block (block j holds the diagonal tile of step j), the others the rows below it.
//
// Items (j, b) with b >= j:
//   b == j  factor the diagonal tile of step j in shared memory (8-column leaves);
//   b >  j  solve the step's columns of row block b against that tile by
//           substitution (x_c = (a_c - sum_{l<c} x_l L_cl) / L_cc; LDL^T: unit L,
//           then division by D), then update the row block's columns right of the
//           step: A[b, c] -= L[b, j] (D_j) L[c, j]^T for every column block c > j
//           (c <= b among the diagonal block's rows; the lower triangle of tile (b, b)).
//
// Dependencies are counters in global memory, per row block: solved[b] = j + 1 once
// its columns of step j are final (for b == j: the factored tile), updated[b] = j + 1
// once its update of step j is done.  CTAs take items from an atomic ticket in a
// fixed order -- step by step, and within a step by row block (the critical tiles
// j and j + 1 of every cblk first) -- and every item depends only on items earlier
// in that order.  A CTA only ever waits for items that running CTAs have already
// taken, so the launch completes whatever the number of resident CTAs.  Every wait
// is bounded: on expiry the CTA sets bit 3 of err and an abort word that ends the
// other CTAs' waits, and returns.
//
// The solves of the tiles next to the critical path overlap with the rest of the
// step's rows and with the following steps (look-ahead without extra launches);
// the launch replaces three to four launches per 64-column step.
#include <algorithm>

#include "b200_internal.h"
#include "kernels.h"
#include "tile_ops.cuh"

namespace b200 {

namespace {

constexpr int PB = 64;   // tile edge
constexpr int LP = 65;   // pitch of the diagonal tile (column-major)
constexpr int XP = 68;   // pitch of the row block's columns (column-major, 16-byte aligned columns)
constexpr int RP = 64;   // pitch of a resident row block (column-major)
constexpr int PT = 256;  // threads per CTA
constexpr long long PANEL_WAIT_CYCLES = 1000000000LL;  // about 0.5 s at the maximum SM clock
constexpr int PANEL_SMEM_ELEMS = PB * LP + PB * XP + PB * PB + 3 * PB;

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait (one thread) until *flag >= target; false on expiry or abort.
__device__ bool panel_wait(const int *flag, int target, const int *abort_word) {
    const long long t0 = clock64();
    for (int it = 0;; it++) {
        if (ld_acquire(flag) >= target) return true;
        if ((it & 15) == 15) {
            if (ld_acquire(abort_word)) return false;
            if (clock64() - t0 > PANEL_WAIT_CYCLES) return false;
        }
        __nanosleep(100);
    }
}

template <typename T>
__device__ __forceinline__ void load4(const T *p, T v[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 q = *reinterpret_cast<const float4 *>(p);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else {
        const double2 q0 = *reinterpret_cast<const double2 *>(p), q1 = *reinterpret_cast<const double2 *>(p + 2);
        v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
    }
}

// Factor the wd x wd diagonal tile a (pitch LP, lower triangle) in place, by
// 8-column leaves, right-looking between leaves:
//   leaf   (warp 0): every lane factors the leaf's 8 x 8 diagonal block in registers
//          (the same values in every lane, no broadcasts), then its two rows below
//          it column by column; static pivoting replaces a pivot below thr in
//          magnitude by +-thr.  The pivot's square root is p * rsqrt(p) (within an
//          ulp of sqrt(p); rsqrt(p) scales the column).
//   update (all warps, warp w = trailing columns j = b + 8 + w, b + 16 + w, ...):
//          a_ij -= l_ik (d_k) l_jk for the leaf's columns k, k ascending.  Every entry
//          receives the factored columns' terms one by one in ascending k, leaf after
//          leaf: the same operations in the same order as a left-looking sum over all
//          earlier columns, spread over the CTA's warps instead of one chain per column.
// LDL^T keeps D on the diagonal and unit L below.  Called by all PT threads.
template <typename T, int FACTO, int LP>
__device__ void factor_tile64(T *a, int wd, double thr, int *s_piv, int *s_err) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    for (int b = 0; b < wd; b += 8) {
        const int bw = min(8, wd - b);
        if (warp == 0) {
            T g[36];  // the leaf's diagonal block, lower part: g[r (r + 1) / 2 + c]
#pragma unroll
            for (int r = 0; r < 8; r++)
#pragma unroll
                for (int c = 0; c <= r; c++) g[r * (r + 1) / 2 + c] = (r < bw) ? a[(b + r) + (b + c) * LP] : (T)0;
            T dv[8], iv[8];
            int piv = 0, neg = 0;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                dv[c] = (T)1;
                iv[c] = (T)1;
                if (c < bw) {
                    T p = g[c * (c + 1) / 2 + c];
                    const bool rep = fabs(p) < (T)thr;
                    if (rep) p = (FACTO == FACTO_POTRF) ? (T)thr : ((p < (T)0) ? (T)(-thr) : (T)thr);
                    T d, inv;
                    if (FACTO == FACTO_POTRF) {
                        if (p < (T)0) { neg = 1; p = -p; }
                        inv = rsqrt(p);
                        d = p * inv;
                    } else {
                        d = p;
                        inv = (T)1 / p;
                    }
                    piv += rep;
                    dv[c] = d;
                    iv[c] = inv;
                    g[c * (c + 1) / 2 + c] = d;
#pragma unroll
                    for (int r = c + 1; r < 8; r++) g[r * (r + 1) / 2 + c] *= inv;
#pragma unroll
                    for (int j = c + 1; j < 8; j++) {
                        const T ljc = g[j * (j + 1) / 2 + c];
#pragma unroll
                        for (int r = j; r < 8; r++) {
                            const T lrc = g[r * (r + 1) / 2 + c];
                            if (FACTO == FACTO_SYTRF) g[r * (r + 1) / 2 + j] += (-d * lrc) * ljc;
                            else g[r * (r + 1) / 2 + j] -= lrc * ljc;
                        }
                    }
                }
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int i = b + lane + 32 * h;
                if (i < wd && i >= b + 8) {
                    T r[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) r[j] = (j < bw) ? a[i + (b + j) * LP] : (T)0;
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        if (c < bw) {
                            r[c] *= iv[c];
                            const T m = (FACTO == FACTO_SYTRF) ? -dv[c] * r[c] : r[c];
#pragma unroll
                            for (int j = c + 1; j < 8; j++) {
                                if (j < bw) {
                                    if (FACTO == FACTO_SYTRF) r[j] += m * g[j * (j + 1) / 2 + c];
                                    else r[j] -= m * g[j * (j + 1) / 2 + c];
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 8; j++)
                        if (j < bw) a[i + (b + j) * LP] = r[j];
                }
            }
            if (lane < bw) {
#pragma unroll
                for (int r = 0; r < 8; r++)
#pragma unroll
                    for (int c = 0; c <= r; c++)
                        if (r == lane) a[(b + r) + (b + c) * LP] = g[r * (r + 1) / 2 + c];
            }
            if (lane == 0) {
                *s_piv += piv;
                if (neg) *s_err = 1;
            }
        }
        __syncthreads();
        if (b + 8 < wd) {
            // rank-bw update of the trailing lower triangle with the leaf's columns
            T dk[8];
#pragma unroll
            for (int c = 0; c < 8; c++) dk[c] = (FACTO == FACTO_SYTRF && c < bw) ? a[(b + c) * (LP + 1)] : (T)1;
            for (int j = b + 8 + warp; j < wd; j += nwarp) {
                T ljk[8];
#pragma unroll
                for (int c = 0; c < 8; c++) ljk[c] = (c < bw) ? a[j + (b + c) * LP] : (T)0;
                for (int i = j + lane; i < wd; i += 32) {
                    T acc = a[i + j * LP];
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        if (c < bw) {
                            const T lik = a[i + (b + c) * LP];
                            if (FACTO == FACTO_SYTRF) acc -= (lik * dk[c]) * ljk[c];
                            else acc -= lik * ljk[c];
                        }
                    }
                    a[i + j * LP] = acc;
                }
            }
            __syncthreads();
        }
    }
}

// Substitution of one row (thread r < 64) of xs (pitch XP) against the unit lower
// tile lt (pitch LP, identity past the step's width), in 16-column blocks: the
// block's right-hand sides minus the solved columns to its left, then the
// triangle inside the block in registers; POTRF scales by rdiag = 1 / L_cc, LDL^T
// divides by D afterwards (dinv = 1 / D).
template <typename T, int FACTO, int XP>
__device__ void trsm_row64(T *xs, const T *lt, const T *rdiag, const T *dinv, int r) {
    T *xr = xs + r;
#pragma unroll 1
    for (int cb = 0; cb < PB; cb += 16) {
        T acc[16];
#pragma unroll
        for (int q = 0; q < 16; q++) acc[q] = xr[(cb + q) * XP];
        for (int l = 0; l < cb; l++) {
            const T xl = xr[l * XP];
            const T *lc = lt + cb + l * LP;
#pragma unroll
            for (int q = 0; q < 16; q++) acc[q] -= xl * lc[q];
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
#pragma unroll
            for (int p2 = 0; p2 < q; p2++) acc[q] -= acc[p2] * lt[(cb + q) + (cb + p2) * LP];
            acc[q] *= rdiag[cb + q];
        }
#pragma unroll
        for (int q = 0; q < 16; q++) xr[(cb + q) * XP] = acc[q];
    }
    if (FACTO == FACTO_SYTRF) {
        for (int c = 0; c < PB; c++) xr[c * XP] *= dinv[c];
    }
}

template <typename T, int FACTO>
__global__ void __launch_bounds__(PT, sizeof(T) == 4 ? 2 : 1) panel_kernel(DevSym s, const PanelCblk *__restrict__ pcb,
                                                   const PanelItem *__restrict__ items, int nitems, int *ticket,
                                                   int *solved, int *updated, int *abort_word, T *L,
                                                   const double *__restrict__ thr_ptr, unsigned long long *npiv,
                                                   int *err) {
    extern __shared__ __align__(16) unsigned char pn_smem[];
    T *lt = reinterpret_cast<T *>(pn_smem);  // diagonal tile of the step (pitch LP)
    T *xs = lt + PB * LP;                    // the row block's columns of the step (pitch XP)
    T *bs = xs + PB * XP;                    // update operand L[c, j] (D_j): bs[l * PB + row]
    T *rdiag = bs + PB * PB, *dinv = rdiag + PB, *dd = dinv + PB;
    __shared__ int s_item, s_ok, s_piv, s_err;
    const int tid = threadIdx.x;
    bool aborted = false;
    for (;;) {
        if (tid == 0) {
            s_item = atomicAdd(ticket, 1);
            s_ok = 1;
            s_piv = 0;
            s_err = 0;
        }
        __syncthreads();
        const int t = s_item;
        if (t >= nitems) break;
        const PanelItem it = items[t];
        const PanelCblk pc = pcb[it.p];
        const int k = pc.k, j = it.j, b = it.b;
        const int W = s.ncols[k], S = s.stride[k], ld = s.ld[k];
        const double thr = cblk_threshold(s, thr_ptr, k);
        T *P = L + s.off[k];
        const int c0 = PB * j, wd = min(PB, W - c0);
        int *sol = solved + pc.flag0, *upd = updated + pc.flag0;
        if (tid == 0) {
            // the row block's update of the previous step, and the factored tile of this step
            if (j > 0 && !panel_wait(upd + b, j, abort_word)) s_ok = 0;
            if (s_ok && b != j && !panel_wait(sol + j, j + 1, abort_word)) s_ok = 0;
        }
        __syncthreads();
        if (!s_ok) {
            aborted = true;
            break;
        }
        if (b == j) {
            // ---------------------------------------------- diagonal tile
            T *A = P + c0 + (size_t)c0 * ld;
            stage_n<PB * PB / PT, T>(
                [&](int u) {
                    const int idx = tid + PT * u, i = idx & 63, jj = idx >> 6;
                    return (i < wd && jj < wd && i >= jj) ? __ldcg(A + i + (size_t)jj * ld) : (T)0;
                },
                [&](int u, T v) {
                    const int idx = tid + PT * u;
                    lt[(idx & 63) + (idx >> 6) * LP] = v;
                });
            __syncthreads();
            factor_tile64<T, FACTO, LP>(lt, wd, thr, &s_piv, &s_err);
            for (int idx = tid; idx < PB * PB; idx += PT) {
                const int i = idx & 63, jj = idx >> 6;
                if (i < wd && jj < wd && i >= jj) A[i + (size_t)jj * ld] = lt[i + jj * LP];
            }
            __syncthreads();
            if (tid == 0) {
                if (s_piv) atomicAdd(cblk_pivot_counter(s, npiv, k), (unsigned long long)s_piv);
                if (s_err) atomicOr(err, 1);
                __threadfence();
                st_release(sol + b, j + 1);
                st_release(upd + b, j + 1);
            }
            __syncthreads();
            continue;
        }
        // -------------------------------------------------- solve of the row block
        const bool drows = b < pc.ns;
        const int r0 = drows ? PB * b : W + PB * (b - pc.ns);
        const int nr = min(PB, (drows ? W : S) - r0);
        const T *Dg = P + c0 + (size_t)c0 * ld;
        T *X = P + r0 + (size_t)c0 * ld;
        stage_n<PB * PB / PT, T>(
            [&](int u) {
                const int idx = tid + PT * u, c = idx & 63, l = idx >> 6;
                T v = 0;
                if (c < wd && l < wd) v = (c > l) ? __ldcg(Dg + c + (size_t)l * ld) : (c == l ? (T)1 : (T)0);
                else if (c == l) v = 1;
                return v;
            },
            [&](int u, T v) {
                const int idx = tid + PT * u;
                lt[(idx & 63) + (idx >> 6) * LP] = v;
            });
        stage_n<PB * PB / PT, T>(
            [&](int u) {
                const int idx = tid + PT * u, r = idx & 63, c = idx >> 6;
                return (r < nr && c < wd) ? __ldcg(X + r + (size_t)c * ld) : (T)0;
            },
            [&](int u, T v) {
                const int idx = tid + PT * u;
                xs[(idx & 63) + (idx >> 6) * XP] = v;
            });
        if (tid < PB) {
            const T dgv = tid < wd ? __ldcg(Dg + (size_t)tid * (ld + 1)) : (T)1;
            rdiag[tid] = (FACTO == FACTO_POTRF) ? (T)1 / dgv : (T)1;
            dinv[tid] = (FACTO == FACTO_SYTRF) ? (T)1 / dgv : (T)1;
            dd[tid] = (FACTO == FACTO_SYTRF) ? dgv : (T)1;
        }
        __syncthreads();
        if (tid < PB) trsm_row64<T, FACTO, XP>(xs, lt, rdiag, dinv, tid);
        __syncthreads();
        for (int idx = tid; idx < PB * wd; idx += PT) {
            const int r = idx & 63, c = idx >> 6;
            if (r < nr) X[r + (size_t)c * ld] = xs[r + c * XP];
        }
        __syncthreads();
        if (tid == 0 && drows) {
            __threadfence();
            st_release(sol + b, j + 1);
        }
        // -------------------------------------------------- update right of the step
        const int cmax = drows ? b : pc.ns - 1;
        const int tx = tid & 15, ty = tid >> 4;
        for (int c = j + 1; c <= cmax; c++) {
            if (tid == 0 && c != b && !panel_wait(sol + c, j + 1, abort_word)) s_ok = 0;
            __syncthreads();
            if (!s_ok) break;
            const int wc = min(PB, W - PB * c);
            const T *B = P + PB * c + (size_t)c0 * ld;
            stage_n<PB * PB / PT, T>(
                [&](int u) {
                    const int idx = tid + PT * u, rr = idx & 63, l = idx >> 6;
                    return (rr < wc && l < wd) ? __ldcg(B + rr + (size_t)l * ld) : (T)0;
                },
                [&](int u, T v) {
                    const int idx = tid + PT * u;
                    bs[idx] = (FACTO == FACTO_SYTRF) ? v * dd[idx >> 6] : v;
                });
            __syncthreads();
            T acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[i][q] = 0;
            for (int l = 0; l < wd; l++) {
                T av[4], bv[4];
                load4(xs + l * XP + 4 * tx, av);
                load4(bs + l * PB + 4 * ty, bv);
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[i][q] += av[i] * bv[q];
            }
            T *C = P + r0 + (size_t)(PB * c) * ld;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int cc = 4 * ty + q;
                if (cc < wc) {
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const int r = 4 * tx + i;
                        if (r < nr && (c != b || r >= cc)) {
                            T *p = C + r + (size_t)cc * ld;
                            *p = __ldcg(p) - acc[i][q];
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (!s_ok) {
            aborted = true;
            break;
        }
        if (tid == 0) {
            __threadfence();
            st_release(upd + b, j + 1);
        }
        __syncthreads();
    }
    if (aborted && tid == 0) {
        atomicOr(err, 8);
        st_release(abort_word, 1);
    }
}

// Row-block form (when a row block x the level's widest cblk fits in shared
// memory): one item per row block b, which keeps its rows resident in shared
// memory for all the steps -- solve of step j's columns, update of its columns
// right of the step, for every j before the row block's own diagonal tile (all ns
// steps for the rows below the diagonal block) -- and, for b < ns, finally
// factors its diagonal tile (b, b).  Each solved step of the diagonal block's
// rows is written back and announced at once (solved[b] = j + 1; b + 1 after the
// factorization), the only cross-item reads being the factored tiles L[j, j] and
// the diagonal block's solved tiles L[c, j].  Row blocks: 64 rows in the diagonal
// block, R rows (64 or 128) below it.  Items: the diagonal blocks' row blocks of
// every cblk first (b ascending), then the rows below.
template <typename T, int FACTO, int R>
__device__ void rows_item(const DevSym &s, const PanelCblk &pc, int b, T *L, T *lt, T *rdiag, T *dinv, T *dd, T *xs,
                          int *sol, const int *abort_word, double thr, int *s_ok, int *s_piv, int *s_err) {
    constexpr int MR = R / 16;  // rows of a thread's update tile
    const int tid = threadIdx.x;
    const int k = pc.k, W = s.ncols[k], S = s.stride[k], ld = s.ld[k];
    T *P = L + s.off[k];
    const bool drows = b < pc.ns;
    const int r0 = drows ? PB * b : W + R * (b - pc.ns);
    const int nr = min(R, (drows ? W : S) - r0);
    const int ncol = drows ? min(W, PB * (b + 1)) : W;  // columns held (lower part for the diagonal block)
    const int nstep = drows ? b : pc.ns;                 // steps solved in this row block
    // the row block: rows past nr, the diagonal tile's upper triangle and (below
    // the diagonal block) the last step's columns past W as zeros
    const int nzero = drows ? ncol : PB * pc.ns;
    constexpr int CG = PT / R;  // column groups of a load pass
    for (int c0s = 0; c0s < nzero; c0s += 4 * CG) {
        stage_n<4, T>(
            [&](int u) {
                const int r = tid % R, c = c0s + tid / R + CG * u;
                const bool keep = r < nr && c < ncol && (!drows || c < PB * b || r >= c - PB * b);
                return keep ? __ldcg(P + r0 + r + (size_t)c * ld) : (T)0;
            },
            [&](int u, T v) {
                const int r = tid % R, c = c0s + tid / R + CG * u;
                if (c < nzero) xs[r + c * R] = v;
            });
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;
    for (int j = 0; j < nstep && *s_ok; j++) {
        const int c0 = PB * j, wd = min(PB, W - c0);
        if (tid == 0 && !panel_wait(sol + j, j + 1, abort_word)) *s_ok = 0;
        __syncthreads();
        if (!*s_ok) break;
        // ---------------------------------------------- solve of step j's columns
        const T *Dg = P + c0 + (size_t)c0 * ld;
        stage_n<PB * PB / PT, T>(
            [&](int u) {
                const int idx = tid + PT * u, c = idx & 63, l = idx >> 6;
                T v = 0;
                if (c < wd && l < wd) v = (c > l) ? __ldcg(Dg + c + (size_t)l * ld) : (c == l ? (T)1 : (T)0);
                else if (c == l) v = 1;
                return v;
            },
            [&](int u, T v) {
                const int idx = tid + PT * u;
                lt[(idx & 63) + (idx >> 6) * LP] = v;
            });
        if (tid < PB) {
            const T dgv = tid < wd ? __ldcg(Dg + (size_t)tid * (ld + 1)) : (T)1;
            rdiag[tid] = (FACTO == FACTO_POTRF) ? (T)1 / dgv : (T)1;
            dinv[tid] = (FACTO == FACTO_SYTRF) ? (T)1 / dgv : (T)1;
            dd[tid] = (FACTO == FACTO_SYTRF) ? dgv : (T)1;
        }
        __syncthreads();
        if (tid < R) trsm_row64<T, FACTO, R>(xs + c0 * R, lt, rdiag, dinv, tid);
        __syncthreads();
        for (int idx = tid; idx < R * wd; idx += PT) {
            const int r = idx % R, c = idx / R;
            if (r < nr) P[r0 + r + (size_t)(c0 + c) * ld] = xs[r + (c0 + c) * R];
        }
        __syncthreads();
        if (tid == 0 && drows) {
            __threadfence();
            st_release(sol + b, j + 1);
        }
        // ---------------------------------------------- update of the columns right of the step
        const int cmax = drows ? b : pc.ns - 1;
        for (int c = j + 1; c <= cmax; c++) {
            if (tid == 0 && c != b && !panel_wait(sol + c, j + 1, abort_word)) *s_ok = 0;
            __syncthreads();
            if (!*s_ok) break;
            const int wc = min(PB, W - PB * c);
            T *bs = lt;  // bs[l * PB + row]
            if (drows && c == b) {
                // this row block's own tile: its solved columns are in shared memory
                for (int idx = tid; idx < PB * PB; idx += PT) {
                    const int rr = idx & 63, l = idx >> 6;
                    const T v = (rr < wc && l < wd) ? xs[rr + (c0 + l) * R] : (T)0;
                    bs[idx] = (FACTO == FACTO_SYTRF) ? v * dd[l] : v;
                }
            } else {
                const T *B = P + PB * c + (size_t)c0 * ld;
                stage_n<PB * PB / PT, T>(
                    [&](int u) {
                        const int idx = tid + PT * u, rr = idx & 63, l = idx >> 6;
                        return (rr < wc && l < wd) ? __ldcg(B + rr + (size_t)l * ld) : (T)0;
                    },
                    [&](int u, T v) {
                        const int idx = tid + PT * u;
                        bs[idx] = (FACTO == FACTO_SYTRF) ? v * dd[idx >> 6] : v;
                    });
            }
            __syncthreads();
            T acc[MR][4];
#pragma unroll
            for (int i = 0; i < MR; i++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[i][q] = 0;
            const T *xa = xs + c0 * R + MR * tx;
            for (int l = 0; l < wd; l++) {
                T av[MR], bv[4];
#pragma unroll
                for (int h = 0; h < MR / 4; h++) load4(xa + l * R + 4 * h, av + 4 * h);
                load4(bs + l * PB + 4 * ty, bv);
#pragma unroll
                for (int i = 0; i < MR; i++)
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[i][q] += av[i] * bv[q];
            }
            T *xc = xs + (PB * c) * R;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int cc = 4 * ty + q;
                if (cc < wc) {
#pragma unroll
                    for (int i = 0; i < MR; i++) {
                        const int r = MR * tx + i;
                        if (!(drows && c == b) || r >= cc) xc[r + cc * R] -= acc[i][q];
                    }
                }
            }
            __syncthreads();
        }
    }
    if (!*s_ok) return;
    if (drows) {
        // ---------------------------------------------- the row block's diagonal tile
        const int c0 = PB * b, wd = min(PB, W - c0);
        factor_tile64<T, FACTO, R>(xs + c0 * R, wd, thr, s_piv, s_err);
        for (int idx = tid; idx < PB * PB; idx += PT) {
            const int i = idx & 63, jj = idx >> 6;
            if (i < wd && jj < wd && i >= jj) P[c0 + i + (size_t)(c0 + jj) * ld] = xs[i + (c0 + jj) * R];
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release(sol + b, b + 1);
        }
    }
}

template <typename T, int FACTO, int RB>
__global__ void __launch_bounds__(PT, 1)
    panel_rows_kernel(DevSym s, const PanelCblk *__restrict__ pcb, const PanelItem *__restrict__ items, int nitems,
                      int *ticket, int *solved, int *abort_word, T *L, const double *__restrict__ thr_ptr,
                      unsigned long long *npiv, int *err) {
    extern __shared__ __align__(16) unsigned char pn_smem[];
    T *lt = reinterpret_cast<T *>(pn_smem);  // L[j, j] (pitch LP) for the solve; L[c, j] (D_j) for the update
    T *rdiag = lt + PB * LP, *dinv = rdiag + PB, *dd = dinv + PB;
    T *xs = dd + PB;                         // the row block, column-major (pitch = its rows)
    __shared__ int s_item, s_ok, s_piv, s_err;
    const int tid = threadIdx.x;
    bool aborted = false;
    for (;;) {
        if (tid == 0) {
            s_item = atomicAdd(ticket, 1);
            s_ok = 1;
            s_piv = 0;
            s_err = 0;
        }
        __syncthreads();
        const int t = s_item;
        if (t >= nitems) break;
        const PanelItem it = items[t];
        const PanelCblk pc = pcb[it.p];
        int *sol = solved + pc.flag0;
        const double thr = cblk_threshold(s, thr_ptr, pc.k);
        if (it.b < pc.ns)
            rows_item<T, FACTO, PB>(s, pc, it.b, L, lt, rdiag, dinv, dd, xs, sol, abort_word, thr, &s_ok, &s_piv,
                                    &s_err);
        else
            rows_item<T, FACTO, RB>(s, pc, it.b, L, lt, rdiag, dinv, dd, xs, sol, abort_word, thr, &s_ok, &s_piv,
                                    &s_err);
        __syncthreads();
        if (!s_ok) {
            aborted = true;
            break;
        }
        if (tid == 0) {
            if (s_piv) atomicAdd(cblk_pivot_counter(s, npiv, pc.k), (unsigned long long)s_piv);
            if (s_err) atomicOr(err, 1);
        }
        __syncthreads();
    }
    if (aborted && tid == 0) {
        atomicOr(err, 8);
        st_release(abort_word, 1);
    }
}

int g_panel_ctas = 0;  // resident CTAs of the panel kernel on the device (all SMs)
int g_sms = 0, g_smem_optin = 0;

constexpr size_t rows_smem_elems(int nsmax, int rb) { return (size_t)PB * LP + 3 * PB + (size_t)rb * PB * nsmax; }

template <typename T, int FACTO>
int panel_occupancy() {
    const size_t smem = PANEL_SMEM_ELEMS * sizeof(T);
    if (cudaFuncSetAttribute(panel_kernel<T, FACTO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 0;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_kernel<T, FACTO>, PT, smem) != cudaSuccess) return 0;
    return occ;
}

}  // namespace

int configure_panel_kernels() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&g_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return -1;
    g_sms = sms;
    const int dyn = g_smem_optin - 64;  // room for the kernels' static shared variables
    if (cudaFuncSetAttribute(panel_rows_kernel<double, FACTO_POTRF, PB>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) ||
        cudaFuncSetAttribute(panel_rows_kernel<double, FACTO_SYTRF, PB>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) ||
        cudaFuncSetAttribute(panel_rows_kernel<float, FACTO_POTRF, PB>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) ||
        cudaFuncSetAttribute(panel_rows_kernel<float, FACTO_SYTRF, PB>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) ||
        cudaFuncSetAttribute(panel_rows_kernel<float, FACTO_POTRF, 2 * PB>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) ||
        cudaFuncSetAttribute(panel_rows_kernel<float, FACTO_SYTRF, 2 * PB>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn))
        return -1;
    int occ = panel_occupancy<double, FACTO_POTRF>();
    occ = std::min(occ, panel_occupancy<double, FACTO_SYTRF>());
    occ = std::min(occ, panel_occupancy<float, FACTO_POTRF>());
    occ = std::min(occ, panel_occupancy<float, FACTO_SYTRF>());
    if (occ <= 0) return -1;
    g_panel_ctas = occ * sms;
    return 0;
}

template <typename T>
void launch_panel(int facto, const DevSym &s, const PanelCblk *pcb, const PanelItem *items, int nitems, int *ticket,
                  int *solved, int *updated, int *abort_word, T *L, const double *thr, unsigned long long *npiv,
                  int *err, cudaStream_t st) {
    if (nitems <= 0) return;
    const int grid = std::min(nitems, g_panel_ctas);
    const size_t smem = PANEL_SMEM_ELEMS * sizeof(T);
    if (facto == FACTO_POTRF)
        panel_kernel<T, FACTO_POTRF><<<grid, PT, smem, st>>>(s, pcb, items, nitems, ticket, solved, updated,
                                                            abort_word, L, thr, npiv, err);
    else
        panel_kernel<T, FACTO_SYTRF><<<grid, PT, smem, st>>>(s, pcb, items, nitems, ticket, solved, updated,
                                                            abort_word, L, thr, npiv, err);
}

int panel_rows_block(int nsmax, size_t esz) {
    const size_t lim = (size_t)g_smem_optin - 64;
    if (esz == 4 && rows_smem_elems(nsmax, 2 * PB) * esz <= lim) return 2 * PB;
    return rows_smem_elems(nsmax, PB) * esz <= lim ? PB : 0;
}

template <typename T, int RB>
static void launch_rows(int facto, const DevSym &s, const PanelCblk *pcb, const PanelItem *items, int nitems,
                        int nsmax, int *ticket, int *solved, int *abort_word, T *L, const double *thr,
                        unsigned long long *npiv, int *err, cudaStream_t st) {
    const size_t smem = rows_smem_elems(nsmax, RB) * sizeof(T);
    int occ = 0;
    if (facto == FACTO_POTRF)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_rows_kernel<T, FACTO_POTRF, RB>, PT, smem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_rows_kernel<T, FACTO_SYTRF, RB>, PT, smem);
    const int grid = std::min(nitems, std::max(occ, 1) * g_sms);
    if (facto == FACTO_POTRF)
        panel_rows_kernel<T, FACTO_POTRF, RB><<<grid, PT, smem, st>>>(s, pcb, items, nitems, ticket, solved,
                                                                     abort_word, L, thr, npiv, err);
    else
        panel_rows_kernel<T, FACTO_SYTRF, RB><<<grid, PT, smem, st>>>(s, pcb, items, nitems, ticket, solved,
                                                                     abort_word, L, thr, npiv, err);
}

template <typename T>
void launch_panel_rows(int facto, const DevSym &s, const PanelCblk *pcb, const PanelItem *items, int nitems,
                       int nsmax, int rb, int *ticket, int *solved, int *abort_word, T *L, const double *thr,
                       unsigned long long *npiv, int *err, cudaStream_t st) {
    if (nitems <= 0) return;
    if constexpr (sizeof(T) == 4) {
        if (rb == 2 * PB) {
            launch_rows<T, 2 * PB>(facto, s, pcb, items, nitems, nsmax, ticket, solved, abort_word, L, thr, npiv, err,
                                   st);
            return;
        }
    }
    launch_rows<T, PB>(facto, s, pcb, items, nitems, nsmax, ticket, solved, abort_word, L, thr, npiv, err, st);
}

template void launch_panel_rows<double>(int, const DevSym &, const PanelCblk *, const PanelItem *, int, int, int, int *,
                                        int *, int *, double *, const double *, unsigned long long *, int *,
                                        cudaStream_t);
template void launch_panel_rows<float>(int, const DevSym &, const PanelCblk *, const PanelItem *, int, int, int, int *,
                                       int *, int *, float *, const double *, unsigned long long *, int *,
                                       cudaStream_t);

template void launch_panel<double>(int, const DevSym &, const PanelCblk *, const PanelItem *, int, int *, int *, int *,
                                   int *, double *, const double *, unsigned long long *, int *, cudaStream_t);
template void launch_panel<float>(int, const DevSym &, const PanelCblk *, const PanelItem *, int, int *, int *, int *,
                                  int *, float *, const double *, unsigned long long *, int *, cudaStream_t);

}  // namespace b200
