// Internal types of the B200 supernodal factorization/solve library.
//
// Device layout of the factor ("panel layout"): every cblk k owns one
// column-major panel of stride_k rows and ncols_k columns, leading dimension
// ld_k = stride_k rounded up to a multiple of 4, starting on a 256-byte
// boundary.  Its blocks are stacked in the panel in PaStiX's block order
// (diagonal block first), block b starting at panel row rowoff[b].  This is
// PaStiX's 1D cblk layout (the !CBLK_LAYOUT_2D case of kernels/cpucblk_zinit.c
// and kernels/core_zgemmsp.c:1D1D) with a padded leading dimension; the
// integer structure is PaStiX's SolverMatrix unchanged, and
// b200_factor_download() converts back to PaStiX's 2D block layout.
// For LU the transposed U factor has its own arena with the same offsets.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

namespace b200 {

constexpr int FACTO_POTRF = 0, FACTO_SYTRF = 1, FACTO_GETRF = 2;

// Structure tables on the device (all 0-based).
struct DevSym {
    int n, cblknbr, bloknbr;
    const int *fcol;      // [cblknbr+1] first column of each cblk
    const int *ncols;     // [cblknbr]
    const int *stride;    // [cblknbr]
    const int *ld;        // [cblknbr] padded leading dimension
    const int64_t *off;   // [cblknbr] panel offset in elements
    const int *fblok;     // [cblknbr+1]
    const int *frow;      // [bloknbr]
    const int *lrow;      // [bloknbr]
    const int *rowoff;    // [bloknbr] first panel row of the block inside its cblk
    const int *fcblk;     // [bloknbr] facing cblk
    const int *csys;      // [cblknbr] system of each cblk of a batch; nullptr: one system
    const int64_t *rbase; // [cblknbr] first entry of cblk k in prow
    const int *prow;      // [sum of strides] global row of every panel row, cblk after cblk
    const int *rmap;      // destination row in f of each row of every update (from Upd::rm0)
};

#ifdef __CUDACC__
// Static-pivoting threshold of cblk k: thr[0], or in a batch of independent
// systems the threshold of k's own system (each system keeps the rule of its own
// factorization, sopalin/pastix_task_sopalin.c:401-425, with its own norm).
__device__ __forceinline__ double cblk_threshold(const DevSym &s, const double *thr, int k) {
    return thr[s.csys ? s.csys[k] : 0];
}
// Counter of the pivots replaced in cblk k: npiv[0], or its system's in a batch.
__device__ __forceinline__ unsigned long long *cblk_pivot_counter(const DevSym &s, unsigned long long *npiv, int k) {
    return npiv + (s.csys ? s.csys[k] : 0);
}
#endif

// One update of the right-looking supernodal factorization: the contribution of
// cblk k's block j (and the blocks below it) to the facing cblk f
// (core_zgemmsp_2d2d, kernels/core_zgemmsp.c:396-465, as one GEMM over the
// stacked rows):  C_f[rows of blocks i >= j (+shift), cols of block j] -=
// A_k[rows i] * B_k[rows j]^T, K = ncols_k.
enum : int {
    UPD_ATOMIC = 1,   // another cblk of the same level updates f: accumulate with atomics
    UPD_SYM = 2,      // only the lower triangle of the diagonal square is needed
    UPD_A_U = 4,      // A operand from the U panel (LU, upper side)
    UPD_B_U = 8,      // B operand from the U panel (LU, lower side)
    UPD_C_U = 16,     // C is the U panel of f
    UPD_SCALE_D = 32  // multiply A by D (LDL^T: C -= (L_i D) L_j^T)
};

struct Upd {
    int k, j, f;
    int colK0;    // first column of k in the K-range (0 except for sub-panel self-updates)
    int rowA0;    // panel row of k where the M-range starts
    int rowB0;    // panel row of k of block j
    int M, N, K;
    int colbase;  // column in f of block j's first row
    int tiles_m, tiles_n;
    int tile0;    // first tile index of this update inside its launch
    int flags;
    int nb;       // tensor-core updates: columns per tile (a multiple of 32, at most the launch's tile width)
    int rm0;      // first entry of its row map (M entries: row rowA0 + i of k -> row of f, or -1)
};

// Item of the tree-bottom launch, in ticket order: fact = 1 factors cblk k (diagonal
// block and panel solve) once its counter is 0, then marks it factored; fact = 0 waits
// for that mark.  Either then applies updates q0 .. q1 - 1 of the launch's list, on the
// rows [r0, r1) of their M-range (one update split by rows, or whole updates).
struct DagItem {
    int k, q0, q1, r0, r1, fact;
};

// Off-diagonal row tile of a cblk panel (TRSM and solve tasks).
struct RowTask {
    int k;
    int row0;  // first panel row of the tile (>= ncols_k)
};

// Off-diagonal tile of a cblk panel for the solves: 64 panel rows x 64 columns.
struct SolveTile {
    int k;
    int row0;  // first panel row (>= ncols_k)
    int col0;  // first column of the cblk
};

// Item of a dataflow solve sweep (one launch per sweep): FI_LEAF up to 16 cblks
// of at most 32 columns of one level (k = first position in the leaf list, n their
// number); FI_DIAG output rows [r0, r0 + 64) x K chunk [n, n + 64) of the
// diagonal-block product of cblk k; FI_OFF panel rows [r0, r0 + 64) x columns
// [n, n + 64) of cblk k.  flist[f0 .. f0 + nf) are the distinct cblks facing the
// item's off-diagonal rows.
enum : int { FI_LEAF = 0, FI_DIAG = 1, FI_OFF = 2 };
struct FlowItem {
    int type, k, r0, n, f0, nf;
};

// Wide cblk of a panel launch (POTRF / LDL^T cblks wider than the one-CTA diagonal
// kernel): ns steps of 64 columns, nrb row blocks of 64 rows (the first ns cover the
// diagonal block, the others the rows below it), flag0 its first slot in the
// per-row-block dependency counters.
struct PanelCblk {
    int k, ns, nrb, flag0;
};

// Item of a panel launch: step j of wide cblk p on row block b (b >= j).
struct PanelItem {
    int p, j, b;
};

// 64 x 64 tile of a panel copied to the row-major operand arena of the tensor-core
// updates.
struct SplitTask {
    int k;
    int row0;
    int col0;
};

struct Level {
    int c0, c1;          // cblks (indices into lvl_cblk)
    int t0, t1;          // row tasks of the off-diagonal panels
    int u0, u1;          // updates
    int ntiles;          // GEMM tiles of the level
    int nmax;            // widest cblk of the level
    int64_t flops;
};

}  // namespace b200
