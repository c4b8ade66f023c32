// Host side of the B200 supernodal factorization/solve library: structure upload,
// level schedules, kernel sequencing (captured into CUDA graphs), the refinement
// drivers and the C ABI declared in include/pastix_b200.h.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <vector>

#include "b200_internal.h"
#include "kernels.h"
#include "pastix_b200.h"

using namespace b200;

namespace {

constexpr int ERR_SUCCESS = 0, ERR_ALLOC = 2, ERR_NOTIMPL = 3, ERR_OOM = 4, ERR_INTERNAL = 6, ERR_BADPARAM = 7;

#define CU(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            fprintf(stderr, "pastix_b200: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_),    \
                    __FILE__, __LINE__);                                                              \
            return e_ == cudaErrorMemoryAllocation ? ERR_OOM : ERR_INTERNAL;                          \
        }                                                                                             \
    } while (0)

#define RET(call)                          \
    do {                                   \
        int r_ = (call);                   \
        if (r_ != ERR_SUCCESS) return r_;  \
    } while (0)

template <typename T>
int dalloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        fprintf(stderr, "pastix_b200: cudaMalloc(%zu bytes) failed: %s\n", count * sizeof(T), cudaGetErrorString(e));
        return ERR_OOM;
    }
    return ERR_SUCCESS;
}

template <typename T>
int upload(T **p, const std::vector<T> &h, cudaStream_t st) {
    RET(dalloc(p, h.size()));
    if (!h.empty()) CU(cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return ERR_SUCCESS;
}

}  // namespace

// Scratch of the solve and refinement calls issued on one CUDA stream: the
// workspace blocks, the per-column scalars, the dataflow sweeps' tickets and
// counters, the sweep status word and the SpMV staging.  Every stream that solves
// gets its own, so calls on different streams (from different host threads) never
// share scratch and their work can overlap on the GPU.
struct Lane {
    cudaStream_t st = nullptr;
    double *d_ws = nullptr;
    size_t ws_cap = 0;
    double *d_scal = nullptr;  // per-column scalars
    int scal_cap = 0;
    // [ticket f, ticket b, abort, pad][cnt_a f][cnt_b f][cnt_a b][cnt_b b], zeroed per solve
    int *d_sflags = nullptr;
    // bit 4 set by a dataflow sweep that gave up waiting; zeroed at the start of every
    // call that runs sweeps (b200_solve_status reads it)
    int *d_serr = nullptr;
    double *d_xt = nullptr;    // n x 16 row-major staging of the multi-column SpMV (allocated on first use)
    double t_solve = 0, t_refine = 0;
    int launches_solve = 0;
};

struct b200_solver_s {
    int facto = 0, prec = 0;
    bool f32 = false;
    size_t esz = 8;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    int n = 0, cblknbr = 0, bloknbr = 0;
    int64_t coefnbr = 0;  // PaStiX's coefficient count (sum of stride * ncols)
    int64_t arena = 0;    // elements of one factor arena (padded layout)

    // host copy of the structure
    std::vector<int> fcol, ncols, stride, ld, fblok, frow, lrow, rowoff, fcblk, peri;
    std::vector<int64_t> off;

    // device structure
    DevSym ds{};
    std::vector<void *> dev_allocs;
    void *dL = nullptr, *dU = nullptr;
    int *d_peri = nullptr;
    int *d_lvl_cblk = nullptr;
    // cblks from cblkschur on form a Schur complement (CBLK_IN_SCHUR): they receive
    // the updates of the others but are neither factored nor swept; n_active cblks
    // and n1 unknowns (columns before the Schur part) remain
    int cblkschur = 0, n_active = 0, n1 = 0;
    RowTask *d_trsm = nullptr;
    SolveTile *d_stile = nullptr;
    std::vector<int> lvl_st0, lvl_st1;  // solve tiles of each level
    SolveTile *d_dtask = nullptr;       // 64 x 64 tiles of the diagonal-block inverses, forward (lower)
    std::vector<int> lvl_dt0, lvl_dt1;
    SolveTile *d_dtaskb = nullptr;      // and backward (upper triangle of the transpose)
    std::vector<int> lvl_db0, lvl_db1;
    int *d_leaf = nullptr;              // cblks of <= 32 columns, solved by the one-warp kernel
    std::vector<int> lvl_lf0, lvl_lf1;
    // inverses of the diagonal blocks: W_L (forward sweep) and, for LU, W_U (backward)
    int64_t *d_woff = nullptr;
    int64_t winv_elems = 0;
    int64_t *d_toff = nullptr;          // tile inverses of the panel TRSM: 32 x ncols (x2 for LU) per cblk
    int64_t tinv_elems = 0;
    void *dTinv = nullptr;
    void *dWL = nullptr, *dWU = nullptr;
    Upd *d_upd = nullptr;
    std::vector<Level> levels;
    // cblks of each level that go through the one-CTA diagonal kernel (the others take the sub-panel path)
    int *d_diag_list = nullptr;
    int *d_inv_small = nullptr, *d_inv_big = nullptr;  // cblks of <= 32 / > 32 columns
    int n_inv_small = 0, n_inv_big = 0;
    std::vector<int> lvl_ds0, lvl_ds1;
    std::vector<int> lvl_dsm0, lvl_dsm1;  // cblks of <= 32 columns (one warp each)
    std::vector<int> lvl_dsm8, lvl_dsm16; // ends of their <= 8 and <= 16 column classes
    // tree-bottom launch: levels 0 .. dag_levels - 1 (every cblk of at most 32
    // columns, no tensor-core update) factored in one launch by dependency counters
    // instead of level by level, when the environment sets B200_TREE_DAG=1 and the
    // tree has at least two such levels (off by default: at 80^3 it ran slower than
    // the level launches it replaces, whose update kernels keep more warps in flight)
    int dag_levels = 0, dag_nitems = 0, dag_grid = 0;
    DagItem *d_dag_item = nullptr;  // the launch's items in ticket order
    Upd *d_dag_upd = nullptr;
    int *d_dag_cnt0 = nullptr;   // [cblknbr] update items each cblk receives from the launch's cblks
    int *d_dag_cnt = nullptr;    // [cblknbr] working copy, then the ticket and the abort word
    // dataflow solve sweeps: items of the forward and backward launches, the facing
    // lists, and per cblk the counts that complete x (need_f / need_b) and aux
    // (nprev_f: diagonal items, nprev_b: off-diagonal items)
    // the levels from flow_level up take the dataflow sweeps (few cblks per level:
    // launch-bound level by level); the levels below, the level-synchronous kernels
    int flow_level = 0;
    FlowItem *d_fitem_f = nullptr, *d_fitem_b = nullptr;
    int n_fitem_f = 0, n_fitem_b = 0;
    int *d_flist = nullptr, *d_need_f = nullptr, *d_need_b = nullptr, *d_nprev_f = nullptr, *d_nprev_b = nullptr;
    // wide POTRF / LDL^T cblks: one panel launch per level over their 64 x 64 tiles
    std::vector<int> lvl_pi0, lvl_pi1;  // items of each level's launch
    std::vector<int> lvl_prows;         // row-block form: rows of the blocks below the diagonal (0: tile items)
    std::vector<int> lvl_pns;           // most 64-column steps of a cblk of the level
    bool panel_steps_only = false;      // environment B200_PANEL_TILES=1: always the tile-item form
    // failure-path tests (environment B200_TEST_WITHHOLD=panel|flow|dag): the first item
    // of every panel launch / of the forward dataflow sweep is never taken, and the last
    // cblk of the tree-bottom launch waits for one update more than it receives, so the
    // waits that depend on them run out and the error path is exercised.  "panel" and
    // "dag" are read when the instance is created (the factorization graph is captured
    // once); "flow" is read by every solve, so one instance can fail a solve and then
    // run a good one
    int test_withhold = 0;
    PanelCblk *d_pcb = nullptr;
    PanelItem *d_pitem = nullptr;
    // [nlev tickets][solved counters][updated counters][abort word], zeroed per factorization
    int *d_pflags = nullptr;
    int n_pflags = 0, n_prb = 0;
    // FP32 updates on the tensor cores (precision TF32 / TF32X3); updates below the
    // size thresholds stay on the SIMT kernel
    bool use_tc = false;
    int op = 0;                         // operand format of the tensor-core updates: 0 TF32, 1 BF16
    b200_tuning_t tuning{};             // kernel choices (b200_solver_create_tuned)
    Upd *d_tcupd = nullptr;
    std::vector<int> lvl_tc_u0, lvl_tc_u1, lvl_tc_tiles, lvl_tc_m0, lvl_tc_wtiles, lvl_tc_mw0;
    int2 *d_tcmapw = nullptr;             // 128-column tiles
    int2 *d_tcmap = nullptr;              // tiles of each tensor-core launch: {update, row | col << 16}
    Upd *d_smallupd = nullptr;            // updates with K <= 16, N <= 32 (one warp each)
    std::vector<int> lvl_us0, lvl_us1;
    std::vector<char> tc_wanted;          // cblks whose panels the tensor-core updates read
    std::vector<int64_t> toff;            // operand copy of cblk k: row-major, pitch ncols rounded up to 16 bytes
    int64_t tsize = 0;                    // elements of one operand arena
    void *d_tarena = nullptr;             // [L hi][L lo][U hi][U lo] (lo only for TF32X3, U only for LU)
    int64_t *d_toffT = nullptr;
    void *d_maps = nullptr;               // 4 x cblknbr tensor maps
    SplitTask *d_split = nullptr;
    std::vector<int> lvl_sp0, lvl_sp1;    // operand copies of each level (before its external updates)
    std::vector<int> lvl_tr;            // TRSM rows per task of each level
    int nmax_all = 0;
    int64_t total_tiles = 0;
    int trsm_smem = 0;                  // dynamic shared memory available to the panel TRSM
    double flops_class[4] = {0, 0, 0, 0};  // algorithmic flops per kernel class (see Trace)
    double flops_kind[9] = {};             // algorithmic flops of the kinds 3 (updates), 4 (panels), 6 (TC updates),
                                           // 8 (the tree-bottom launch's updates)
    double bytes_scatter = 0;

    // bcsc
    int64_t nnz = -1;
    int64_t *d_colptr = nullptr;
    int *d_rowtab = nullptr;
    double *d_Lv = nullptr, *d_Uv = nullptr;
    // the input matrix's own values -> bcsc entries (b200_spm_map): d_Lv[e] =
    // spm[lmap[e]], d_Uv[e] = spm[umap[e]]; d_spmv holds the uploaded spm values
    int64_t nnz_spm = 0;
    int64_t *d_lmap = nullptr, *d_umap = nullptr;
    double *d_spmv = nullptr;
    int64_t *d_dest = nullptr;
    std::vector<int64_t> h_colptr, h_rowtab;
    double anorm = 0.0;

    // numfact
    double *d_thr = nullptr;
    unsigned long long *d_npiv = nullptr;
    int *d_err = nullptr;
    cudaGraphExec_t fact_graph = nullptr;
    bool factored = false;
    double thr_used = 0.0;
    int64_t last_npiv = 0;

    // batch of independent systems (b200_batch_set): one elimination forest whose
    // trees are the systems, each with its own pivot threshold and refinement
    int nsys = 0;
    int *d_csys = nullptr;     // [cblknbr] system of each cblk
    int *d_sys_col = nullptr;  // [nsys+1] first (permuted) column of each system
    int *d_segid = nullptr;    // [n] system of each permuted row
    std::vector<double> last_berr;  // per-problem backward errors of the last refinement
    std::vector<unsigned long long> last_piv_sys;  // pivots replaced per system by the last numfact

    // device of the instance and the address of the no-allocation scratch on it
    // (looked up when the instance is created)
    int device = 0;
    double *noalloc_scratch = nullptr;

    // per-stream scratch of the solves: main is the instance's own stream's; others
    // are created on a stream's first solve (lane_mu guards the map)
    Lane main;
    std::map<cudaStream_t, Lane *> lanes;
    std::mutex lane_mu;
    // device copies of the host vectors of b200_solve / b200_refine / b200_spmv,
    // sized on first use and grown only when a call needs more
    double *d_stage = nullptr;
    size_t stage_cap = 0;

    double t_fact = 0;
    int launches_fact = 0;
    std::atomic<long long> kernel_launches{0};  // kernels this instance has run (graph replays included)
    std::mutex berr_mu;                           // last_berr, written by refinements on any stream
    std::vector<std::pair<int, double>> trace_detail;  // per-launch times of the last trace
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    template <typename T>
    int dmalloc(T **p, size_t count) {
        RET(dalloc(p, count));
        dev_allocs.push_back((void *)*p);
        return ERR_SUCCESS;
    }
    template <typename T>
    int dupload(T **p, const std::vector<T> &h) {
        RET(upload(p, h, st));
        dev_allocs.push_back((void *)*p);
        return ERR_SUCCESS;
    }
};

extern "C" {
static int sweep_status(Lane *ln);
}

namespace {

int build_schedule(b200_solver_t *s) {
    const int N = s->cblknbr;
    // level = 1 + max level of the cblks that update it; facing cblks have larger indices
    std::vector<int> level(N, 0);
    for (int k = 0; k < N; k++)
        for (int b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++) {
            const int f = s->fcblk[b];
            if (f <= k || f >= N) return ERR_BADPARAM;
            level[f] = std::max(level[f], level[k] + 1);
        }
    const int nlev = N ? *std::max_element(level.begin(), level.end()) + 1 : 0;
    // the level lists hold the cblks before the Schur complement only
    const int cs = s->cblkschur;
    s->n_active = cs;
    s->n1 = cs < N ? s->fcol[cs] : s->n;
    std::vector<int> cnt(nlev + 1, 0);
    for (int k = 0; k < cs; k++) cnt[level[k] + 1]++;
    for (int l = 0; l < nlev; l++) cnt[l + 1] += cnt[l];
    std::vector<int> lvl_cblk(std::max(cs, 1));
    {
        std::vector<int> pos(cnt.begin(), cnt.end() - 1);
        for (int k = 0; k < cs; k++) lvl_cblk[pos[level[k]]++] = k;
    }
    std::vector<RowTask> trsm;
    std::vector<SolveTile> stile;
    std::vector<Upd> upds;
    std::vector<int> diag_list;
    std::vector<PanelCblk> pcbs;
    std::vector<PanelItem> pitems;
    std::vector<Upd> tcupds;
    // destination rows of the updates: for update u, entry u.rm0 + i is the panel row
    // of f receiving row rowA0 + i of k (the block of f that contains it,
    // is_block_inside_fblock, blend/solver.h:358, as core_zgemmsp_2d2d's facing-block
    // walk, kernels/core_zgemmsp.c:420-440), so that
    // the update kernels read one entry instead of searching the block tables
    std::vector<int> rmap;
    auto map_rows = [&](Upd &u) -> bool {
        if (rmap.size() + (size_t)u.M > (size_t)INT32_MAX) return false;
        u.rm0 = (int)rmap.size();
        rmap.resize(rmap.size() + u.M, -1);
        int bf = s->fblok[u.f];
        const int bfe = s->fblok[u.f + 1];
        for (int b = s->fblok[u.k] + 1; b < s->fblok[u.k + 1]; b++) {
            const int r0 = s->rowoff[b], nbr = s->lrow[b] - s->frow[b] + 1;
            if (r0 + nbr <= u.rowA0) continue;
            for (int t = 0; t < nbr; t++) {
                const int prow = r0 + t, grow = s->frow[b] + t;
                if (prow < u.rowA0) continue;
                while (bf < bfe && s->lrow[bf] < grow) bf++;
                int d = -1;
                if (bf < bfe && grow >= s->frow[bf] && grow <= s->lrow[bf]) d = s->rowoff[bf] + (grow - s->frow[bf]);
                rmap[(size_t)u.rm0 + (prow - u.rowA0)] = d;
            }
        }
        return true;
    };
    std::vector<int2> tcmap, tcmapw;  // tile maps of the 64- and 128-column tensor-core launches
    std::vector<Upd> smallupds;
    s->lvl_us0.assign(nlev, 0);
    s->lvl_us1.assign(nlev, 0);
    std::vector<SplitTask> splits;
    std::vector<char> ext_wanted(N, 0);   // cblks with external tensor-core updates
    s->lvl_sp0.assign(nlev, 0);
    s->lvl_sp1.assign(nlev, 0);
    s->tc_wanted.assign(N, 0);
    s->lvl_tc_u0.assign(nlev, 0);
    s->lvl_tc_u1.assign(nlev, 0);
    s->lvl_tc_tiles.assign(nlev, 0);
    s->lvl_tc_m0.assign(nlev, 0);
    s->lvl_tc_mw0.assign(nlev, 0);
    s->lvl_tc_wtiles.assign(nlev, 0);
    // kernel of an FP32 update by the tuning table: 0 CUDA cores, 64 or 128 the
    // tensor cores with tiles of that many columns
    auto tc_choice = [&](const Upd &u) -> int {
        if (!s->use_tc || (u.flags & UPD_SCALE_D) || !(u.colK0 == 0 || u.K % 32 == 0)) return 0;
        const int w = u.K < 16 ? 0 : u.K < 32 ? 1 : u.K < 48 ? 2 : u.K < 64 ? 3 : u.K < 128 ? 4 : 5;
        const int h = u.M < 64 ? 0 : u.M < 128 ? 1 : u.M < 256 ? 2 : u.M < 512 ? 3 : 4;
        const int wide = u.N > 64 ? 128 : 64;
        switch (s->tuning.update[w][h]) {
            case B200_UPD_SIMT: return 0;
            case B200_UPD_TC: return wide;
            case B200_UPD_TC64: return 64;
            default: return (u.K >= 32 && u.M >= 64) ? wide : 0;
        }
    };
    // tensor-core tiles: 128 x 64
    // useful flops of an update: the lower triangle of the diagonal square when symmetric
    auto upd_flops = [](const Upd &u) {
        const double mn = (u.flags & UPD_SYM) ? (double)u.N * (u.M - u.N) + 0.5 * u.N * (u.N + 1.0)
                                              : (double)u.M * u.N;
        return 2.0 * mn * u.K;
    };
    // base: first update of the launch the update belongs to (map entries are relative)
    // updates more than 64 columns wide take 128-column tiles (half the operand
    // traffic per flop of the 64-column tiles)
    // tiles of the launch's width bn (64 or 128 columns).  Narrower tiles that split N
    // evenly (N = 278: 3 of 96 instead of 3 of 128) issue 30 % fewer MMAs at 80^3 but
    // ran 5 % slower: the kernel is bound by the TMA round trips and barrier hand-offs
    // per K chunk and per tile, which a narrower tile does not shorten
    auto push_tc = [&](Upd u, int bn, int &t0, int &t0w, int base) {
        s->flops_kind[6] += upd_flops(u);
        u.nb = bn;
        u.tiles_m = (u.M + 127) / 128;
        u.tiles_n = (u.N + u.nb - 1) / u.nb;
        const int ui = (int)tcupds.size() - base;
        for (int nt = 0; nt < u.tiles_n; nt++)
            for (int mt = 0; mt < u.tiles_m; mt++) {
                if ((u.flags & UPD_SYM) && mt * 128 + 127 < nt * u.nb) continue;  // above the diagonal
                (bn == 128 ? tcmapw : tcmap).push_back(make_int2(ui, mt | (nt << 16)));
                (bn == 128 ? t0w : t0)++;
            }
        s->tc_wanted[u.k] = 1;
        if (!map_rows(u)) return false;
        tcupds.push_back(u);
        return true;
    };
    s->lvl_ds0.assign(nlev, 0);
    s->lvl_ds1.assign(nlev, 0);
    s->lvl_dsm0.assign(nlev, 0);
    s->lvl_dsm8.assign(nlev, 0);
    s->lvl_dsm16.assign(nlev, 0);
    s->lvl_dsm1.assign(nlev, 0);
    s->lvl_pi0.assign(nlev, 0);
    s->lvl_pi1.assign(nlev, 0);
    s->lvl_prows.assign(nlev, 0);
    s->lvl_pns.assign(nlev, 0);
    const int split_min = 96;  // wider POTRF / LDL^T cblks take the sub-panel path
    auto is_big = [&](int k) { return s->facto != FACTO_GETRF && s->ncols[k] > split_min; };
    s->lvl_st0.assign(nlev, 0);
    s->lvl_st1.assign(nlev, 0);
    s->lvl_dt0.assign(nlev, 0);
    s->lvl_dt1.assign(nlev, 0);
    std::vector<SolveTile> dtask, dtaskb;
    std::vector<int> leaf;
    s->lvl_db0.assign(nlev, 0);
    s->lvl_db1.assign(nlev, 0);
    s->lvl_lf0.assign(nlev, 0);
    s->lvl_lf1.assign(nlev, 0);
    s->levels.assign(nlev, Level{});
    s->lvl_tr.assign(nlev, 64);
    std::vector<int> src_count(N, 0), src_last(N, -1);
    // the update of block j of cblk k (side 0; for LU side 1, the upper side, from the
    // U panel rows below block j): false when the block has no such update
    auto make_upd = [&](int k, int j, int side, int atomic, Upd &u) -> bool {
        u = Upd{};
        u.k = k;
        u.j = j;
        u.f = s->fcblk[j];
        u.rowB0 = s->rowoff[j];
        if (side == 0) {
            u.rowA0 = s->rowoff[j];
            u.flags = atomic;
            if (s->facto != FACTO_GETRF) u.flags |= UPD_SYM;
            if (s->facto == FACTO_SYTRF) u.flags |= UPD_SCALE_D;
            if (s->facto == FACTO_GETRF) u.flags |= UPD_B_U;
        } else {
            if (j + 1 >= s->fblok[k + 1]) return false;
            u.rowA0 = s->rowoff[j + 1];
            u.flags = atomic | UPD_A_U | UPD_C_U;
        }
        u.M = s->stride[k] - u.rowA0;
        u.N = s->lrow[j] - s->frow[j] + 1;
        u.K = s->ncols[k];
        u.colbase = s->frow[j] - s->fcol[u.f];
        return true;
    };
    const size_t trsm_smem = (size_t)s->trsm_smem;
    for (int l = 0; l < nlev; l++) {
        Level &L = s->levels[l];
        L.c0 = cnt[l];
        L.c1 = cnt[l + 1];
        L.nmax = 0;
        for (int i = L.c0; i < L.c1; i++) L.nmax = std::max(L.nmax, s->ncols[lvl_cblk[i]]);
        if (L.nmax > 1024) {
            fprintf(stderr, "pastix_b200: cblk of %d columns exceeds the supported width 1024\n", L.nmax);
            return ERR_NOTIMPL;
        }
        int TR = 64;
        while (TR > 16 && (size_t)TR * L.nmax * s->esz > trsm_smem) TR >>= 1;
        if ((size_t)TR * L.nmax * s->esz > trsm_smem) return ERR_NOTIMPL;
        s->lvl_tr[l] = TR;
        L.t0 = (int)trsm.size();
        s->lvl_st0[l] = (int)stile.size();
        s->lvl_dt0[l] = (int)dtask.size();
        s->lvl_db0[l] = (int)dtaskb.size();
        // diagonal blocks: <= 32 columns by the one-warp kernel, up to the sub-panel
        // width by the one-CTA kernel
        s->lvl_ds0[l] = (int)diag_list.size();
        for (int i = L.c0; i < L.c1; i++)
            if (!is_big(lvl_cblk[i]) && s->ncols[lvl_cblk[i]] > 32) diag_list.push_back(lvl_cblk[i]);
        s->lvl_ds1[l] = (int)diag_list.size();
        // cblks of at most 32 columns by width class (8, 16, 32: one kernel instance each)
        s->lvl_dsm0[l] = (int)diag_list.size();
        for (int i = L.c0; i < L.c1; i++)
            if (s->ncols[lvl_cblk[i]] <= 8) diag_list.push_back(lvl_cblk[i]);
        s->lvl_dsm8[l] = (int)diag_list.size();
        for (int i = L.c0; i < L.c1; i++)
            if (s->ncols[lvl_cblk[i]] > 8 && s->ncols[lvl_cblk[i]] <= 16) diag_list.push_back(lvl_cblk[i]);
        s->lvl_dsm16[l] = (int)diag_list.size();
        for (int i = L.c0; i < L.c1; i++)
            if (s->ncols[lvl_cblk[i]] > 16 && s->ncols[lvl_cblk[i]] <= 32) diag_list.push_back(lvl_cblk[i]);
        s->lvl_dsm1[l] = (int)diag_list.size();
        {
            // wide cblks: items (step j, row block b >= j) of the level's panel launch,
            // step by step, then by the row block's distance from the step's diagonal
            // tile, then by cblk (every item depends only on items before it)
            s->lvl_pi0[l] = (int)pitems.size();
            const int p0 = (int)pcbs.size();
            int nsmax = 0, nrbmax = 0;
            for (int i = L.c0; i < L.c1; i++) {
                const int k = lvl_cblk[i];
                if (!is_big(k)) continue;
                PanelCblk pc;
                pc.k = k;
                pc.ns = (s->ncols[k] + 63) / 64;
                pc.nrb = pc.ns + (s->stride[k] - s->ncols[k] + 63) / 64;
                pc.flag0 = s->n_prb;
                s->n_prb += pc.nrb;
                pcbs.push_back(pc);
                nsmax = std::max(nsmax, pc.ns);
                nrbmax = std::max(nrbmax, pc.nrb);
                // diagonal factorization, panel solve and the updates inside the panel
                const double nc = s->ncols[k], m = s->stride[k] - s->ncols[k];
                s->flops_kind[4] += nc * nc * nc / 3.0 + m * nc * nc;
            }
            s->lvl_pns[l] = nsmax;
            const int rb = s->panel_steps_only ? 0 : panel_rows_block(nsmax, s->esz);
            s->lvl_prows[l] = rb;
            if (rb) {
                // row blocks: the diagonal blocks' first (by row block, then cblk), then the
                // rb-row blocks below them
                for (int b = 0; b < nsmax; b++)
                    for (int p = p0; p < (int)pcbs.size(); p++)
                        if (b < pcbs[p].ns) pitems.push_back({p, 0, b});
                for (int b = 0; b < nrbmax; b++)
                    for (int p = p0; p < (int)pcbs.size(); p++) {
                        const int k = pcbs[p].k, nbelow = (s->stride[k] - s->ncols[k] + rb - 1) / rb;
                        if (b < nbelow) pitems.push_back({p, 0, pcbs[p].ns + b});
                    }
            } else {
                for (int j = 0; j < nsmax; j++)
                    for (int d = 0; d < nrbmax - j; d++)
                        for (int p = p0; p < (int)pcbs.size(); p++)
                            if (j < pcbs[p].ns && j + d < pcbs[p].nrb) pitems.push_back({p, j, j + d});
            }
            s->lvl_pi1[l] = (int)pitems.size();
        }
        s->lvl_lf0[l] = (int)leaf.size();
        for (int i = L.c0; i < L.c1; i++) {
            const int k = lvl_cblk[i];
            // (cblks of at most 32 columns solve their rows in the one-warp diagonal kernel)
            if (!is_big(k) && s->ncols[k] > 32)
                for (int r0 = s->ncols[k]; r0 < s->stride[k]; r0 += TR) trsm.push_back({k, r0});
            if (s->ncols[k] <= 32) {
                // small cblk: both parts of each sweep in the one-warp kernel
                leaf.push_back(k);
                continue;
            }
            // tiles of W_k: forward the lower triangle (K chunk <= row tile), backward
            // the upper triangle of W_k^T (K chunk >= output tile)
            for (int r0 = 0; r0 < s->ncols[k]; r0 += 64)
                for (int c0 = 0; c0 < s->ncols[k]; c0 += 64) {
                    if (c0 <= r0) dtask.push_back({k, r0, c0});
                    if (c0 >= r0) dtaskb.push_back({k, r0, c0});
                }
            for (int r0 = s->ncols[k]; r0 < s->stride[k]; r0 += 64)
                for (int c0 = 0; c0 < s->ncols[k]; c0 += 64) stile.push_back({k, r0, c0});
        }
        s->lvl_lf1[l] = (int)leaf.size();
        s->lvl_st1[l] = (int)stile.size();
        s->lvl_dt1[l] = (int)dtask.size();
        s->lvl_db1[l] = (int)dtaskb.size();
        L.t1 = (int)trsm.size();
        // number of sources of this level facing each cblk
        for (int i = L.c0; i < L.c1; i++) {
            const int k = lvl_cblk[i];
            for (int b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++) {
                const int f = s->fcblk[b];
                if (src_last[f] != k) {
                    src_last[f] = k;
                    src_count[f]++;
                }
            }
        }
        L.u0 = (int)upds.size();
        s->lvl_us0[l] = (int)smallupds.size();
        s->lvl_tc_u0[l] = (int)tcupds.size();
        s->lvl_tc_m0[l] = (int)tcmap.size();
        s->lvl_tc_mw0[l] = (int)tcmapw.size();
        int tile0 = 0, tc_tile0 = 0, tc_tilew = 0;
        int64_t flops = 0;
        for (int i = L.c0; i < L.c1; i++) {
            const int k = lvl_cblk[i];
            const int nc = s->ncols[k];
            flops += (int64_t)nc * nc * nc / 3;
            const double m = (double)(s->stride[k] - nc);
            s->flops_class[1] += (s->facto == FACTO_GETRF ? 2.0 : 1.0) * nc * (double)nc * nc / 3.0;
            s->flops_class[2] += (s->facto == FACTO_GETRF ? 2.0 : 1.0) * m * nc * nc;
            for (int j = s->fblok[k] + 1; j < s->fblok[k + 1]; j++) {
                const int f = s->fcblk[j];
                const int atomic = src_count[f] > 1 ? UPD_ATOMIC : 0;
                for (int side = 0; side < (s->facto == FACTO_GETRF ? 2 : 1); side++) {
                    Upd u{};
                    if (!make_upd(k, j, side, atomic, u)) continue;
                    // useful work: the lower triangle of the diagonal square for symmetric updates
                    const double mn = (u.flags & UPD_SYM) ? (double)u.N * (u.M - u.N) + 0.5 * u.N * (u.N + 1.0)
                                                          : (double)u.M * u.N;
                    flops += (int64_t)(2.0 * mn * u.K);
                    s->flops_class[3] += 2.0 * mn * u.K;
                    if (const int bn = tc_choice(u)) {
                        if (!push_tc(u, bn, tc_tile0, tc_tilew, s->lvl_tc_u0[l])) return ERR_NOTIMPL;
                        ext_wanted[k] = 1;
                        continue;
                    }
                    if (!map_rows(u)) return ERR_NOTIMPL;
                    if (u.K <= 16 && u.N <= 32) {
                        s->flops_kind[3] += upd_flops(u);
                        smallupds.push_back(u);
                        continue;
                    }
                    u.tiles_m = (u.M + 63) / 64;
                    u.tiles_n = (u.N + 63) / 64;
                    const int nt = (u.flags & UPD_SYM) ? u.tiles_n * u.tiles_m - u.tiles_n * (u.tiles_n - 1) / 2
                                                       : u.tiles_n * u.tiles_m;
                    u.tile0 = tile0;
                    tile0 += nt;
                    s->flops_kind[3] += upd_flops(u);
                    upds.push_back(u);
                }
            }
        }
        L.u1 = (int)upds.size();
        L.ntiles = tile0;
        s->lvl_us1[l] = (int)smallupds.size();
        s->lvl_tc_u1[l] = (int)tcupds.size();
        s->lvl_tc_tiles[l] = tc_tile0;
        s->lvl_tc_wtiles[l] = tc_tilew;
        // operand copies of the off-diagonal rows of the level's panels read by them
        s->lvl_sp0[l] = (int)splits.size();
        for (int i = L.c0; i < L.c1; i++) {
            const int k = lvl_cblk[i];
            if (!ext_wanted[k]) continue;
            // 64 x 64 tiles from the first off-diagonal row rounded down to a multiple
            // of 4 (16-byte column loads; the few diagonal-block rows copied with them
            // are never read by the updates)
            for (int r0 = s->ncols[k] & ~3; r0 < s->stride[k]; r0 += 64)
                for (int c0 = 0; c0 < s->ncols[k]; c0 += 64) splits.push_back({k, r0, c0});
        }
        s->lvl_sp1[l] = (int)splits.size();
        L.flops = flops;
        s->total_tiles += tile0;
        // reset the per-level source counters
        for (int i = L.c0; i < L.c1; i++) {
            const int k = lvl_cblk[i];
            for (int b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++) {
                src_count[s->fcblk[b]] = 0;
                src_last[s->fcblk[b]] = -1;
            }
        }
        s->nmax_all = std::max(s->nmax_all, L.nmax);
    }
    // tree-bottom launch: the first levels whose cblks all have at most 32 columns and
    // whose updates all stay off the tensor cores, when there are at least two of them
    {
        bool on = false;
        if (const char *e = getenv("B200_TREE_DAG")) on = atoi(e) != 0;
        int lb = 0;
        while (on && lb < nlev) {
            const Level &L = s->levels[lb];
            if (L.nmax > 32 || s->lvl_tc_tiles[lb] + s->lvl_tc_wtiles[lb] > 0 || s->lvl_sp1[lb] > s->lvl_sp0[lb] ||
                s->lvl_pi1[lb] > s->lvl_pi0[lb] || s->lvl_ds1[lb] > s->lvl_ds0[lb])
                break;
            lb++;
        }
        const int ndag = lb >= 2 ? s->levels[lb - 1].c1 : 0;
        const int grid = ndag > 0 ? dag_bottom_grid(s->facto, s->f32, ndag) : 0;
        if (grid > 0) {
            // items level by level: the level's factor items, then the update items of
            // its cblks whose updates are not run by the factor item itself (every
            // dependency of an item is an earlier item).  Item sizes in multiply-adds:
            // a cblk's updates up to kInline run in its factor item; the others are
            // grouped into items of about kChunk, an update above kChunk split by rows
            constexpr double kInline = 16384.0, kChunk = 16384.0;
            std::vector<DagItem> items, upd_items;
            std::vector<Upd> dupd;
            std::vector<int> cnt0(N, 0);
            auto fma = [&](const Upd &u) { return 0.5 * upd_flops(u); };
            int last_fact = -1;
            for (int l = 0; l < lb; l++) {
                upd_items.clear();
                for (int i = s->levels[l].c0; i < s->levels[l].c1; i++) {
                    const int k = lvl_cblk[i];
                    const int q0 = (int)dupd.size();
                    double work = 0.0;
                    for (int j = s->fblok[k] + 1; j < s->fblok[k + 1]; j++)
                        for (int side = 0; side < (s->facto == FACTO_GETRF ? 2 : 1); side++) {
                            Upd u{};
                            if (!make_upd(k, j, side, UPD_ATOMIC, u)) continue;
                            if (!map_rows(u)) return ERR_NOTIMPL;
                            // the same updates the level launches would have run on CUDA cores
                            s->flops_kind[3] -= upd_flops(u);
                            s->flops_kind[8] += upd_flops(u);
                            work += fma(u);
                            dupd.push_back(u);
                        }
                    const int q1 = (int)dupd.size();
                    last_fact = (int)items.size();
                    if (work <= kInline) {
                        items.push_back({k, q0, q1, 0, INT32_MAX, 1});
                        continue;
                    }
                    items.push_back({k, q0, q0, 0, INT32_MAX, 1});
                    double acc = 0.0;
                    int qa = q0;
                    for (int q = q0; q < q1; q++) {
                        const double w = fma(dupd[q]);
                        if (w > kChunk) {
                            if (qa < q) upd_items.push_back({k, qa, q, 0, INT32_MAX, 0});
                            const int M = dupd[q].M;
                            const int pieces = std::min((M + 31) / 32, (int)std::ceil(w / kChunk));
                            const int R = ((M + pieces - 1) / pieces + 31) / 32 * 32;
                            for (int r0 = 0; r0 < M; r0 += R) upd_items.push_back({k, q, q + 1, r0, std::min(M, r0 + R), 0});
                            qa = q + 1;
                            acc = 0.0;
                            continue;
                        }
                        if (acc + w > kChunk && qa < q) {
                            upd_items.push_back({k, qa, q, 0, INT32_MAX, 0});
                            qa = q;
                            acc = 0.0;
                        }
                        acc += w;
                    }
                    if (qa < q1) upd_items.push_back({k, qa, q1, 0, INT32_MAX, 0});
                }
                items.insert(items.end(), upd_items.begin(), upd_items.end());
            }
            // every item decrements the counter of each update's facing cblk once
            for (const DagItem &it : items)
                for (int q = it.q0; q < it.q1; q++) cnt0[dupd[q].f]++;
            if (s->test_withhold & 4) cnt0[items[last_fact].k]++;  // an update that never comes
            RET(s->dupload(&s->d_dag_item, items));
            RET(s->dupload(&s->d_dag_upd, dupd));
            RET(s->dupload(&s->d_dag_cnt0, cnt0));
            RET(s->dmalloc(&s->d_dag_cnt, (size_t)N + 2));
            s->dag_levels = lb;
            s->dag_nitems = (int)items.size();
            s->dag_grid = dag_bottom_grid(s->facto, s->f32, s->dag_nitems);
            if (s->dag_grid <= 0) return ERR_INTERNAL;
        }
    }
    RET(s->dupload(&s->d_lvl_cblk, lvl_cblk));
    RET(s->dupload(&s->d_trsm, trsm));
    RET(s->dupload(&s->d_stile, stile));
    RET(s->dupload(&s->d_dtask, dtask));
    RET(s->dupload(&s->d_dtaskb, dtaskb));
    RET(s->dupload(&s->d_leaf, leaf));
    {
        // dataflow sweep items, level by level (forward bottom-up, backward top-down)
        std::vector<FlowItem> fwd, bwd;
        std::vector<int> flist, need_f(N, 0), need_b(N, 0), nprev_f(N, 0), nprev_b(N, 0);
        std::vector<int> mark(N, -1);
        int stamp = 0;
        auto facing = [&](int k, int r0, int r1, FlowItem &it) {  // distinct cblks facing panel rows [r0, r1)
            for (int b = s->fblok[k] + 1; b < s->fblok[k + 1]; b++) {
                const int b0 = s->rowoff[b], b1 = b0 + s->lrow[b] - s->frow[b] + 1;
                if (b1 <= r0 || b0 >= r1) continue;
                const int f = s->fcblk[b];
                if (mark[f] == stamp) continue;
                mark[f] = stamp;
                flist.push_back(f);
                it.nf++;
            }
        };
        std::vector<std::vector<FlowItem>> lvl_bwd(nlev);
        // first level with fewer than flow_min cblks (tuning table; environment
        // B200_FLOW_MIN overrides it, for tests of both sweep forms)
        int flow_min = s->tuning.flow_min > 0 ? s->tuning.flow_min : 8;
        if (const char *e = getenv("B200_FLOW_MIN")) flow_min = atoi(e);
        s->flow_level = nlev;
        for (int l = 0; l < nlev; l++)
            if (s->levels[l].c1 - s->levels[l].c0 < flow_min) {
                s->flow_level = l;
                break;
            }
        for (int l = s->flow_level; l < nlev; l++) {
            const Level &L = s->levels[l];
            for (int p = s->lvl_lf0[l]; p < s->lvl_lf1[l]; p += 16) {
                FlowItem it{FI_LEAF, p, 0, std::min(16, s->lvl_lf1[l] - p), (int)flist.size(), 0};
                stamp++;
                for (int q = 0; q < it.n; q++) {
                    const int k = leaf[p + q];
                    facing(k, s->ncols[k], s->stride[k], it);
                    need_b[k] = 1;
                }
                for (int q = 0; q < it.nf; q++) need_f[flist[it.f0 + q]]++;
                fwd.push_back(it);
                lvl_bwd[l].push_back(it);
            }
            for (int i = L.c0; i < L.c1; i++) {
                const int k = lvl_cblk[i], nc = s->ncols[k];
                if (nc <= 32) continue;
                // W_k lower triangular: forward chunks c0 <= r0, backward (W_k^T) c0 >= r0
                std::vector<FlowItem> diagf, diagb, off;
                for (int r0 = 0; r0 < nc; r0 += 64)
                    for (int c0 = 0; c0 < nc; c0 += 64) {
                        if (c0 <= r0) diagf.push_back({FI_DIAG, k, r0, c0, 0, 0});
                        if (c0 >= r0) diagb.push_back({FI_DIAG, k, r0, c0, 0, 0});
                    }
                for (int r0 = nc; r0 < s->stride[k]; r0 += 64) {
                    FlowItem it{FI_OFF, k, r0, 0, (int)flist.size(), 0};
                    stamp++;
                    facing(k, r0, std::min(r0 + 64, s->stride[k]), it);
                    for (int c0 = 0; c0 < nc; c0 += 64) {
                        it.n = c0;
                        for (int q = 0; q < it.nf; q++) need_f[flist[it.f0 + q]]++;
                        off.push_back(it);
                    }
                }
                nprev_f[k] = (int)diagf.size();
                nprev_b[k] = (int)off.size();
                need_b[k] = (int)diagb.size();
                fwd.insert(fwd.end(), diagf.begin(), diagf.end());
                fwd.insert(fwd.end(), off.begin(), off.end());
                lvl_bwd[l].insert(lvl_bwd[l].end(), off.begin(), off.end());
                lvl_bwd[l].insert(lvl_bwd[l].end(), diagb.begin(), diagb.end());
            }
        }
        for (int l = nlev - 1; l >= s->flow_level; l--) bwd.insert(bwd.end(), lvl_bwd[l].begin(), lvl_bwd[l].end());
        s->n_fitem_f = (int)fwd.size();
        s->n_fitem_b = (int)bwd.size();
        if (flist.empty()) flist.push_back(0);
        RET(s->dupload(&s->d_fitem_f, fwd));
        RET(s->dupload(&s->d_fitem_b, bwd));
        RET(s->dupload(&s->d_flist, flist));
        RET(s->dupload(&s->d_need_f, need_f));
        RET(s->dupload(&s->d_need_b, need_b));
        RET(s->dupload(&s->d_nprev_f, nprev_f));
        RET(s->dupload(&s->d_nprev_b, nprev_b));
        RET(dalloc(&s->main.d_sflags, (size_t)4 * N + 4));  // freed with the main lane
    }
    RET(s->dupload(&s->d_diag_list, diag_list));
    {
        std::vector<int> small, big;
        for (int k = 0; k < cs; k++) (s->ncols[k] <= 32 && !is_big(k) ? small : big).push_back(k);
        // widest first: their inverses take the longest, so they start before the many
        // narrow ones instead of forming the launch's tail
        std::stable_sort(big.begin(), big.end(), [&](int a, int b) { return s->ncols[a] > s->ncols[b]; });
        s->n_inv_small = (int)small.size();
        s->n_inv_big = (int)big.size();
        RET(s->dupload(&s->d_inv_small, small));
        RET(s->dupload(&s->d_inv_big, big));
    }
    RET(s->dupload(&s->d_pcb, pcbs));
    RET(s->dupload(&s->d_pitem, pitems));
    s->n_pflags = nlev + 2 * s->n_prb + 1;
    RET(s->dmalloc(&s->d_pflags, (size_t)s->n_pflags));
    // inverse arena: n_k x n_k per cblk, 256-byte aligned
    std::vector<int64_t> woff(N);
    int64_t wpos = 0;
    const int64_t walign = s->f32 ? 64 : 32;
    for (int k = 0; k < N; k++) {
        wpos = (wpos + walign - 1) / walign * walign;
        woff[k] = wpos;
        wpos += (int64_t)s->ncols[k] * s->ncols[k];
    }
    s->winv_elems = (wpos + walign - 1) / walign * walign;
    RET(s->dupload(&s->d_woff, woff));
    std::vector<int64_t> toff(N);
    int64_t tpos = 0;
    for (int k = 0; k < N; k++) {
        toff[k] = tpos;
        tpos += (int64_t)32 * s->ncols[k] * (s->facto == FACTO_GETRF ? 2 : 1);
    }
    s->tinv_elems = tpos;
    RET(s->dupload(&s->d_toff, toff));
    RET(s->dupload(&s->d_upd, upds));
    RET(s->dupload(&s->d_tcupd, tcupds));
    RET(s->dupload(&s->d_tcmap, tcmap));
    RET(s->dupload(&s->d_tcmapw, tcmapw));
    if (!rmap.empty()) {
        int *d_rmap = nullptr;
        RET(s->dupload(&d_rmap, rmap));
        s->ds.rmap = d_rmap;
    }
    RET(s->dupload(&s->d_smallupd, smallupds));
    RET(s->dupload(&s->d_split, splits));
    s->toff.assign(N, 0);
    int64_t tp = 0;
    const int oesz = s->op ? 2 : 4, pad = 16 / oesz;  // operand element bytes; pitch in 16-byte units
    for (int k = 0; k < N; k++) {
        if (!s->tc_wanted[k]) continue;
        s->toff[k] = tp;
        tp += (int64_t)s->stride[k] * ((s->ncols[k] + pad - 1) / pad * pad);
        tp = (tp + 256 / oesz - 1) / (256 / oesz) * (256 / oesz);  // 256-byte starts
    }
    s->tsize = tp;
    RET(s->dupload(&s->d_toffT, s->toff));
    return ERR_SUCCESS;
}

int ensure_ws(Lane *ln, size_t doubles) {
    if (doubles <= ln->ws_cap) return ERR_SUCCESS;
    if (ln->d_ws) {
        CU(cudaStreamSynchronize(ln->st));
        cudaFree(ln->d_ws);
    }
    ln->d_ws = nullptr;
    ln->ws_cap = 0;
    RET(dalloc(&ln->d_ws, doubles));
    ln->ws_cap = doubles;
    return ERR_SUCCESS;
}

void free_lane(Lane *ln) {
    if (ln->d_ws) cudaFree(ln->d_ws);
    if (ln->d_scal) cudaFree(ln->d_scal);
    if (ln->d_sflags) cudaFree(ln->d_sflags);
    if (ln->d_serr) cudaFree(ln->d_serr);
    if (ln->d_xt) cudaFree(ln->d_xt);
    *ln = Lane{};
}

// The scratch of the solves issued on stream st (NULL or the instance's own stream:
// the main lane, allocated when the instance was created).  Another stream's lane is
// created on its first call: tickets, counters and status word here, workspaces as
// its calls need them.
int lane_for(b200_solver_t *s, cudaStream_t st, Lane **out) {
    if (!st || st == s->st) {
        *out = &s->main;
        return ERR_SUCCESS;
    }
    std::lock_guard<std::mutex> lock(s->lane_mu);
    auto it = s->lanes.find(st);
    if (it != s->lanes.end()) {
        *out = it->second;
        return ERR_SUCCESS;
    }
    Lane *ln = new Lane();
    ln->st = st;
    int rc = dalloc(&ln->d_sflags, (size_t)4 * s->cblknbr + 4);
    if (!rc) rc = dalloc(&ln->d_serr, 1);
    if (!rc && cudaMemsetAsync(ln->d_serr, 0, sizeof(int), st) != cudaSuccess) rc = ERR_INTERNAL;
    if (rc) {
        free_lane(ln);
        delete ln;
        return rc;
    }
    s->lanes[st] = ln;
    *out = ln;
    return ERR_SUCCESS;
}

// Device copies of host vectors (the host-pointer entry points): one buffer per
// instance, grown only when a call needs more, so repeated calls allocate nothing
// and never pay cudaFree's device synchronization.
int ensure_stage(b200_solver_t *s, size_t doubles) {
    if (doubles <= s->stage_cap) return ERR_SUCCESS;
    if (s->d_stage) {
        CU(cudaStreamSynchronize(s->st));
        cudaFree(s->d_stage);
    }
    s->d_stage = nullptr;
    s->stage_cap = 0;
    RET(dalloc(&s->d_stage, doubles));
    s->stage_cap = doubles;
    return ERR_SUCCESS;
}

int ensure_scal(Lane *ln, int count) {
    if (count <= ln->scal_cap) return ERR_SUCCESS;
    if (ln->d_scal) {
        CU(cudaStreamSynchronize(ln->st));
        cudaFree(ln->d_scal);
    }
    ln->d_scal = nullptr;
    RET(dalloc(&ln->d_scal, (size_t)count));
    ln->scal_cap = count;
    return ERR_SUCCESS;
}

// ---------------------------------------------------------------- numfact

// Per-kernel-class timing of one factorization (kernels_trace,
// kernels/kernels_trace.h:206-300): class 0 arena clear + bcsc scatter, 1 diagonal
// blocks, 2 panel TRSM, 3 GEMM-scatter updates.
// Fine kernel kinds recorded in the per-launch detail; ids 0-3 are the classes
// above, 4 panel factorizations of wide cblks, 5 diagonal-block inverses, 6 updates
// on the tensor cores, 7 operand copies for them, 8 the tree-bottom launch (diagonal
// blocks, panel solves and updates of the bottom levels) (summed into classes 1, 1,
// 3, 3, 3).
struct Trace {
    static constexpr int NK = 9;
    static int coarse(int c) { return c < 4 ? c : c < 6 ? 1 : 3; }
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[NK];
    cudaEvent_t open = nullptr;
    void begin(cudaStream_t st) {
        cudaEventCreate(&open);
        cudaEventRecord(open, st);
    }
    void end(int cls, cudaStream_t st) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        ev[cls].push_back({open, e});
        open = nullptr;
    }
    std::vector<std::pair<int, double>> *detail = nullptr;  // (class, ms) per launch, in class order
    void finish(double *ms) {
        if (detail) detail->clear();
        for (int c = 0; c < 4; c++) ms[c] = 0;
        for (int c = 0; c < NK; c++) {
            for (auto &pr : ev[c]) {
                float t = 0;
                cudaEventElapsedTime(&t, pr.first, pr.second);
                ms[coarse(c)] += t;
                if (detail) detail->push_back({c, (double)t});
                cudaEventDestroy(pr.first);
                cudaEventDestroy(pr.second);
            }
            ev[c].clear();
        }
    }
};

// Row-major (split) copies of the panel tiles sp0..sp1 for the tensor-core updates.
void enqueue_split(b200_solver_t *s, int sp0, int sp1, cudaStream_t st) {
    const bool split = s->prec == B200_PREC_TF32X3 || s->prec == B200_PREC_BF16X3;
    char *a = (char *)s->d_tarena;
    const size_t part_bytes = (size_t)s->tsize * (s->op ? 2 : 4);
    const int parts = split ? 2 : 1;
    for (int side = 0; side < (s->facto == FACTO_GETRF ? 2 : 1); side++) {
        char *hi = a + (size_t)(side * parts) * part_bytes;
        char *lo = split ? hi + part_bytes : nullptr;
        launch_panel_split(s->ds, s->d_split + sp0, sp1 - sp0, (const float *)(side ? s->dU : s->dL), s->d_toffT, hi,
                           lo, s->op, st);
    }
}

template <typename T>
int enqueue_numfact(b200_solver_t *s, cudaStream_t st, Trace *tr = nullptr) {
    T *L = (T *)s->dL, *U = (T *)s->dU;
    int launches = 0;
    if (tr) tr->begin(st);
    CU(cudaMemsetAsync(L, 0, s->arena * sizeof(T), st));
    if (U) CU(cudaMemsetAsync(U, 0, s->arena * sizeof(T), st));
    CU(cudaMemsetAsync(s->d_npiv, 0, (size_t)std::max(s->nsys, 1) * sizeof(unsigned long long), st));
    CU(cudaMemsetAsync(s->d_err, 0, sizeof(int), st));
    CU(cudaMemsetAsync(s->d_pflags, 0, (size_t)s->n_pflags * sizeof(int), st));
    if (s->test_withhold & 1)
        for (size_t l = 0; l < s->levels.size(); l++)
            if (s->lvl_pi1[l] > s->lvl_pi0[l]) CU(cudaMemsetAsync(s->d_pflags + l, 1, 1, st));  // ticket = 1
    launch_scatter<T>(s->nnz, s->d_dest, s->d_Lv, s->d_Uv, L, U, st);
    if (tr) tr->end(0, st);
    launches++;
    if (s->dag_levels > 0) {
        // the bottom levels in one launch, ordered by dependency counters
        if (tr) tr->begin(st);
        const int N = s->cblknbr;
        CU(cudaMemcpyAsync(s->d_dag_cnt, s->d_dag_cnt0, (size_t)N * sizeof(int), cudaMemcpyDeviceToDevice, st));
        CU(cudaMemsetAsync(s->d_dag_cnt + N, 0, 2 * sizeof(int), st));
        launch_dag_bottom<T>(s->facto, s->ds, s->dag_grid, s->d_dag_item, s->dag_nitems, s->d_dag_upd,
                             s->d_dag_cnt, s->d_dag_cnt + N, s->d_dag_cnt + N + 1, L, U, (T *)s->dTinv, s->d_toff,
                             s->d_thr, s->d_npiv, s->d_err, st);
        launches++;
        if (tr) tr->end(8, st);
    }
    for (size_t l = (size_t)s->dag_levels; l < s->levels.size(); l++) {
        const Level &Lv = s->levels[l];
        if (tr) tr->begin(st);
        launch_diag<T>(s->facto, s->ds, s->d_diag_list + s->lvl_ds0[l], s->lvl_ds1[l] - s->lvl_ds0[l], L, U,
                       (T *)s->dTinv, s->d_toff, s->d_thr, s->d_npiv, s->d_err, st);
        {
            const int b[4] = {s->lvl_dsm0[l], s->lvl_dsm8[l], s->lvl_dsm16[l], s->lvl_dsm1[l]};
            const int nb[3] = {8, 16, 32};
            for (int c = 0; c < 3; c++) {
                launch_diag_small<T>(s->facto, s->ds, s->d_diag_list + b[c], b[c + 1] - b[c], nb[c], L, U,
                                     (T *)s->dTinv, s->d_toff, s->d_thr, s->d_npiv, s->d_err, st);
                launches += (b[c + 1] > b[c]);
            }
        }
        if (tr) tr->end(1, st);
        launches++;
        const int nt = Lv.t1 - Lv.t0;
        if (tr) tr->begin(st);
        if (nt > 0) {
            const int TR = s->lvl_tr[l];
            const T *ti = (const T *)s->dTinv;
            if (s->facto == FACTO_POTRF) {
                launch_trsm<T>(s->ds, s->d_trsm + Lv.t0, nt, TR, Lv.nmax, L, L, 1, ti, s->d_toff, 0, 0, 0, st);
            } else if (s->facto == FACTO_SYTRF) {
                launch_trsm<T>(s->ds, s->d_trsm + Lv.t0, nt, TR, Lv.nmax, L, L, 0, ti, s->d_toff, 0, 0, 1, st);
            } else {
                launch_trsm<T>(s->ds, s->d_trsm + Lv.t0, nt, TR, Lv.nmax, L, L, 0, ti, s->d_toff, 1, 1, 0, st);
                launch_trsm<T>(s->ds, s->d_trsm + Lv.t0, nt, TR, Lv.nmax, U, L, 1, ti, s->d_toff, 0, 1, 0, st);
                launches++;
            }
            launches++;
        }
        if (tr) tr->end(2, st);
        // wide cblks: the whole panel factorization in one launch
        if (s->lvl_pi1[l] > s->lvl_pi0[l]) {
            if (tr) tr->begin(st);
            int *tickets = s->d_pflags, *solved = tickets + s->levels.size(), *updated = solved + s->n_prb;
            int *abort_word = updated + s->n_prb;
            if (s->lvl_prows[l])
                launch_panel_rows<T>(s->facto, s->ds, s->d_pcb, s->d_pitem + s->lvl_pi0[l],
                                     s->lvl_pi1[l] - s->lvl_pi0[l], s->lvl_pns[l], s->lvl_prows[l], tickets + l,
                                     solved, abort_word, L, s->d_thr, s->d_npiv, s->d_err, st);
            else
                launch_panel<T>(s->facto, s->ds, s->d_pcb, s->d_pitem + s->lvl_pi0[l], s->lvl_pi1[l] - s->lvl_pi0[l],
                                tickets + l, solved, updated, abort_word, L, s->d_thr, s->d_npiv, s->d_err, st);
            launches++;
            if (tr) tr->end(4, st);
        }
        if (tr) tr->begin(st);
        if (s->lvl_us1[l] > s->lvl_us0[l]) {
            launch_update_small<T>(s->ds, s->d_smallupd + s->lvl_us0[l], s->lvl_us1[l] - s->lvl_us0[l], L, U, st);
            launches++;
        }
        if (Lv.ntiles > 0) {
            if (sizeof(T) == 8)
                launch_update_f64(s->ds, s->d_upd + Lv.u0, Lv.u1 - Lv.u0, Lv.ntiles, (double *)L, (double *)U, st);
            else
                launch_update_f32(s->ds, s->d_upd + Lv.u0, Lv.u1 - Lv.u0, Lv.ntiles, (float *)L, (float *)U, st);
            launches++;
        }
        if (tr) tr->end(3, st);
        if (s->lvl_tc_tiles[l] + s->lvl_tc_wtiles[l] > 0) {
            if (tr) tr->begin(st);
            enqueue_split(s, s->lvl_sp0[l], s->lvl_sp1[l], st);
            launches += 1 + (s->facto == FACTO_GETRF);
            if (tr) tr->end(7, st);
            if (tr) tr->begin(st);
            const int split = s->prec == B200_PREC_TF32X3 || s->prec == B200_PREC_BF16X3;
            launch_update_tc(s->ds, s->d_tcupd + s->lvl_tc_u0[l], s->d_tcmap + s->lvl_tc_m0[l], s->lvl_tc_tiles[l],
                             s->d_maps, (float *)L, (float *)U, split, 64, s->op, s->d_err, st);
            launch_update_tc(s->ds, s->d_tcupd + s->lvl_tc_u0[l], s->d_tcmapw + s->lvl_tc_mw0[l],
                             s->lvl_tc_wtiles[l], s->d_maps, (float *)L, (float *)U, split, 128, s->op, s->d_err, st);
            launches += (s->lvl_tc_tiles[l] > 0) + (s->lvl_tc_wtiles[l] > 0);
            if (tr) tr->end(6, st);
        }
    }
    // inverses of the diagonal blocks for the solves (W_L of L; for LU also W_U of the stored U^T)
    if (tr) tr->begin(st);
    launch_copy_tile_inverse<T>(s->ds, s->d_inv_small, s->n_inv_small, (const T *)s->dTinv, s->d_toff, (T *)s->dWL,
                                s->d_woff, 0, st);
    launch_diag_inverse<T>(s->ds, s->d_inv_big, s->n_inv_big, L, (T *)s->dWL, s->d_woff, s->facto != FACTO_POTRF, st);
    launches += 2;
    if (s->facto == FACTO_GETRF) {
        launch_copy_tile_inverse<T>(s->ds, s->d_inv_small, s->n_inv_small, (const T *)s->dTinv, s->d_toff,
                                    (T *)s->dWU, s->d_woff, 1, st);
        launch_diag_inverse<T>(s->ds, s->d_inv_big, s->n_inv_big, U, (T *)s->dWU, s->d_woff, 0, st);
        launches += 2;
    }
    if (tr) tr->end(5, st);
    CU(cudaGetLastError());
    s->launches_fact = launches;
    return ERR_SUCCESS;
}

// ---------------------------------------------------------------- solve (permuted basis)

// The two sweeps in the permuted basis.  x holds b on entry and the solution on
// exit; aux (same shape) receives the forward solution.  Per level, forward:
// aux_k = W_L,k x_k, then x[ancestor rows] -= P_k aux_k; backward (levels in
// reverse): aux_k -= P_k^T x[ancestor rows], then x_k = W_B,k^T aux_k.
// parts of the sweeps: the forward sweep leaves L^{-1} b in aux (the Schur rows of
// x updated), the backward sweep reads its input from aux
enum { SWEEP_FORWARD = 1, SWEEP_BACKWARD = 2, SWEEP_BOTH = 3 };

// B200_TEST_WITHHOLD=flow: the forward dataflow sweep's first item is withheld
bool flow_withheld() {
    const char *e = getenv("B200_TEST_WITHHOLD");
    return e && !strcmp(e, "flow");
}

template <typename T>
int enqueue_sweeps(b200_solver_t *s, Lane *ln, T *x, T *aux, int64_t ldx, int nrhs, cudaStream_t st, int *launches,
                   Trace *tr = nullptr, int parts = SWEEP_BOTH) {
    const T *L = (const T *)s->dL;
    const T *Ub = (s->facto == FACTO_GETRF) ? (const T *)s->dU : L;
    const T *WL = (const T *)s->dWL;
    const T *WB = (s->facto == FACTO_GETRF) ? (const T *)s->dWU : WL;
    const int N = s->cblknbr, nlev = (int)s->levels.size(), fl0 = s->flow_level;
    int *fl = ln->d_sflags, *abort_word = fl + 2;
    CU(cudaMemsetAsync(fl, 0, ((size_t)4 * N + 4) * sizeof(int), st));
    if (flow_withheld()) CU(cudaMemsetAsync(fl, 1, 1, st));  // forward ticket = 1
    // the diagonal products accumulate their K chunks: zero their outputs (aux now, x
    // before the backward sweep; the Schur rows of x stay, they are the caller's)
    if (parts & SWEEP_FORWARD) {
    CU(cudaMemset2DAsync(aux, (size_t)ldx * sizeof(T), 0, (size_t)s->n * sizeof(T), nrhs, st));
    for (int l = 0; l < fl0; l++) {
        const int nlf = s->lvl_lf1[l] - s->lvl_lf0[l];
        if (nlf > 0) {
            if (tr) tr->begin(st);
            launch_solve_leaf<T>(s->ds, s->d_leaf + s->lvl_lf0[l], nlf, L, WL, s->d_woff, x, aux, ldx, nrhs, 0, st);
            if (tr) tr->end(1, st);
            *launches += 1;
        }
        const int nd = s->lvl_dt1[l] - s->lvl_dt0[l];
        if (tr) tr->begin(st);
        launch_solve_diag_inv<T>(s->ds, s->d_dtask + s->lvl_dt0[l], nd, WL, s->d_woff, x, aux, ldx, nrhs, 0, st);
        const int ns = s->lvl_st1[l] - s->lvl_st0[l];
        launch_solve_tiles<T>(s->ds, s->d_stile + s->lvl_st0[l], ns, L, aux, x, ldx, nrhs, 0, st);
        if (tr) tr->end(1, st);
        *launches += (nd > 0) + (ns > 0);
    }
    if (fl0 < nlev) {
        if (tr) tr->begin(st);
        launch_solve_flow<T, T>(s->ds, s->d_fitem_f, s->n_fitem_f, s->d_leaf, s->d_flist, s->d_need_f, s->d_nprev_f,
                                L, WL, s->d_woff, x, aux, ldx, nrhs, 0, fl, fl + 4, fl + 4 + N, abort_word, ln->d_serr,
                                st);
        if (tr) tr->end(1, st);
        *launches += 1;
    }
    }
    if (s->facto == FACTO_SYTRF && parts == SWEEP_BOTH) {
        if (tr) tr->begin(st);
        launch_solve_scale_diag<T>(s->ds, s->d_lvl_cblk, s->n_active, L, aux, ldx, nrhs, st);
        if (tr) tr->end(3, st);
        *launches += 1;
    }
    if (!(parts & SWEEP_BACKWARD)) return ERR_SUCCESS;
    if (s->n1 > 0) CU(cudaMemset2DAsync(x, (size_t)ldx * sizeof(T), 0, (size_t)s->n1 * sizeof(T), nrhs, st));
    if (fl0 < nlev) {
        if (tr) tr->begin(st);
        launch_solve_flow<T, T>(s->ds, s->d_fitem_b, s->n_fitem_b, s->d_leaf, s->d_flist, s->d_need_b, s->d_nprev_b,
                                Ub, WB, s->d_woff, x, aux, ldx, nrhs, 1, fl + 1, fl + 4 + 2 * N, fl + 4 + 3 * N,
                                abort_word, ln->d_serr, st);
        if (tr) tr->end(2, st);
        *launches += 1;
    }
    for (int l = fl0 - 1; l >= 0; l--) {
        const int nlf = s->lvl_lf1[l] - s->lvl_lf0[l];
        if (nlf > 0) {
            if (tr) tr->begin(st);
            launch_solve_leaf<T>(s->ds, s->d_leaf + s->lvl_lf0[l], nlf, Ub, WB, s->d_woff, x, aux, ldx, nrhs, 1, st);
            if (tr) tr->end(2, st);
            *launches += 1;
        }
        const int ns = s->lvl_st1[l] - s->lvl_st0[l];
        if (tr) tr->begin(st);
        launch_solve_tiles<T>(s->ds, s->d_stile + s->lvl_st0[l], ns, Ub, x, aux, ldx, nrhs, 1, st);
        const int nd = s->lvl_db1[l] - s->lvl_db0[l];
        launch_solve_diag_inv<T>(s->ds, s->d_dtaskb + s->lvl_db0[l], nd, WB, s->d_woff, aux, x, ldx, nrhs, 1, st);
        if (tr) tr->end(2, st);
        *launches += (nd > 0) + (ns > 0);
    }
    CU(cudaGetLastError());
    return ERR_SUCCESS;
}

// Sweeps on the permuted block x (double, leading dimension ldx) with the scratch
// aux (n x nrhs doubles).  An FP32 factor runs the sweeps in FP32 -- they apply the
// preconditioner of an FP64 refinement -- on two n x nrhs float blocks held in aux,
// converted from and back to x.
int sweeps(b200_solver_t *s, Lane *ln, double *x, double *aux, int64_t ldx, int nrhs, cudaStream_t st,
           int *launches, Trace *tr = nullptr) {
    if (!s->f32) return enqueue_sweeps<double>(s, ln, x, aux, ldx, nrhs, st, launches, tr);
    float *xf = reinterpret_cast<float *>(aux), *af = xf + (size_t)s->n * nrhs;
    launch_convert<double, float>(s->n, nrhs, x, ldx, xf, s->n, st);
    RET(enqueue_sweeps<float>(s, ln, xf, af, s->n, nrhs, st, launches, tr));
    launch_convert<float, double>(s->n, nrhs, xf, s->n, x, ldx, st);
    *launches += 2;
    return ERR_SUCCESS;
}

// One step of the solve on the permuted block x (pastix_subtask_trsm /
// pastix_subtask_diag, sopalin/pastix_task_solve.c:194-407): 0 the forward sweep
// (x <- L^{-1} x on the unknowns before the Schur part; the Schur rows receive the
// contributions of the others), 1 the backward sweep (L^T or U, reading the Schur
// rows of x as given), 2 x <- D^{-1} x (LDL^T).  aux: n x nrhs doubles of scratch.
template <typename T>
int sweep_step_t(b200_solver_t *s, Lane *ln, T *x, T *aux, int64_t ldx, int nrhs, int step, cudaStream_t st,
                 int *launches) {
    const size_t pitch = (size_t)ldx * sizeof(T);
    if (step == 0) {
        RET(enqueue_sweeps<T>(s, ln, x, aux, ldx, nrhs, st, launches, nullptr, SWEEP_FORWARD));
        if (s->n1 > 0) CU(cudaMemcpy2DAsync(x, pitch, aux, pitch, (size_t)s->n1 * sizeof(T), nrhs, cudaMemcpyDeviceToDevice, st));
    } else if (step == 1) {
        if (s->n1 > 0) CU(cudaMemcpy2DAsync(aux, pitch, x, pitch, (size_t)s->n1 * sizeof(T), nrhs, cudaMemcpyDeviceToDevice, st));
        RET(enqueue_sweeps<T>(s, ln, x, aux, ldx, nrhs, st, launches, nullptr, SWEEP_BACKWARD));
    } else if (s->facto == FACTO_SYTRF) {
        launch_solve_scale_diag<T>(s->ds, s->d_lvl_cblk, s->n_active, (const T *)s->dL, x, ldx, nrhs, st);
        *launches += 1;
    }
    return ERR_SUCCESS;
}

int sweep_step(b200_solver_t *s, Lane *ln, double *x, double *aux, int64_t ldx, int nrhs, int step, cudaStream_t st,
               int *launches) {
    if (!s->f32) return sweep_step_t<double>(s, ln, x, aux, ldx, nrhs, step, st, launches);
    float *xf = reinterpret_cast<float *>(aux), *af = xf + (size_t)s->n * nrhs;
    launch_convert<double, float>(s->n, nrhs, x, ldx, xf, s->n, st);
    RET(sweep_step_t<float>(s, ln, xf, af, s->n, nrhs, step, st, launches));
    launch_convert<float, double>(s->n, nrhs, xf, s->n, x, ldx, st);
    *launches += 2;
    return ERR_SUCCESS;
}

// Full solve of device b (original ordering) on the lane of stream st: permute,
// sweeps, permute back, with the lane's ws[0 : 2 n nrhs] as the permuted block and
// the sweeps' scratch.
int solve_device(b200_solver_t *s, Lane *ln, int nrhs, double *b, int64_t ldb, cudaStream_t st) {
    const int n = s->n;
    RET(ensure_ws(ln, (size_t)2 * n * nrhs));
    double *xp = ln->d_ws, *aux = ln->d_ws + (size_t)n * nrhs;
    int launches = 2;
    launch_permute(n, nrhs, s->d_peri, b, ldb, xp, n, 1, st);
    RET(sweeps(s, ln, xp, aux, n, nrhs, st, &launches));
    launch_permute(n, nrhs, s->d_peri, xp, n, b, ldb, 0, st);
    CU(cudaGetLastError());
    ln->launches_solve = launches;
    s->kernel_launches += launches;
    return ERR_SUCCESS;
}

// ---------------------------------------------------------------- refinement (permuted basis, double)

struct RefineCtx {
    b200_solver_t *s;
    Lane *ln;
    cudaStream_t st;
    int n, nrhs;
    // independent problems: one per right-hand side column, or in a batch one per
    // (column, system), problem r * nseg + system
    int nseg = 1;
    const int *seg = nullptr;    // [nseg+1] first permuted row of each system
    const int *segid = nullptr;  // [n] system of each permuted row
    int np() const { return nrhs * nseg; }
    // A x in the permuted basis with the bcsc
    int spmv(const double *x, double *y, double alpha, double beta) {
        const double *vals = (s->facto == FACTO_GETRF) ? s->d_Uv : s->d_Lv;
        if (nrhs > 1 && !ln->d_xt) RET(dalloc(&ln->d_xt, (size_t)n * 16));
        launch_spmv(n, nrhs, s->d_colptr, s->d_rowtab, vals, x, n, y, n, alpha, beta, st, ln->d_xt);
        s->kernel_launches += nrhs > 1 ? 2 * ((nrhs + 15) / 16) : 1;
        return ERR_SUCCESS;
    }
    // z <- M^{-1} z with the factor (sweeps only, already permuted)
    double *aux = nullptr;  // n x nrhs scratch of the sweeps
    int spsv(double *z) {
        int l = 0;
        int rc = sweeps(s, ln, z, aux, n, nrhs, st, &l);
        s->kernel_launches += l;
        return rc;
    }
    // one BLAS-1 kernel launched by the caller
    void count(int k = 1) { s->kernel_launches += k; }
    int dots(const double *x, const double *y, std::vector<double> &out) {
        if (segid) launch_seg_dots(nseg, seg, nrhs, x, n, y, n, ln->d_scal, st);
        else launch_dots(n, nrhs, x, n, y, n, ln->d_scal, st);
        s->kernel_launches++;
        out.resize(np());
        CU(cudaMemcpyAsync(out.data(), ln->d_scal, np() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        return ERR_SUCCESS;
    }
    int set_scal(const std::vector<double> &v, int slot) {
        CU(cudaMemcpyAsync(ln->d_scal + (size_t)slot * np(), v.data(), np() * sizeof(double), cudaMemcpyHostToDevice,
                           st));
        return ERR_SUCCESS;
    }
    double *scal(int slot) { return ln->d_scal + (size_t)slot * np(); }
    // vector operations over n x nrhs blocks with per-problem scalars from slot
    void copy(const double *x, double *y) {
        launch_copy(n, nrhs, x, n, y, n, st);
        count();
    }
    void axpys(int slot, double sign, const double *x, double *y) {
        launch_axpys(n, nrhs, scal(slot), sign, x, n, y, n, st, nseg, segid);
        count();
    }
    void xpbys(const double *x, int slot, double *y) {
        launch_xpbys(n, nrhs, x, n, scal(slot), y, n, st, nseg, segid);
        count();
    }
    void scal_cols(int slot, const double *x, double *y) {
        launch_scal_cols(n, nrhs, scal(slot), x, n, y, n, st, nseg, segid);
        count();
    }
};

// z_pivot_smp (refinement/z_refine_pivot.c:45-140), all right-hand sides together,
// each column with its own stopping rule.
int refine_sr(RefineCtx &c, const double *b, double *x, int itermax, double eps, int64_t *niter,
              std::vector<double> &berr) {
    const int n = c.n, R = c.np();
    double *r = c.ln->d_ws + (size_t)2 * n * c.nrhs, *dx = r + (size_t)n * c.nrhs;
    std::vector<double> nb, nr, last(R, 0.0), mask(R, 1.0);
    RET(c.dots(b, b, nb));
    for (auto &v : nb) v = std::sqrt(v);
    int iter = 0;
    bool any = true;
    berr.assign(R, 0.0);
    while (any) {
        c.copy(b, r);
        RET(c.spmv(x, r, -1.0, 1.0));
        RET(c.dots(r, r, nr));
        any = false;
        for (int j = 0; j < R; j++) {
            const double be = std::sqrt(nr[j]) / (nb[j] > 0 ? nb[j] : 1.0);
            if (mask[j] == 0.0) continue;
            berr[j] = be;
            if (iter == 0) last[j] = 3 * be;
            if (iter < itermax && be > eps && be <= last[j] / 2.0) {
                last[j] = be;
                any = true;
            } else {
                mask[j] = 0.0;
            }
        }
        if (!any) break;
        c.copy(r, dx);
        RET(c.spsv(dx));
        RET(c.set_scal(mask, 0));
        c.axpys(0, 1.0, dx, x);
        iter++;
    }
    *niter = iter;
    return ERR_SUCCESS;
}

// z_grad_smp (refinement/z_refine_grad.c:46-156): preconditioned CG.
int refine_cg(RefineCtx &c, const double *b, double *x, int itermax, double eps, int64_t *niter,
              std::vector<double> &berr) {
    const int n = c.n, R = c.np();
    const size_t blk = (size_t)n * c.nrhs;
    double *gr = c.ln->d_ws + 2 * blk, *gp = gr + blk, *gz = gp + blk, *g2 = gz + blk;
    std::vector<double> nb, nx, nr, beta, alpha, tmp;
    RET(c.dots(b, b, nb));
    RET(c.dots(x, x, nx));
    for (auto &v : nb) v = std::sqrt(v);
    c.copy(b, gr);
    RET(c.spmv(x, gr, -1.0, 1.0));
    RET(c.dots(gr, gr, nr));
    std::vector<double> resid(R), active(R, 1.0);
    bool any = false;
    for (int j = 0; j < R; j++) {
        resid[j] = std::sqrt(nr[j]) / (nb[j] > 0 ? nb[j] : 1.0);
        if (resid[j] > eps) any = true; else active[j] = 0.0;
    }
    c.copy(gr, gz);
    RET(c.spsv(gz));
    c.copy(gz, gp);
    int iter = 0;
    while (any && iter < itermax) {
        iter++;
        RET(c.spmv(gp, g2, 1.0, 0.0));
        RET(c.dots(gr, gz, beta));
        RET(c.dots(g2, gp, alpha));
        for (int j = 0; j < R; j++) alpha[j] = (active[j] != 0.0 && alpha[j] != 0.0) ? beta[j] / alpha[j] : 0.0;
        RET(c.set_scal(alpha, 0));
        c.axpys(0, 1.0, gp, x);
        c.axpys(0, -1.0, g2, gr);
        // convergence test on the updated residual before the next preconditioner
        // application, which the last iteration does not need
        RET(c.dots(gr, gr, nr));
        any = false;
        for (int j = 0; j < R; j++) {
            if (active[j] == 0.0) continue;
            resid[j] = std::sqrt(nr[j]) / (nb[j] > 0 ? nb[j] : 1.0);
            if (resid[j] > eps) any = true; else active[j] = 0.0;
        }
        if (!any || iter >= itermax) break;
        c.copy(gr, gz);
        RET(c.spsv(gz));
        RET(c.dots(gr, gz, tmp));
        for (int j = 0; j < R; j++) tmp[j] = (beta[j] != 0.0) ? tmp[j] / beta[j] : 0.0;
        RET(c.set_scal(tmp, 1));
        c.xpbys(gz, 1, gp);
    }
    berr = resid;
    *niter = iter;
    return ERR_SUCCESS;
}

// z_bicgstab_smp (refinement/z_refine_bicgstab.c:46-200): preconditioned
// BiCGSTAB in PaStiX's order, three applications of the preconditioner per iteration
// (to p, to s, and to t for the ratio w = (M^-1 t, M^-1 s) / (M^-1 t, M^-1 t)); every
// right-hand side (every (column, system) of a batch) with its own scalars and
// stopping rule, a stopped one kept unchanged by zero steps.
int refine_bicgstab(RefineCtx &c, const double *b, double *x, int itermax, double eps, int64_t *niter,
                    std::vector<double> &berr) {
    const int n = c.n, R = c.np();
    const size_t blk = (size_t)n * c.nrhs;
    double *gr = c.ln->d_ws + 2 * blk, *gr2 = gr + blk, *gp = gr2 + blk, *gy = gp + blk, *gv = gy + blk;
    double *gs = gv + blk, *gz = gs + blk, *gt = gz + blk, *g2 = gt + blk;
    std::vector<double> nb, nr, vr2, rr2, v1, v2, alpha(R), w(R), beta(R);
    RET(c.dots(b, b, nb));
    for (auto &v : nb) v = std::sqrt(v);
    c.copy(b, gr);  // r = b - A x
    RET(c.spmv(x, gr, -1.0, 1.0));
    RET(c.dots(gr, gr, nr));
    c.copy(gr, gr2);
    c.copy(gr, gp);
    std::vector<double> resid(R), active(R, 1.0);
    bool any = false;
    for (int j = 0; j < R; j++) {
        resid[j] = std::sqrt(nr[j]) / (nb[j] > 0 ? nb[j] : 1.0);
        if (resid[j] > eps) any = true; else active[j] = 0.0;
    }
    int iter = 0;
    while (any && iter < itermax) {
        iter++;
        c.copy(gp, gy);  // y = M^-1 p
        RET(c.spsv(gy));
        RET(c.spmv(gy, gv, 1.0, 0.0));  // v = A y
        RET(c.dots(gv, gr2, vr2));      // alpha = (r, r2) / (v, r2)
        RET(c.dots(gr, gr2, rr2));
        for (int j = 0; j < R; j++) alpha[j] = (active[j] != 0.0 && vr2[j] != 0.0) ? rr2[j] / vr2[j] : 0.0;
        RET(c.set_scal(alpha, 0));
        c.copy(gr, gs);  // s = r - alpha v
        c.axpys(0, -1.0, gv, gs);
        c.copy(gs, gz);  // z = M^-1 s
        RET(c.spsv(gz));
        RET(c.spmv(gz, gt, 1.0, 0.0));  // t = A z
        c.copy(gt, g2);                 // M^-1 t
        RET(c.spsv(g2));
        RET(c.dots(g2, gz, v1));
        RET(c.dots(g2, g2, v2));
        for (int j = 0; j < R; j++) w[j] = (active[j] != 0.0 && v2[j] != 0.0) ? v1[j] / v2[j] : 0.0;
        RET(c.set_scal(alpha, 0));  // slot 0 again: dots() returns its results through it
        c.axpys(0, 1.0, gy, x);     // x += alpha y + w z
        RET(c.set_scal(w, 1));
        c.axpys(1, 1.0, gz, x);
        c.copy(gs, gr);  // r = s - w t
        c.axpys(1, -1.0, gt, gr);
        RET(c.dots(gr, gr2, v1));  // beta = (r', r2) / (r, r2) * (alpha / w)
        for (int j = 0; j < R; j++)
            beta[j] = (active[j] != 0.0 && rr2[j] != 0.0 && w[j] != 0.0) ? v1[j] / rr2[j] * (alpha[j] / w[j]) : 0.0;
        c.axpys(1, -1.0, gv, gp);  // p = r + beta (p - w v)
        RET(c.set_scal(beta, 0));
        c.xpbys(gr, 0, gp);
        RET(c.dots(gr, gr, nr));
        any = false;
        for (int j = 0; j < R; j++) {
            if (active[j] == 0.0) continue;
            resid[j] = std::sqrt(nr[j]) / (nb[j] > 0 ? nb[j] : 1.0);
            if (resid[j] > eps) any = true; else active[j] = 0.0;
        }
    }
    berr = resid;
    *niter = iter;
    return ERR_SUCCESS;
}

// z_gmres_smp (refinement/z_refine_gmres.c:46-352): right-preconditioned
// restarted GMRES(im) with Givens rotations; the Gram-Schmidt projections of all
// right-hand sides are computed together.
int refine_gmres(RefineCtx &c, const double *b, double *x, int itermax, int im, double eps, int64_t *niter,
                 std::vector<double> &berr) {
    const int n = c.n, R = c.np();
    const size_t blk = (size_t)n * c.nrhs;
    double *V = c.ln->d_ws + 2 * blk;              // (im+1) blocks
    double *W = V + (size_t)(im + 1) * blk;         // im blocks
    const int im1 = im + 1;
    std::vector<double> nb, nr, h, tmp;
    RET(c.dots(b, b, nb));
    for (auto &v : nb) v = std::sqrt(v);
    std::vector<std::vector<double>> H(R, std::vector<double>((size_t)im * im1, 0.0));
    std::vector<std::vector<double>> G(R, std::vector<double>(im1, 0.0)), cs(R, std::vector<double>(im, 0.0)),
        sn(R, std::vector<double>(im, 0.0));
    std::vector<double> resid_b(R, 0.0);
    std::vector<char> done(R, 0);
    int iters = 0;
    bool outer = true;
    while (outer) {
        c.copy(b, V);
        RET(c.spmv(x, V, -1.0, 1.0));
        RET(c.dots(V, V, nr));
        bool any = false;
        std::vector<double> inv(R, 0.0);
        for (int j = 0; j < R; j++) {
            const double resid = std::sqrt(nr[j]);
            resid_b[j] = resid / (nb[j] > 0 ? nb[j] : 1.0);
            done[j] = resid_b[j] <= eps;
            if (!done[j]) any = true;
            inv[j] = (!done[j] && resid > 0) ? 1.0 / resid : 0.0;
            std::fill(G[j].begin(), G[j].end(), 0.0);
            G[j][0] = done[j] ? 0.0 : resid;
            std::fill(H[j].begin(), H[j].end(), 0.0);
        }
        if (!any) break;
        RET(c.set_scal(inv, 0));
        c.scal_cols(0, V, V);
        int i = -1;
        bool inner = true;
        while (inner) {
            i++;
            double *Vi = V + (size_t)i * blk, *Wi = W + (size_t)i * blk, *Vn = V + (size_t)(i + 1) * blk;
            c.copy(Vi, Wi);
            RET(c.spsv(Wi));
            RET(c.spmv(Wi, Vn, 1.0, 0.0));
            for (int jj = 0; jj <= i; jj++) {
                RET(c.dots(Vn, V + (size_t)jj * blk, h));
                for (int j = 0; j < R; j++) H[j][(size_t)i * im1 + jj] = h[j];
                RET(c.set_scal(h, 0));
                c.axpys(0, -1.0, V + (size_t)jj * blk, Vn);
            }
            RET(c.dots(Vn, Vn, nr));
            std::vector<double> sc(R, 1.0);
            for (int j = 0; j < R; j++) {
                const double norm = std::sqrt(nr[j]);
                double *Hi = &H[j][(size_t)i * im1];
                Hi[i + 1] = norm;
                sc[j] = norm > 1e-50 ? 1.0 / norm : 1.0;
                for (int q = 0; q < i; q++) {
                    const double t = Hi[q];
                    Hi[q] = cs[j][q] * t + sn[j][q] * Hi[q + 1];
                    Hi[q + 1] = cs[j][q] * Hi[q + 1] - sn[j][q] * t;
                }
                double t = std::sqrt(Hi[i] * Hi[i] + Hi[i + 1] * Hi[i + 1]);
                if (std::fabs(t) <= eps) t = eps;
                cs[j][i] = Hi[i] / t;
                sn[j][i] = Hi[i + 1] / t;
                G[j][i + 1] = -sn[j][i] * G[j][i];
                G[j][i] = cs[j][i] * G[j][i];
                Hi[i] = cs[j][i] * Hi[i] + sn[j][i] * Hi[i + 1];
                if (!done[j]) resid_b[j] = std::fabs(G[j][i + 1]) / (nb[j] > 0 ? nb[j] : 1.0);
            }
            RET(c.set_scal(sc, 0));
            c.scal_cols(0, Vn, Vn);
            iters++;
            bool all_conv = true;
            for (int j = 0; j < R; j++)
                if (!done[j] && resid_b[j] > eps) all_conv = false;
            if (i + 1 >= im || all_conv || iters >= itermax) inner = false;
        }
        // y = H^{-1} g (upper triangular, i+1 columns), x += W y
        for (int j = 0; j < R; j++) {
            std::vector<double> &g = G[j];
            for (int q = i; q >= 0; q--) {
                double v = g[q];
                for (int p = q + 1; p <= i; p++) v -= H[j][(size_t)p * im1 + q] * g[p];
                const double d = H[j][(size_t)q * im1 + q];
                g[q] = (d != 0.0) ? v / d : 0.0;
            }
        }
        for (int q = 0; q <= i; q++) {
            std::vector<double> y(R);
            for (int j = 0; j < R; j++) y[j] = G[j][q];
            RET(c.set_scal(y, 0));
            c.axpys(0, 1.0, W + (size_t)q * blk, x);
        }
        if (iters >= itermax) outer = false;
    }
    berr = resid_b;
    *niter = iters;
    return ERR_SUCCESS;
}

int refine_device(b200_solver_t *s, Lane *ln, int nrhs, const double *b, int64_t ldb, double *x, int64_t ldx,
                  int method, double eps, int64_t itermax, int64_t im, int64_t *niter, double *berr, cudaStream_t st) {
    const int n = s->n;
    if (im < 1) im = 25;
    const size_t blk = (size_t)n * nrhs;
    size_t need = 2 * blk;
    if (method == B200_REFINE_SR) need += 2 * blk;
    else if (method == B200_REFINE_CG) need += 4 * blk;
    else if (method == B200_REFINE_BICGSTAB) need += 9 * blk;
    else need += (size_t)(2 * im + 1) * blk;
    const size_t aux_at = need;
    need += blk;  // scratch of the sweeps
    RET(ensure_ws(ln, need));
    const int nseg = s->nsys > 0 ? s->nsys : 1;
    RET(ensure_scal(ln, 2 * nrhs * nseg));
    double *bp = ln->d_ws, *xp = ln->d_ws + blk;
    launch_permute(n, nrhs, s->d_peri, b, ldb, bp, n, 1, st);
    launch_permute(n, nrhs, s->d_peri, x, ldx, xp, n, 1, st);
    s->kernel_launches += 3;
    RefineCtx c{s, ln, st, n, nrhs};
    if (s->nsys > 0) {
        c.nseg = s->nsys;
        c.seg = s->d_sys_col;
        c.segid = s->d_segid;
    }
    c.aux = ln->d_ws + aux_at;
    std::vector<double> be;
    int64_t it = 0;
    int rc;
    if (method == B200_REFINE_SR) rc = refine_sr(c, bp, xp, (int)itermax, eps, &it, be);
    else if (method == B200_REFINE_CG) rc = refine_cg(c, bp, xp, (int)itermax, eps, &it, be);
    else if (method == B200_REFINE_BICGSTAB) rc = refine_bicgstab(c, bp, xp, (int)itermax, eps, &it, be);
    else rc = refine_gmres(c, bp, xp, (int)itermax, (int)im, eps, &it, be);
    if (rc) return rc;
    launch_permute(n, nrhs, s->d_peri, xp, n, x, ldx, 0, st);
    CU(cudaGetLastError());
    if (niter) *niter = it;
    {
        std::lock_guard<std::mutex> lock(s->berr_mu);
        s->last_berr = be;
    }
    // per column: the largest backward error of its problems (its systems in a batch)
    if (berr)
        for (int j = 0; j < nrhs; j++) {
            berr[j] = 0.0;
            for (int q = 0; q < nseg; q++) berr[j] = std::max(berr[j], be[(size_t)j * nseg + q]);
        }
    return ERR_SUCCESS;
}

}  // namespace

// ====================================================================== no-allocation solve

// Scratch of b200_solve_device_noalloc: the permuted right-hand sides.  A
// file-scope device array, so the entry point never allocates.  In host code
// the name is only a host-side handle; its device address is looked up once per
// device with cudaGetSymbolAddress and passed to the kernels.
static __device__ __align__(256) double g_noalloc_scratch[B200_NOALLOC_SCRATCH_DOUBLES];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
double *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on device dev, which must be the current
// device.  Looked up once per device, when the first instance is created on it: the
// lookup loads this module on the device (under lazy module loading) and so reserves
// the array there, before any no-allocation solve runs.
int noalloc_scratch(int dev, double **out) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return ERR_INTERNAL;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_addr[dev] == nullptr) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            fprintf(stderr, "pastix_b200: cudaGetSymbolAddress of the no-alloc scratch failed: %s\n",
                    cudaGetErrorString(e));
            return ERR_INTERNAL;
        }
        g_noalloc_addr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_addr[dev];
    return ERR_SUCCESS;
}
}  // namespace

// ====================================================================== C ABI

extern "C" {

const char *b200_strerror(int code) {
    switch (code) {
        case 0: return "success";
        case ERR_ALLOC: return "allocation error";
        case ERR_NOTIMPL: return "not implemented";
        case ERR_OOM: return "out of device memory";
        case ERR_INTERNAL: return "internal error (CUDA failure or negative pivot in Cholesky)";
        case ERR_BADPARAM: return "bad parameter";
        default: return "unknown error";
    }
}

int b200_solver_create(const b200_symbol_t *sym, int facto, int precision, void *stream, b200_solver_t **out) {
    return sym ? b200_solver_create_schur(sym, facto, precision, stream, sym->cblknbr, out) : ERR_BADPARAM;
}

int b200_solver_create_schur(const b200_symbol_t *sym, int facto, int precision, void *stream, int64_t cblkschur,
                             b200_solver_t **out) {
    return b200_solver_create_tuned(sym, facto, precision, stream, cblkschur, nullptr, out);
}

int b200_solver_create_tuned(const b200_symbol_t *sym, int facto, int precision, void *stream, int64_t cblkschur,
                             const b200_tuning_t *tuning, b200_solver_t **out) {
    if (tuning)
        for (int w = 0; w < B200_TUNE_WCLASSES; w++)
            for (int h = 0; h < B200_TUNE_HCLASSES; h++)
                if (tuning->update[w][h] < 0 || tuning->update[w][h] > B200_UPD_TC64) return ERR_BADPARAM;
    if (!sym || !out || facto < 0 || facto > 2 || precision < 0 || precision > 4) return ERR_BADPARAM;
    if (sym->n <= 0 || sym->cblknbr <= 0 || sym->n >= (1LL << 31) || sym->bloknbr >= (1LL << 31)) return ERR_BADPARAM;
    if (cblkschur < 1 || cblkschur > sym->cblknbr) return ERR_BADPARAM;
    int dev = 0;
    CU(cudaGetDevice(&dev));
    b200_solver_t *s = new b200_solver_t();
    *out = nullptr;
    s->facto = facto;
    s->prec = precision;
    s->f32 = precision != B200_PREC_FP64;
    s->esz = s->f32 ? 4 : 8;
    s->use_tc = precision == B200_PREC_TF32 || precision == B200_PREC_TF32X3 || precision == B200_PREC_BF16X3;
    s->op = precision == B200_PREC_BF16X3 ? 1 : 0;
    if (tuning) s->tuning = *tuning;
    s->panel_steps_only = s->tuning.panel_tiles != 0;
    if (const char *e = getenv("B200_PANEL_TILES")) s->panel_steps_only = atoi(e) != 0;
    if (const char *e = getenv("B200_TEST_WITHHOLD"))
        s->test_withhold = !strcmp(e, "panel") ? 1 : !strcmp(e, "flow") ? 2 : !strcmp(e, "dag") ? 4 : 0;
    if (stream) {
        s->st = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
            delete s;
            return ERR_INTERNAL;
        }
        s->own_stream = true;
    }
    const int N = (int)sym->cblknbr, B = (int)sym->bloknbr;
    s->n = (int)sym->n;
    s->cblknbr = N;
    s->cblkschur = (int)cblkschur;
    s->bloknbr = B;
    s->fcol.resize(N + 1);
    s->ncols.resize(N);
    s->stride.resize(N);
    s->ld.resize(N);
    s->off.resize(N);
    s->fblok.resize(N + 1);
    s->frow.resize(B);
    s->lrow.resize(B);
    s->rowoff.resize(B);
    s->fcblk.resize(B);
    s->peri.resize(s->n);
    int64_t pos = 0, coef = 0;
    const int64_t align = s->f32 ? 64 : 32;  // 256-byte panel starts
    for (int k = 0; k <= N; k++) {
        s->fcol[k] = (int)sym->cblk_fcolnum[k];
        s->fblok[k] = (int)sym->cblk_fblok[k];
    }
    for (int k = 0; k < N; k++) {
        s->ncols[k] = (int)(sym->cblk_lcolnum[k] - sym->cblk_fcolnum[k] + 1);
        s->stride[k] = (int)sym->cblk_stride[k];
        s->ld[k] = (s->stride[k] + 3) & ~3;
        pos = (pos + align - 1) / align * align;
        s->off[k] = pos;
        pos += (int64_t)s->ld[k] * s->ncols[k];
        coef += (int64_t)s->stride[k] * s->ncols[k];
        if (s->fblok[k + 1] <= s->fblok[k] || s->ncols[k] <= 0) {
            delete s;
            return ERR_BADPARAM;
        }
        int row = 0;
        for (int b = s->fblok[k]; b < s->fblok[k + 1]; b++) {
            s->frow[b] = (int)sym->blok_frownum[b];
            s->lrow[b] = (int)sym->blok_lrownum[b];
            s->fcblk[b] = (int)sym->blok_fcblknm[b];
            s->rowoff[b] = row;
            row += s->lrow[b] - s->frow[b] + 1;
        }
        if (row != s->stride[k]) {
            delete s;
            return ERR_BADPARAM;
        }
    }
    for (int i = 0; i < s->n; i++) s->peri[i] = (int)sym->peritab[i];
    s->arena = (pos + align - 1) / align * align;
    s->coefnbr = coef;
    int rc = ERR_SUCCESS;
    s->trsm_smem = configure_factor_kernels();
    if (s->trsm_smem < 0 || configure_solve_kernels() < 0 || configure_inverse_kernels() < 0 ||
        configure_panel_kernels() < 0 || (s->use_tc && configure_tc_kernels() < 0)) {
        fprintf(stderr, "pastix_b200: cannot configure the shared memory of the kernels\n");
        rc = ERR_INTERNAL;
    }
    int *d_fcol, *d_ncols, *d_stride, *d_ld, *d_fblok, *d_frow, *d_lrow, *d_rowoff, *d_fcblk;
    int64_t *d_off;
    if (!rc) rc = s->dupload(&d_fcol, s->fcol);
    if (!rc) rc = s->dupload(&d_ncols, s->ncols);
    if (!rc) rc = s->dupload(&d_stride, s->stride);
    if (!rc) rc = s->dupload(&d_ld, s->ld);
    if (!rc) rc = s->dupload(&d_off, s->off);
    if (!rc) rc = s->dupload(&d_fblok, s->fblok);
    if (!rc) rc = s->dupload(&d_frow, s->frow);
    if (!rc) rc = s->dupload(&d_lrow, s->lrow);
    if (!rc) rc = s->dupload(&d_rowoff, s->rowoff);
    if (!rc) rc = s->dupload(&d_fcblk, s->fcblk);
    if (!rc) rc = s->dupload(&s->d_peri, s->peri);
    if (!rc) {
        // global row of every panel row (blocks stacked in block order in the panel)
        std::vector<int64_t> rbase(N);
        std::vector<int> prow;
        int64_t pos = 0;
        for (int k = 0; k < N && !rc; k++) {
            rbase[k] = pos;
            for (int b = s->fblok[k]; b < s->fblok[k + 1]; b++)
                for (int r = s->frow[b]; r <= s->lrow[b]; r++) prow.push_back(r);
            pos = (int64_t)prow.size();
            if (pos - rbase[k] != s->stride[k]) rc = ERR_BADPARAM;
        }
        int64_t *d_rbase = nullptr;
        int *d_prow = nullptr;
        if (!rc) rc = s->dupload(&d_rbase, rbase);
        if (!rc) rc = s->dupload(&d_prow, prow);
        if (!rc && cudaStreamSynchronize(s->st) != cudaSuccess) rc = ERR_INTERNAL;  // before the vectors go
        if (!rc) {
            s->ds = DevSym{s->n, N, B, d_fcol, d_ncols, d_stride, d_ld, d_off, d_fblok, d_frow, d_lrow, d_rowoff, d_fcblk};
            s->ds.rbase = d_rbase;
            s->ds.prow = d_prow;
            rc = build_schedule(s);
        }
    }
    if (!rc) rc = dalloc((char **)&s->dL, (size_t)s->arena * s->esz);
    if (!rc && facto == FACTO_GETRF) rc = dalloc((char **)&s->dU, (size_t)s->arena * s->esz);
    if (!rc) rc = dalloc((char **)&s->dWL, (size_t)s->winv_elems * s->esz);
    if (!rc) rc = dalloc((char **)&s->dTinv, (size_t)s->tinv_elems * s->esz);
    if (!rc && facto == FACTO_GETRF) rc = dalloc((char **)&s->dWU, (size_t)s->winv_elems * s->esz);
    if (!rc && s->use_tc) {
        // operand arenas and their tensor maps
        const int parts = (precision == B200_PREC_TF32X3 || precision == B200_PREC_BF16X3) ? 2 : 1;
        const int sides = facto == FACTO_GETRF ? 2 : 1, oesz = s->op ? 2 : 4;
        rc = dalloc((char **)&s->d_tarena, (size_t)std::max<int64_t>(s->tsize, 128) * parts * sides * oesz);
        std::vector<CUtensorMap> maps((size_t)4 * N);
        for (int side = 0; side < sides && !rc; side++)
            for (int part = 0; part < parts && !rc; part++) {
                char *arena = (char *)s->d_tarena + (size_t)(side * parts + part) * s->tsize * oesz;
                if (encode_operand_maps(s->toff, s->stride, s->ncols, s->tc_wanted, arena, s->op,
                                        maps.data() + (size_t)(side * 2 + part) * N)) {
                    fprintf(stderr, "pastix_b200: cannot encode the tensor maps of the operand copies\n");
                    rc = ERR_INTERNAL;
                }
            }
        CUtensorMap *d = nullptr;
        if (!rc) rc = s->dmalloc(&d, maps.size());
        if (!rc && cudaMemcpy(d, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = ERR_INTERNAL;
        s->d_maps = d;
    }
    if (!rc) rc = s->dmalloc(&s->d_thr, 1);
    if (!rc) rc = s->dmalloc(&s->d_npiv, 1);
    if (!rc) rc = s->dmalloc(&s->d_err, 1);
    s->main.st = s->st;
    if (!rc) rc = dalloc(&s->main.d_serr, 1);
    if (!rc && cudaMemsetAsync(s->main.d_serr, 0, sizeof(int), s->st) != cudaSuccess) rc = ERR_INTERNAL;
    s->device = dev;
    if (!rc) rc = noalloc_scratch(dev, &s->noalloc_scratch);
    if (!rc && cudaEventCreate(&s->ev0) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc && cudaEventCreate(&s->ev1) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc && cudaStreamSynchronize(s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (rc) {
        b200_solver_destroy(s);
        return rc;
    }
    *out = s;
    return ERR_SUCCESS;
}

int b200_solver_destroy(b200_solver_t *s) {
    if (!s) return ERR_SUCCESS;
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->fact_graph) cudaGraphExecDestroy(s->fact_graph);
    for (auto &kv : s->lanes) {
        free_lane(kv.second);
        delete kv.second;
    }
    s->lanes.clear();
    for (void *p : s->dev_allocs) cudaFree(p);
    if (s->dL) cudaFree(s->dL);
    if (s->dU) cudaFree(s->dU);
    if (s->dWL) cudaFree(s->dWL);
    if (s->dTinv) cudaFree(s->dTinv);
    if (s->d_tarena) cudaFree(s->d_tarena);
    if (s->dWU) cudaFree(s->dWU);
    if (s->d_colptr) cudaFree(s->d_colptr);
    if (s->d_rowtab) cudaFree(s->d_rowtab);
    if (s->d_Lv) cudaFree(s->d_Lv);
    if (s->d_Uv) cudaFree(s->d_Uv);
    if (s->d_lmap) cudaFree(s->d_lmap);
    if (s->d_umap) cudaFree(s->d_umap);
    if (s->d_spmv) cudaFree(s->d_spmv);
    if (s->d_dest) cudaFree(s->d_dest);
    free_lane(&s->main);
    if (s->d_stage) cudaFree(s->d_stage);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->own_stream && s->st) cudaStreamDestroy(s->st);
    delete s;
    return ERR_SUCCESS;
}

int b200_bcsc_values(b200_solver_t *s, const double *Lvalues, const double *Uvalues, double anorm) {
    if (!s || s->nnz < 0 || !Lvalues) return ERR_BADPARAM;
    if (s->facto == FACTO_GETRF && (!Uvalues || !s->d_Uv)) return ERR_BADPARAM;
    CU(cudaMemcpyAsync(s->d_Lv, Lvalues, s->nnz * sizeof(double), cudaMemcpyHostToDevice, s->st));
    if (Uvalues && s->d_Uv) CU(cudaMemcpyAsync(s->d_Uv, Uvalues, s->nnz * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
    s->anorm = anorm;
    s->factored = false;
    return ERR_SUCCESS;
}

// bcsc_zinit_centralized (bcsc/bcsc_zinit.c:52-541) on the device for a matrix whose
// pattern is the one of the last b200_bcsc_load: the permutation and symmetric
// expansion of the input values is a gather through maps built once on the host
// (by running PaStiX's own bcsc construction on the entry indices).
int b200_spm_map(b200_solver_t *s, int64_t nnz_spm, const int64_t *lmap, const int64_t *umap) {
    if (!s || s->nnz < 0 || nnz_spm <= 0 || !lmap) return ERR_BADPARAM;
    if (s->facto == FACTO_GETRF && !umap) return ERR_BADPARAM;
    for (int64_t e = 0; e < s->nnz; e++) {
        if (lmap[e] < 0 || lmap[e] >= nnz_spm) return ERR_BADPARAM;
        if (s->facto == FACTO_GETRF && (umap[e] < 0 || umap[e] >= nnz_spm)) return ERR_BADPARAM;
    }
    if (s->d_lmap) cudaFree(s->d_lmap);
    if (s->d_umap) cudaFree(s->d_umap);
    if (s->d_spmv) cudaFree(s->d_spmv);
    s->d_lmap = s->d_umap = nullptr;
    s->d_spmv = nullptr;
    s->nnz_spm = 0;
    RET(dalloc(&s->d_lmap, (size_t)s->nnz));
    RET(dalloc(&s->d_spmv, (size_t)nnz_spm));
    CU(cudaMemcpy(s->d_lmap, lmap, s->nnz * sizeof(int64_t), cudaMemcpyHostToDevice));
    if (s->facto == FACTO_GETRF) {
        RET(dalloc(&s->d_umap, (size_t)s->nnz));
        CU(cudaMemcpy(s->d_umap, umap, s->nnz * sizeof(int64_t), cudaMemcpyHostToDevice));
    }
    s->nnz_spm = nnz_spm;
    return ERR_SUCCESS;
}

int b200_spm_values_device(b200_solver_t *s, const double *d_values, double anorm, void *stream) {
    if (!s || s->nnz < 0 || !s->nnz_spm || !d_values) return ERR_BADPARAM;
    cudaStream_t st = stream ? (cudaStream_t)stream : s->st;
    launch_gather_values(s->nnz, s->d_lmap, d_values, s->d_Lv, st);
    if (s->facto == FACTO_GETRF) launch_gather_values(s->nnz, s->d_umap, d_values, s->d_Uv, st);
    if (anorm < 0.0) {
        // ||A||_F over the expanded bcsc (both triangles), as spmNorm(SpmFrobeniusNorm)
        Lane *ln = nullptr;
        RET(lane_for(s, st, &ln));
        RET(ensure_scal(ln, 4));
        CU(cudaMemsetAsync(ln->d_scal, 0, sizeof(double), st));
        launch_dots((int)s->nnz, 1, s->d_Lv, s->nnz, s->d_Lv, s->nnz, ln->d_scal, st);
        double ss = 0.0;
        CU(cudaMemcpyAsync(&ss, ln->d_scal, sizeof(double), cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        anorm = std::sqrt(ss);
    }
    if (st != s->st) {
        // the factorization runs on the solver's stream
        CU(cudaEventRecord(s->ev1, st));
        CU(cudaStreamWaitEvent(s->st, s->ev1, 0));
    }
    s->anorm = anorm;
    s->factored = false;
    return ERR_SUCCESS;
}

int b200_get_diag(b200_solver_t *s, double *D, int64_t incD) {
    if (!s || !D || incD <= 0) return ERR_BADPARAM;
    if (!s->factored) return ERR_BADPARAM;  // pastixGetDiag requires the numerical factorization
    const int n = s->n;
    RET(ensure_ws(&s->main, (size_t)n));
    if (s->f32) launch_get_diag<float>(s->ds, (const float *)s->dL, s->main.d_ws, s->st);
    else launch_get_diag<double>(s->ds, (const double *)s->dL, s->main.d_ws, s->st);
    CU(cudaMemcpy2DAsync(D, incD * sizeof(double), s->main.d_ws, sizeof(double), sizeof(double), n, cudaMemcpyDeviceToHost,
                         s->st));
    CU(cudaStreamSynchronize(s->st));
    return ERR_SUCCESS;
}

int b200_batch_set(b200_solver_t *s, int64_t nsys, const int64_t *sys_cblk) {
    if (!s || !sys_cblk || nsys < 1 || nsys > s->cblknbr || s->nsys != 0) return ERR_BADPARAM;
    if (s->cblkschur < s->cblknbr) return ERR_BADPARAM;  // a batch has no Schur complement
    if (sys_cblk[0] != 0 || sys_cblk[nsys] != s->cblknbr) return ERR_BADPARAM;
    std::vector<int> csys(s->cblknbr), col(nsys + 1), segid(s->n);
    for (int64_t i = 0; i < nsys; i++) {
        if (sys_cblk[i + 1] <= sys_cblk[i]) return ERR_BADPARAM;
        for (int64_t k = sys_cblk[i]; k < sys_cblk[i + 1]; k++) {
            csys[k] = (int)i;
            // the systems are independent: every block of a system's cblk faces a cblk of it
            for (int b = s->fblok[k]; b < s->fblok[k + 1]; b++)
                if (s->fcblk[b] < sys_cblk[i] || s->fcblk[b] >= sys_cblk[i + 1]) return ERR_BADPARAM;
        }
        col[i] = s->fcol[sys_cblk[i]];
        for (int r = col[i]; r < s->fcol[sys_cblk[i + 1]]; r++) segid[r] = (int)i;
    }
    col[nsys] = s->n;
    double *thr = nullptr;
    unsigned long long *npiv = nullptr;
    RET(s->dmalloc(&npiv, (size_t)nsys));
    RET(s->dupload(&s->d_csys, csys));
    RET(s->dupload(&s->d_sys_col, col));
    RET(s->dupload(&s->d_segid, segid));
    RET(s->dmalloc(&thr, (size_t)nsys));
    CU(cudaStreamSynchronize(s->st));
    s->d_thr = thr;
    s->d_npiv = npiv;
    s->ds.csys = s->d_csys;
    s->nsys = (int)nsys;
    // the captured factorization holds the structure tables by value: capture again
    if (s->fact_graph) {
        cudaGraphExecDestroy(s->fact_graph);
        s->fact_graph = nullptr;
    }
    s->factored = false;
    return ERR_SUCCESS;
}

int b200_batch_thresholds(b200_solver_t *s, double *thr, int64_t nsys) {
    if (!s || !thr || s->nsys == 0 || nsys != s->nsys || !s->factored) return ERR_BADPARAM;
    CU(cudaMemcpyAsync(thr, s->d_thr, (size_t)nsys * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    return ERR_SUCCESS;
}

int b200_batch_pivots(b200_solver_t *s, int64_t *npiv, int64_t nsys) {
    if (!s || !npiv || s->nsys == 0 || nsys != s->nsys || !s->factored) return ERR_BADPARAM;
    for (int64_t i = 0; i < nsys; i++) npiv[i] = (int64_t)s->last_piv_sys[i];
    return ERR_SUCCESS;
}

int b200_batch_berr(b200_solver_t *s, double *berr, int64_t count) {
    if (!s || !berr || count != (int64_t)s->last_berr.size() || count == 0) return ERR_BADPARAM;
    std::copy(s->last_berr.begin(), s->last_berr.end(), berr);
    return ERR_SUCCESS;
}

int b200_get_schur(b200_solver_t *s, double *S, int64_t lds) {
    if (!s || !S || !s->factored) return ERR_BADPARAM;
    const int cs = s->cblkschur, N = s->cblknbr;
    const int64_t ns = s->n - s->n1;
    if (cs >= N || lds < ns) return ERR_BADPARAM;
    // the Schur cblks' panels sit at the end of the arena(s)
    const int64_t off0 = s->off[cs], len = s->arena - off0;
    std::vector<double> pl((size_t)len), pu(s->facto == FACTO_GETRF ? (size_t)len : 0);
    auto fetch = [&](const void *arena, std::vector<double> &dst) -> int {
        if (s->f32) {
            std::vector<float> tmp((size_t)len);
            CU(cudaMemcpy(tmp.data(), (const float *)arena + off0, len * sizeof(float), cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < len; i++) dst[i] = tmp[i];
        } else {
            CU(cudaMemcpy(dst.data(), (const double *)arena + off0, len * sizeof(double), cudaMemcpyDeviceToHost));
        }
        return ERR_SUCCESS;
    };
    CU(cudaStreamSynchronize(s->st));
    RET(fetch(s->dL, pl));
    if (s->facto == FACTO_GETRF) RET(fetch(s->dU, pu));
    // coeftab_zgetschur / cpucblk_zgetschur_fr (sopalin/coeftab_z.c:413-437,
    // kernels/cpucblk_zschur.c:114-150): S zeroed, every block of every Schur cblk
    // copied at (its rows, the cblk's columns); for LU the U part added transposed
    for (int64_t j = 0; j < ns; j++) std::fill(S + j * lds, S + j * lds + ns, 0.0);
    for (int k = cs; k < N; k++) {
        const int64_t c0 = s->fcol[k] - s->n1, ld = s->ld[k], po = s->off[k] - off0;
        for (int b = s->fblok[k]; b < s->fblok[k + 1]; b++) {
            const int64_t r0 = s->frow[b] - s->n1, nr = s->lrow[b] - s->frow[b] + 1, ro = s->rowoff[b];
            for (int64_t j = 0; j < s->ncols[k]; j++)
                for (int64_t i = 0; i < nr; i++) {
                    const int64_t src = po + ro + i + j * ld;
                    S[(r0 + i) + (c0 + j) * lds] += pl[(size_t)src];
                    if (s->facto == FACTO_GETRF) S[(c0 + j) + (r0 + i) * lds] += pu[(size_t)src];
                }
        }
    }
    return ERR_SUCCESS;
}

int b200_applyorder(b200_solver_t *s, int dir, int64_t nrhs, double *b, int64_t ldb) {
    if (!s || (dir != 0 && dir != 1) || nrhs < 0 || ldb < s->n || (!b && nrhs)) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    const int n = s->n;
    RET(ensure_ws(&s->main, (size_t)2 * n * nrhs));
    double *d = s->main.d_ws, *p = s->main.d_ws + (size_t)n * nrhs;
    CU(cudaMemcpy2DAsync(d, n * sizeof(double), b, ldb * sizeof(double), n * sizeof(double), nrhs,
                         cudaMemcpyHostToDevice, s->st));
    launch_permute(n, (int)nrhs, s->d_peri, d, n, p, n, dir == 0 ? 1 : 0, s->st);
    CU(cudaMemcpy2DAsync(b, ldb * sizeof(double), p, n * sizeof(double), n * sizeof(double), nrhs,
                         cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    return ERR_SUCCESS;
}

int b200_trsm(b200_solver_t *s, int step, int64_t nrhs, double *b, int64_t ldb) {
    if (!s || !s->factored || step < 0 || step > 2 || nrhs < 0 || ldb < s->n || (!b && nrhs)) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    const int n = s->n;
    RET(ensure_ws(&s->main, (size_t)2 * n * nrhs));
    double *x = s->main.d_ws, *aux = s->main.d_ws + (size_t)n * nrhs;
    CU(cudaMemsetAsync(s->main.d_serr, 0, sizeof(int), s->st));
    CU(cudaMemcpy2DAsync(x, n * sizeof(double), b, ldb * sizeof(double), n * sizeof(double), nrhs,
                         cudaMemcpyHostToDevice, s->st));
    int launches = 0;
    RET(sweep_step(s, &s->main, x, aux, n, (int)nrhs, step, s->st, &launches));
    s->kernel_launches += launches;
    CU(cudaMemcpy2DAsync(b, ldb * sizeof(double), x, n * sizeof(double), n * sizeof(double), nrhs,
                         cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    return sweep_status(&s->main);
}

int b200_spm_values(b200_solver_t *s, const double *values, double anorm) {
    if (!s || s->nnz < 0 || !s->nnz_spm || !values) return ERR_BADPARAM;
    CU(cudaMemcpyAsync(s->d_spmv, values, s->nnz_spm * sizeof(double), cudaMemcpyHostToDevice, s->st));
    RET(b200_spm_values_device(s, s->d_spmv, anorm, s->st));
    CU(cudaStreamSynchronize(s->st));
    return ERR_SUCCESS;
}

int b200_bcsc_load(b200_solver_t *s, int64_t nnz, const int64_t *colptr, const int64_t *rowtab, const double *Lvalues,
                   const double *Uvalues, double anorm) {
    if (!s || nnz < 0 || !colptr || !rowtab || !Lvalues) return ERR_BADPARAM;
    if (s->facto == FACTO_GETRF && !Uvalues) return ERR_BADPARAM;
    const int n = s->n;
    if (colptr[0] != 0 || colptr[n] != nnz) return ERR_BADPARAM;
    bool same = (s->nnz == nnz) && std::equal(colptr, colptr + n + 1, s->h_colptr.begin()) &&
                std::equal(rowtab, rowtab + nnz, s->h_rowtab.begin());
    if (!same) {
        if (s->d_colptr) cudaFree(s->d_colptr);
        if (s->d_rowtab) cudaFree(s->d_rowtab);
        if (s->d_Lv) cudaFree(s->d_Lv);
        if (s->d_Uv) cudaFree(s->d_Uv);
        if (s->d_dest) cudaFree(s->d_dest);
        s->d_colptr = nullptr; s->d_rowtab = nullptr; s->d_Lv = nullptr; s->d_Uv = nullptr; s->d_dest = nullptr;
        s->d_lmap = nullptr; s->d_umap = nullptr; s->d_spmv = nullptr;  // a new pattern invalidates the spm map
        s->nnz_spm = 0;
        if (s->fact_graph) cudaGraphExecDestroy(s->fact_graph);
        s->fact_graph = nullptr;
        s->h_colptr.assign(colptr, colptr + n + 1);
        s->h_rowtab.assign(rowtab, rowtab + nnz);
        // destination of every bcsc entry in the panel arena (cpucblk_zfillin_fr,
        // kernels/cpucblk_zinit.c:229-309): rows above the diagonal are skipped,
        // bit 62 marks strictly-lower entries that also go to the U arena
        std::vector<int64_t> dest(nnz, -1);
        std::vector<int> rows32(nnz);
        for (int k = 0; k < s->cblknbr; k++) {
            for (int col = s->fcol[k]; col < s->fcol[k] + s->ncols[k] && col < n; col++) {
                const int jc = col - s->fcol[k];
                for (int64_t e = colptr[col]; e < colptr[col + 1]; e++) {
                    const int64_t r = rowtab[e];
                    if (r < 0 || r >= n) return ERR_BADPARAM;
                    rows32[e] = (int)r;
                    if (r < col) continue;
                    int lo = s->fblok[k], hi = s->fblok[k + 1] - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (s->frow[mid] <= r) lo = mid; else hi = mid - 1;
                    }
                    if (r < s->frow[lo] || r > s->lrow[lo]) continue;  // dropped, as PaStiX does
                    int64_t d = s->off[k] + s->rowoff[lo] + (r - s->frow[lo]) + (int64_t)jc * s->ld[k];
                    if (r > col) d |= (int64_t)1 << 62;
                    dest[e] = d;
                }
            }
        }
        RET(dalloc(&s->d_colptr, (size_t)n + 1));
        RET(dalloc(&s->d_rowtab, (size_t)nnz));
        RET(dalloc(&s->d_dest, (size_t)nnz));
        RET(dalloc(&s->d_Lv, (size_t)nnz));
        if (Uvalues) RET(dalloc(&s->d_Uv, (size_t)nnz));
        CU(cudaMemcpyAsync(s->d_colptr, colptr, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s->st));
        CU(cudaMemcpyAsync(s->d_rowtab, rows32.data(), nnz * sizeof(int), cudaMemcpyHostToDevice, s->st));
        CU(cudaMemcpyAsync(s->d_dest, dest.data(), nnz * sizeof(int64_t), cudaMemcpyHostToDevice, s->st));
        CU(cudaStreamSynchronize(s->st));
        s->nnz = nnz;
    }
    CU(cudaMemcpyAsync(s->d_Lv, Lvalues, nnz * sizeof(double), cudaMemcpyHostToDevice, s->st));
    if (Uvalues && s->d_Uv) CU(cudaMemcpyAsync(s->d_Uv, Uvalues, nnz * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
    s->anorm = anorm;
    s->factored = false;
    return ERR_SUCCESS;
}

int b200_numfact(b200_solver_t *s, double epsilon_magn_ctrl, int64_t *nbpivots) {
    if (!s || s->nnz < 0) return ERR_BADPARAM;
    // threshold rule of pastix_subtask_sopalin (sopalin/pastix_task_sopalin.c:401-425)
    double thr;
    if (epsilon_magn_ctrl < 0.0) thr = -epsilon_magn_ctrl;
    else if (epsilon_magn_ctrl == 0.0) {
        const double eps = s->f32 ? std::ldexp(1.0, -24) : std::ldexp(1.0, -53);  // LAPACK xlamch('e')
        thr = std::sqrt(eps) * s->anorm;
    } else thr = epsilon_magn_ctrl * s->anorm;
    if (s->nsys > 0) {
        // one threshold per system, from its own norm (computed from the bcsc on the device)
        const double eps = s->f32 ? std::ldexp(1.0, -24) : std::ldexp(1.0, -53);
        const double c = epsilon_magn_ctrl < 0.0 ? -epsilon_magn_ctrl
                                                 : (epsilon_magn_ctrl == 0.0 ? std::sqrt(eps) : epsilon_magn_ctrl);
        launch_batch_threshold(s->nsys, s->d_sys_col, s->d_colptr, s->d_Lv, c, epsilon_magn_ctrl >= 0.0, s->d_thr,
                               s->st);
        CU(cudaGetLastError());
        s->kernel_launches++;
        s->thr_used = -1.0;
    } else {
        s->thr_used = thr;
        CU(cudaMemcpyAsync(s->d_thr, &thr, sizeof(double), cudaMemcpyHostToDevice, s->st));
    }
    if (!s->fact_graph) {
        cudaGraph_t g;
        CU(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
        int rc = s->f32 ? enqueue_numfact<float>(s, s->st) : enqueue_numfact<double>(s, s->st);
        cudaError_t ec = cudaStreamEndCapture(s->st, &g);
        if (rc) return rc;
        CU(ec);
        // B200_GRAPH_DOT=<file>: the captured graph in Graphviz form (debugging aid)
        if (const char *dot = getenv("B200_GRAPH_DOT")) cudaGraphDebugDotPrint(g, dot, 0);
        CU(cudaGraphInstantiate(&s->fact_graph, g, 0));
        cudaGraphDestroy(g);
    }
    CU(cudaEventRecord(s->ev0, s->st));
    CU(cudaGraphLaunch(s->fact_graph, s->st));
    s->kernel_launches += s->launches_fact;
    CU(cudaEventRecord(s->ev1, s->st));
    unsigned long long piv = 0;
    int err = 0;
    s->last_piv_sys.assign(std::max(s->nsys, 1), 0ull);
    CU(cudaMemcpyAsync(s->last_piv_sys.data(), s->d_npiv, s->last_piv_sys.size() * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, s->st));
    CU(cudaMemcpyAsync(&err, s->d_err, sizeof(err), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    for (unsigned long long v : s->last_piv_sys) piv += v;
    float ms = 0;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    s->t_fact = ms;
    s->last_npiv = (int64_t)piv;
    if (nbpivots) *nbpivots = (int64_t)piv;
    if (err & 2) fprintf(stderr, "pastix_b200: a tensor-core update timed out waiting for its operands\n");
    if (err & 8) fprintf(stderr, "pastix_b200: a panel factorization timed out waiting for a tile\n");
    if (err & 32) fprintf(stderr, "pastix_b200: the tree-bottom launch timed out waiting for a cblk's updates\n");
    if (err & 1) fprintf(stderr, "pastix_b200: negative diagonal term in the Cholesky factorization\n");
    if (err) return ERR_INTERNAL;
    s->factored = true;
    return ERR_SUCCESS;
}

int b200_numfact_trace(b200_solver_t *s, double epsilon_magn_ctrl, double *ms, double *flops) {
    if (!s || s->nnz < 0 || !ms) return ERR_BADPARAM;
    int64_t piv = 0;
    RET(b200_numfact(s, epsilon_magn_ctrl, &piv));  // sets the threshold and checks the factorization
    Trace tr;
    tr.detail = &s->trace_detail;
    int rc = s->f32 ? enqueue_numfact<float>(s, s->st, &tr) : enqueue_numfact<double>(s, s->st, &tr);
    if (rc) return rc;
    CU(cudaStreamSynchronize(s->st));
    s->kernel_launches += s->launches_fact;
    tr.finish(ms);
    if (flops) {
        flops[0] = 0.0;
        for (int c = 1; c < 4; c++) flops[c] = s->flops_class[c];
    }
    return ERR_SUCCESS;
}

int b200_solve_trace(b200_solver_t *s, int64_t nrhs, double *ms, double *bytes) {
    if (!s || !s->factored || nrhs <= 0 || !ms) return ERR_BADPARAM;
    const int n = s->n;
    RET(ensure_ws(&s->main, (size_t)2 * n * nrhs));
    double *xp = s->main.d_ws, *aux = s->main.d_ws + (size_t)n * nrhs;
    CU(cudaMemsetAsync(xp, 0, (size_t)n * nrhs * sizeof(double), s->st));
    Trace tr;
    tr.detail = &s->trace_detail;
    int launches = 0;
    tr.begin(s->st);
    tr.end(0, s->st);
    int rc = sweeps(s, &s->main, xp, aux, n, (int)nrhs, s->st, &launches, &tr);
    if (rc) return rc;
    CU(cudaStreamSynchronize(s->st));
    s->kernel_launches += launches;
    tr.finish(ms);
    if (bytes) {
        // algorithmic traffic of each sweep: every factor entry once (diagonal blocks:
        // their inverses' triangles), x_k and aux_k read or written once, the rows
        // below read and written once
        for (int c = 0; c < 4; c++) bytes[c] = 0;
        for (int k = 0; k < s->cblknbr; k++) {
            const double nc = s->ncols[k], m = s->stride[k] - nc, v = (double)nrhs * s->esz;
            const double per_sweep = (nc * nc * 0.5 + m * nc) * s->esz + 2.0 * nc * v + 2.0 * m * v;
            bytes[1] += per_sweep;
            bytes[2] += per_sweep;
        }
    }
    return ERR_SUCCESS;
}

int b200_trace_kinds(b200_solver_t *s, double *ms, double *flops, int nkinds) {
    if (!s || nkinds < 0) return -ERR_BADPARAM;
    const int nk = std::min(nkinds, 9);
    for (int i = 0; i < nk; i++) {
        if (ms) ms[i] = 0.0;
        if (flops) flops[i] = s->flops_kind[i];
    }
    if (ms)
        for (auto &pr : s->trace_detail)
            if (pr.first < nk) ms[pr.first] += pr.second;
    return nk;
}

int64_t b200_trace_launches(b200_solver_t *s, double *ms, int32_t *cls, int64_t cap) {
    if (!s) return -ERR_BADPARAM;
    const int64_t cnt = (int64_t)s->trace_detail.size();
    for (int64_t i = 0; i < cnt && i < cap; i++) {
        if (ms) ms[i] = s->trace_detail[i].second;
        if (cls) cls[i] = s->trace_detail[i].first;
    }
    return cnt;
}

int b200_solve_device(b200_solver_t *s, int64_t nrhs, double *d_b, int64_t ldb, void *stream) {
    if (s && s->cblkschur < s->cblknbr) return ERR_BADPARAM;
    if (!s || !s->factored || nrhs < 0 || ldb < s->n) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    cudaStream_t st = stream ? (cudaStream_t)stream : s->st;
    Lane *ln = nullptr;
    RET(lane_for(s, st, &ln));
    CU(cudaMemsetAsync(ln->d_serr, 0, sizeof(int), st));
    return solve_device(s, ln, (int)nrhs, d_b, ldb, st);
}

int b200_solve_device_noalloc(b200_solver_t *s, int64_t nrhs, double *d_b, int64_t ldb, void *stream) {
    if (s && s->cblkschur < s->cblknbr) return ERR_BADPARAM;
    if (!s || !s->factored || nrhs < 0 || ldb < s->n || (!d_b && nrhs)) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    const int n = s->n;
    if (2 * (uint64_t)n * (uint64_t)nrhs > (uint64_t)B200_NOALLOC_SCRATCH_DOUBLES) {
        fprintf(stderr,
                "pastix_b200: b200_solve_device_noalloc: 2 * n * nrhs = %lld exceeds its fixed scratch of %d doubles\n",
                2LL * n * (long long)nrhs, B200_NOALLOC_SCRATCH_DOUBLES);
        return ERR_BADPARAM;
    }
    // the scratch's address on the instance's device, looked up when it was created
    double *xp = s->noalloc_scratch;
    if (!xp) return ERR_INTERNAL;
    double *aux = xp + (size_t)n * nrhs;
    cudaStream_t st = stream ? (cudaStream_t)stream : s->st;
    // the sweeps' tickets, counters and status word: the main lane's, whatever the
    // stream (allocated with the instance; a stream's own lane would be allocated here)
    Lane *ln = &s->main;
    CU(cudaMemsetAsync(ln->d_serr, 0, sizeof(int), st));
    // every entry of the scratch used here is written before it is read: the first half
    // by the permutation, the second by the forward diagonal products (for an FP32
    // factor, the two float blocks of the sweeps by the conversion and the products)
    int launches = 2;
    launch_permute(n, (int)nrhs, s->d_peri, d_b, ldb, xp, n, 1, st);
    RET(sweeps(s, ln, xp, aux, n, (int)nrhs, st, &launches));
    launch_permute(n, (int)nrhs, s->d_peri, xp, n, d_b, ldb, 0, st);
    CU(cudaGetLastError());
    s->kernel_launches += launches;
    return ERR_SUCCESS;
}

// Bit 4 of a lane's sweep status word: a dataflow sweep of the last solve /
// refinement call on that stream gave up waiting for its inputs (its result is not
// to be used).  Every call that runs sweeps clears the word first.  Read after the
// stream has been synchronized.
static int sweep_status(Lane *ln) {
    int err = 0;
    if (cudaMemcpy(&err, ln->d_serr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return ERR_INTERNAL;
    if (err & 16) {
        fprintf(stderr, "pastix_b200: a solve sweep timed out waiting for its inputs\n");
        return ERR_INTERNAL;
    }
    return ERR_SUCCESS;
}

int b200_solve_status(b200_solver_t *s, void *stream) {
    if (!s) return ERR_BADPARAM;
    Lane *ln = nullptr;
    RET(lane_for(s, stream ? (cudaStream_t)stream : s->st, &ln));
    return sweep_status(ln);
}

int b200_solve(b200_solver_t *s, int64_t nrhs, double *b, int64_t ldb) {
    if (s && s->cblkschur < s->cblknbr) return ERR_BADPARAM;  // the Schur part is the caller's: b200_trsm
    if (!s || !s->factored || nrhs < 0 || ldb < s->n || (!b && nrhs)) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    const int n = s->n;
    RET(ensure_stage(s, (size_t)n * nrhs));
    double *db = s->d_stage;
    int rc = ERR_SUCCESS;
    if (cudaMemsetAsync(s->main.d_serr, 0, sizeof(int), s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc && cudaMemcpy2DAsync(db, n * sizeof(double), b, ldb * sizeof(double), n * sizeof(double), nrhs,
                                 cudaMemcpyHostToDevice, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc) {
        cudaEventRecord(s->ev0, s->st);
        rc = solve_device(s, &s->main, (int)nrhs, db, n, s->st);
        cudaEventRecord(s->ev1, s->st);
    }
    if (!rc && cudaMemcpy2DAsync(b, ldb * sizeof(double), db, n * sizeof(double), n * sizeof(double), nrhs,
                                 cudaMemcpyDeviceToHost, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (cudaStreamSynchronize(s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc) rc = sweep_status(&s->main);
    float ms = 0;
    if (!rc) cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    s->main.t_solve = ms;
    return rc;
}

// Single-precision host vectors (a float matrix's b and x, as pastix_task_solve /
// pastix_task_refine take them for PastixFloat, sopalin/pastix_task_solve.c:550):
// uploaded as floats, widened to double on the device, solved or refined there in
// double and narrowed back.
int b200_solve_float(b200_solver_t *s, int64_t nrhs, float *b, int64_t ldb) {
    if (s && s->cblkschur < s->cblknbr) return ERR_BADPARAM;
    if (!s || !s->factored || nrhs < 0 || ldb < s->n || (!b && nrhs)) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    const int n = s->n;
    const size_t blk = (size_t)n * nrhs;
    RET(ensure_stage(s, blk + (blk + 1) / 2));
    double *db = s->d_stage;
    float *fb = reinterpret_cast<float *>(s->d_stage + blk);
    int rc = ERR_SUCCESS;
    if (cudaMemsetAsync(s->main.d_serr, 0, sizeof(int), s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc && cudaMemcpy2DAsync(fb, n * sizeof(float), b, ldb * sizeof(float), n * sizeof(float), nrhs,
                                 cudaMemcpyHostToDevice, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc) {
        launch_convert<float, double>(n, (int)nrhs, fb, n, db, n, s->st);
        rc = solve_device(s, &s->main, (int)nrhs, db, n, s->st);
    }
    if (!rc) launch_convert<double, float>(n, (int)nrhs, db, n, fb, n, s->st);
    if (!rc && cudaMemcpy2DAsync(b, ldb * sizeof(float), fb, n * sizeof(float), n * sizeof(float), nrhs,
                                 cudaMemcpyDeviceToHost, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (cudaStreamSynchronize(s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc) rc = sweep_status(&s->main);
    s->kernel_launches += 2;
    return rc;
}

int b200_refine_float(b200_solver_t *s, int64_t nrhs, const float *b, int64_t ldb, float *x, int64_t ldx, int method,
                      double eps, int64_t itermax, int64_t gmres_im, int64_t *niter, double *berr) {
    if (!s || !s->factored || nrhs < 0 || ldb < s->n || ldx < s->n) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    const int n = s->n;
    const size_t blk = (size_t)n * nrhs;
    RET(ensure_stage(s, 3 * blk));
    double *db = s->d_stage, *dx = s->d_stage + blk;
    float *fb = reinterpret_cast<float *>(s->d_stage + 2 * blk), *fx = fb + blk;
    int rc = ERR_SUCCESS;
    if (cudaMemcpy2DAsync(fb, n * sizeof(float), b, ldb * sizeof(float), n * sizeof(float), nrhs,
                          cudaMemcpyHostToDevice, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc && cudaMemcpy2DAsync(fx, n * sizeof(float), x, ldx * sizeof(float), n * sizeof(float), nrhs,
                                 cudaMemcpyHostToDevice, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc) {
        launch_convert<float, double>(n, (int)nrhs, fb, n, db, n, s->st);
        launch_convert<float, double>(n, (int)nrhs, fx, n, dx, n, s->st);
        rc = b200_refine_device(s, nrhs, db, n, dx, n, method, eps, itermax, gmres_im, niter, berr, s->st);
    }
    if (!rc) launch_convert<double, float>(n, (int)nrhs, dx, n, fx, n, s->st);
    if (!rc && cudaMemcpy2DAsync(x, ldx * sizeof(float), fx, n * sizeof(float), n * sizeof(float), nrhs,
                                 cudaMemcpyDeviceToHost, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (cudaStreamSynchronize(s->st) != cudaSuccess) rc = ERR_INTERNAL;
    s->kernel_launches += 3;
    return rc;
}

int b200_refine_device(b200_solver_t *s, int64_t nrhs, const double *d_b, int64_t ldb, double *d_x, int64_t ldx,
                       int method, double eps, int64_t itermax, int64_t gmres_im, int64_t *niter, double *berr,
                       void *stream) {
    if (s && s->cblkschur < s->cblknbr) return ERR_BADPARAM;
    if (!s || !s->factored || nrhs < 0 || ldb < s->n || ldx < s->n || method < 0 || method > 3) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    cudaStream_t st = stream ? (cudaStream_t)stream : s->st;
    auto t0 = std::chrono::steady_clock::now();
    Lane *ln = nullptr;
    RET(lane_for(s, st, &ln));
    CU(cudaMemsetAsync(ln->d_serr, 0, sizeof(int), st));
    int rc = refine_device(s, ln, (int)nrhs, d_b, ldb, d_x, ldx, method, eps, itermax, gmres_im, niter, berr, st);
    if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc) rc = sweep_status(ln);
    ln->t_refine = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int b200_refine(b200_solver_t *s, int64_t nrhs, const double *b, int64_t ldb, double *x, int64_t ldx, int method,
                double eps, int64_t itermax, int64_t gmres_im, int64_t *niter, double *berr) {
    if (!s || !s->factored || nrhs < 0 || ldb < s->n || ldx < s->n) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    const int n = s->n;
    RET(ensure_stage(s, (size_t)2 * n * nrhs));
    double *db = s->d_stage, *dx = s->d_stage + (size_t)n * nrhs;
    int rc = ERR_SUCCESS;
    if (cudaMemcpy2DAsync(dx, n * sizeof(double), x, ldx * sizeof(double), n * sizeof(double), nrhs,
                          cudaMemcpyHostToDevice, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc && cudaMemcpy2DAsync(db, n * sizeof(double), b, ldb * sizeof(double), n * sizeof(double), nrhs,
                                 cudaMemcpyHostToDevice, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc) rc = b200_refine_device(s, nrhs, db, n, dx, n, method, eps, itermax, gmres_im, niter, berr, s->st);
    if (!rc && cudaMemcpy2DAsync(x, ldx * sizeof(double), dx, n * sizeof(double), n * sizeof(double), nrhs,
                                 cudaMemcpyDeviceToHost, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (cudaStreamSynchronize(s->st) != cudaSuccess) rc = ERR_INTERNAL;
    return rc;
}

int b200_spmv(b200_solver_t *s, int64_t nrhs, double alpha, const double *x, int64_t ldx, double beta, double *y,
              int64_t ldy) {
    if (!s || s->nnz < 0 || nrhs < 0 || ldx < s->n || ldy < s->n) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    const int n = s->n;
    const size_t blk = (size_t)n * nrhs;
    RET(ensure_stage(s, 4 * blk));
    double *d = s->d_stage;
    double *dx = d, *dy = d + blk, *px = d + 2 * blk, *py = d + 3 * blk;
    int rc = ERR_SUCCESS;
    if (cudaMemcpy2DAsync(dx, n * sizeof(double), x, ldx * sizeof(double), n * sizeof(double), nrhs,
                          cudaMemcpyHostToDevice, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc && cudaMemcpy2DAsync(dy, n * sizeof(double), y, ldy * sizeof(double), n * sizeof(double), nrhs,
                                 cudaMemcpyHostToDevice, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    if (!rc) {
        launch_permute(n, (int)nrhs, s->d_peri, dx, n, px, n, 1, s->st);
        launch_permute(n, (int)nrhs, s->d_peri, dy, n, py, n, 1, s->st);
        const double *vals = (s->facto == FACTO_GETRF) ? s->d_Uv : s->d_Lv;
        if (nrhs > 1 && !s->main.d_xt && dalloc(&s->main.d_xt, (size_t)n * 16)) rc = ERR_OOM;
        if (!rc)
            launch_spmv(n, (int)nrhs, s->d_colptr, s->d_rowtab, vals, px, n, py, n, alpha, beta, s->st, s->main.d_xt);
        launch_permute(n, (int)nrhs, s->d_peri, py, n, dy, n, 0, s->st);
        if (cudaMemcpy2DAsync(y, ldy * sizeof(double), dy, n * sizeof(double), n * sizeof(double), nrhs,
                              cudaMemcpyDeviceToHost, s->st) != cudaSuccess) rc = ERR_INTERNAL;
    }
    if (cudaStreamSynchronize(s->st) != cudaSuccess) rc = ERR_INTERNAL;
    return rc;
}

int b200_spmv_device(b200_solver_t *s, int64_t nrhs, double alpha, const double *d_x, int64_t ldx, double beta,
                     double *d_y, int64_t ldy, void *stream) {
    if (!s || s->nnz < 0 || nrhs < 0 || ldx < s->n || ldy < s->n || nrhs > (1 << 20)) return ERR_BADPARAM;
    if (nrhs == 0) return ERR_SUCCESS;
    if (!d_x || !d_y) return ERR_BADPARAM;
    const int n = s->n;
    const size_t blk = (size_t)n * nrhs;
    cudaStream_t st = stream ? (cudaStream_t)stream : s->st;
    Lane *ln = nullptr;
    RET(lane_for(s, st, &ln));
    RET(ensure_ws(ln, 2 * blk));
    double *px = ln->d_ws, *py = ln->d_ws + blk;
    if (nrhs > 1 && !ln->d_xt) RET(dalloc(&ln->d_xt, (size_t)n * 16));
    const double *vals = (s->facto == FACTO_GETRF) ? s->d_Uv : s->d_Lv;
    launch_permute(n, (int)nrhs, s->d_peri, d_x, ldx, px, n, 1, st);
    launch_permute(n, (int)nrhs, s->d_peri, d_y, ldy, py, n, 1, st);
    launch_spmv(n, (int)nrhs, s->d_colptr, s->d_rowtab, vals, px, n, py, n, alpha, beta, st, ln->d_xt);
    launch_permute(n, (int)nrhs, s->d_peri, py, n, d_y, ldy, 0, st);
    CU(cudaGetLastError());
    s->kernel_launches += 3 + (nrhs > 1 ? 2 * ((nrhs + 15) / 16) : 1);
    return ERR_SUCCESS;
}

int b200_factor_download(b200_solver_t *s, double *L, double *U) {
    if (!s || !L || !s->factored) return ERR_BADPARAM;
    std::vector<char> host((size_t)s->arena * s->esz);
    for (int side = 0; side < 2; side++) {
        double *out = side == 0 ? L : U;
        void *src = side == 0 ? s->dL : s->dU;
        if (!out) continue;
        if (!src) return ERR_BADPARAM;
        CU(cudaMemcpyAsync(host.data(), src, host.size(), cudaMemcpyDeviceToHost, s->st));
        CU(cudaStreamSynchronize(s->st));
        int64_t pos = 0;
        for (int k = 0; k < s->cblknbr; k++) {
            const int nc = s->ncols[k], ld = s->ld[k];
            for (int b = s->fblok[k]; b < s->fblok[k + 1]; b++) {
                const int m = s->lrow[b] - s->frow[b] + 1;
                for (int j = 0; j < nc; j++)
                    for (int i = 0; i < m; i++) {
                        const int64_t src_i = s->off[k] + s->rowoff[b] + i + (int64_t)j * ld;
                        out[pos + i + (int64_t)j * m] =
                            s->f32 ? (double)((float *)host.data())[src_i] : ((double *)host.data())[src_i];
                    }
                pos += (int64_t)m * nc;
            }
        }
    }
    return ERR_SUCCESS;
}

int b200_stats(b200_solver_t *s, double *out) {
    if (!s || !out) return ERR_BADPARAM;
    out[0] = s->t_fact;
    out[1] = s->main.t_solve;
    out[2] = s->main.t_refine;
    out[3] = (double)s->last_npiv;
    out[4] = s->thr_used;
    out[5] = ((double)s->arena + s->winv_elems) * s->esz * (s->dU ? 2 : 1);
    out[6] = (double)s->levels.size();
    out[7] = s->launches_fact;
    out[8] = s->main.launches_solve;
    out[9] = (double)s->coefnbr;
    out[10] = (double)s->kernel_launches;
    out[11] = (double)s->main.ws_cap * sizeof(double);
    out[12] = (double)s->stage_cap * sizeof(double);
    return ERR_SUCCESS;
}

}  // extern "C"
