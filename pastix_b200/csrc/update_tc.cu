// GEMM + scatter-add update of FP32 factors on the 5th-generation tensor cores
// (sm_100a: TMA, tcgen05.mma kind::tf32, accumulators in tensor memory).
//
// Same operation as update_simt_f32_kernel (core_zgemmsp_2d2d,
// kernels/core_zgemmsp.c:396-465): C_f[rows, cols of block j] -= A_k[rows] B_k[j]^T
// with K = ncols_k, scattered into the facing cblk f through the block index map.
//
// Operand copies.  kind::tf32 reads its operands K-major (the MN-major form leaves
// the accumulator untouched on sm_100a) while the factor panels are column-major,
// so once a panel is final (after its TRSM) panel_split_kernel writes it row-major
// (row r of cblk k at toff[k] + r * kp_k, kp_k = ncols_k rounded up to 16 bytes)
// into an operand arena, split for TF32X3: x = hi + lo with hi = x with its 13 low
// mantissa bits cleared (exact in TF32) and lo = x - hi (exact); D += hi_A hi_B +
// hi_A lo_B + lo_A hi_B keeps close to FP32 accuracy.  TF32 keeps x once and D += A B.
// BF16X3 (kind::f16, both operands BF16, FP32 accumulation): hi = x rounded to BF16,
// lo = (x - hi) rounded to BF16, the same three products -- x = hi + lo to about 2^-17
// relative, half the bytes per operand and twice the MMA rate of TF32; a 128-byte
// operand row then holds 64 K values instead of 32.
//
// update_tc_kernel is persistent (one CTA per SM, tiles of 128 rows x at most BN = 64
// or 128 columns striding over the launch's tile list) and warp-specialised:
//  * warp 0 (one lane): TMA producer.  One 2D tensor map per panel copy (K
//    innermost, boxes of 32 K x 64 rows, 128-byte swizzle: stacked, exactly the
//    canonical K-major UMMA layout), a ring of [A hi][B hi]([A lo][B lo]) stages in
//    shared memory, K in chunks of 32.
//  * warp 1 (one lane): allocates 2 BN TMEM columns (two 128 x BN FP32
//    accumulators) and issues tcgen05.mma (M = 128, N = the update's tile width, K =
//    8; the N field of the instruction descriptor is set per tile), skipping the K
//    steps of a chunk's zero-filled tail; each stage is released to the producer and
//    each accumulator to the epilogue by tcgen05.commit on an mbarrier.
//  * warps 2-9: epilogue.  Thread = accumulator row (TMEM lane quarter = warp % 4),
//    two warps per quarter with BN / 2 columns each; tcgen05.ld, release the
//    accumulator, scatter-add into f with reductions (red.global.add), overlapping
//    the next tile's MMAs.
//  * Every mbarrier wait is bounded and also gives up once another role has given
//    up; the kernel then records bit 2 of err, waits (bounded) for its TMA loads and
//    MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include "b200_internal.h"
#include "kernels.h"

namespace b200 {

constexpr int TC_BM = 128, TC_BK = 32;          // TC_BK: K of a 128-byte row of FP32 (TF32) operands
constexpr int TC_A_BYTES = TC_BM * TC_BK * 4;  // 16 KB: 128 rows of 128 bytes, for either format

// operand formats: OP_TF32 (FP32 storage, kind::tf32) and OP_BF16 (kind::f16 on BF16)
enum { OP_TF32 = 0, OP_BF16 = 1 };
template <int OP>
struct OpFmt {
    static constexpr int BK = OP == OP_BF16 ? 64 : 32;     // K values per 128-byte operand row (a stage)
    static constexpr int KSTEP = OP == OP_BF16 ? 16 : 8;   // K of one MMA: 32 bytes of the row
    static constexpr uint32_t FMT = OP == OP_BF16 ? 1u : 2u;  // A/B format in the instruction descriptor
};
constexpr long long TC_WAIT_CYCLES = 1000000000LL;  // about 0.5 s at the maximum SM clock
constexpr int TC_THREADS = 320;  // producer, MMA, 8 epilogue warps
constexpr int TC_EPI_WARPS = 8;

// BN = tile columns (64 or 128); a stage holds [A hi][B hi]([A lo][B lo]), as many
// stages as fit in about 192 KB
template <int SPLIT, int BN>
struct TcCfg {
    static constexpr int B_BYTES = BN * TC_BK * 4;
    static constexpr int STAGE = SPLIT ? 2 * (TC_A_BYTES + B_BYTES) : (TC_A_BYTES + B_BYTES);
    static constexpr int NST = (192 * 1024) / STAGE;
    static constexpr int SMEM = NST * STAGE + 1024;  // + alignment slack
    static constexpr uint32_t TMEM_COLS = 2 * BN;    // two accumulators
};

// instruction descriptor: D F32, A and B of the same format fmt (TF32 = 2 for
// kind::tf32, BF16 = 1 for kind::f16), both K-major, M = 128, N = n (a multiple of 16)
__device__ __forceinline__ uint32_t tc_idesc(int n, uint32_t fmt) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the given phase parity.  Returns false if the limit expired or,
// when abort is given, once *abort is set by another role.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort) {
    const long long t0 = clock64();
    for (int it = 0;; it++) {
        if (mbar_test(bar, parity)) return true;
        if ((it & 63) == 63) {
            if (abort && *abort) return false;
            if (clock64() - t0 > TC_WAIT_CYCLES) return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// UMMA shared-memory descriptor, 128-byte swizzle: K-major operand with one
// 128-byte line per row, SBO = 1024 bytes between 8-row groups; LBO unused.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                  // LBO (ignored for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;        // SBO
    d |= (uint64_t)1 << 46;                  // descriptor version (sm100)
    d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
    return d;
}

template <int OP>
__device__ __forceinline__ void umma_op(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc,
                                        uint32_t accumulate) {
    if (OP == OP_BF16)
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
            : "memory");
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
            : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}

// Tile t of the launch from the host-built tile map {update, row tile | column
// tile << 16} (tiles entirely above the diagonal of a symmetric update are not
// listed): two loads instead of a search.
struct TcTile {
    Upd u;
    int mt, nt;
};

__device__ __forceinline__ void tc_decode(const Upd *__restrict__ upds, const int2 *__restrict__ tmap, int t,
                                          TcTile &tt) {
    const int2 e = tmap[t];
    tt.u = upds[e.x];
    tt.mt = e.y & 0xffff;
    tt.nt = e.y >> 16;
}

// ---------------------------------------------------------------- operand copies

// 16 bytes of one operand row (4 FP32 or 8 BF16 values), split into hi and lo and
// stored as one vector each.
__device__ __forceinline__ void split_store16(float *dh, float *dl, size_t i, const float (&x)[4]) {
    float h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        h[j] = dl ? __uint_as_float(__float_as_uint(x[j]) & 0xFFFFE000u) : x[j];
        l[j] = x[j] - h[j];
    }
    *reinterpret_cast<float4 *>(dh + i) = make_float4(h[0], h[1], h[2], h[3]);
    if (dl) *reinterpret_cast<float4 *>(dl + i) = make_float4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ void split_store16(__nv_bfloat16 *dh, __nv_bfloat16 *dl, size_t i, const float (&x)[8]) {
    __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        h[j] = __float2bfloat16_rn(x[j]);
        l[j] = __float2bfloat16_rn(x[j] - __bfloat162float(h[j]));
    }
    *reinterpret_cast<uint4 *>(dh + i) = *reinterpret_cast<const uint4 *>(h);
    if (dl) *reinterpret_cast<uint4 *>(dl + i) = *reinterpret_cast<const uint4 *>(l);
}

// One 64 x 64 tile of a panel (rows row0 .., a multiple of 4; columns col0 ..) to the
// row-major operand arena(s) of element type E (float for TF32 operands, BF16); the row
// pitch kp is ncols rounded up to 16 bytes, columns ncols .. kp - 1 written as zeros.
// Loads: four consecutive rows of one column as one 16-byte vector (panels start on
// 256-byte boundaries and their leading dimension is a multiple of 4); stores: 16 bytes
// of one row per thread and part (4 FP32 or 8 BF16 columns), through a padded transpose.
template <typename E>
__global__ void __launch_bounds__(256) panel_split_kernel(DevSym s, const SplitTask *__restrict__ tasks,
                                                          const float *__restrict__ P,
                                                          const int64_t *__restrict__ toff, E *hi, E *lo) {
    __shared__ float t[64][65];  // t[column][row]
    constexpr int PAD = 16 / sizeof(E);
    const SplitTask tk = tasks[blockIdx.x];
    const int k = tk.k, tid = threadIdx.x;
    const int stride = s.stride[k], nc = s.ncols[k], ld = s.ld[k], kp = (nc + PAD - 1) / PAD * PAD;
    const float *src = P + s.off[k];
    float4 v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int idx = tid + 256 * u, r = tk.row0 + 4 * (idx & 15), c = tk.col0 + (idx >> 4);
        const float *p = src + r + (size_t)c * ld;
        if (c < nc && r + 3 < stride) {
            v[u] = __ldg(reinterpret_cast<const float4 *>(p));
        } else {
            v[u].x = (c < nc && r < stride) ? p[0] : 0.f;
            v[u].y = (c < nc && r + 1 < stride) ? p[1] : 0.f;
            v[u].z = (c < nc && r + 2 < stride) ? p[2] : 0.f;
            v[u].w = 0.f;
        }
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int idx = tid + 256 * u, r4 = 4 * (idx & 15), c = idx >> 4;
        t[c][r4] = v[u].x;
        t[c][r4 + 1] = v[u].y;
        t[c][r4 + 2] = v[u].z;
        t[c][r4 + 3] = v[u].w;
    }
    __syncthreads();
    E *dh = hi + toff[k];
    E *dl = lo ? lo + toff[k] : nullptr;
    constexpr int VE = 16 / sizeof(E), G = 64 / VE;  // values per 16-byte unit, units per tile row
#pragma unroll
    for (int u = 0; u < 64 * G / 256; u++) {
        const int idx = tid + 256 * u, g = idx % G, rr = idx / G;
        const int r = tk.row0 + rr, c0 = tk.col0 + VE * g;
        if (r < stride && c0 < kp) {
            float x[VE];
#pragma unroll
            for (int j = 0; j < VE; j++) x[j] = t[VE * g + j][rr];
            split_store16(dh, dl, (size_t)r * kp + c0, x);
        }
    }
}

void launch_panel_split(const DevSym &s, const SplitTask *tasks, int ntasks, const float *P, const int64_t *toff,
                        void *hi, void *lo, int op, cudaStream_t st) {
    if (ntasks <= 0) return;
    if (op == OP_BF16)
        panel_split_kernel<__nv_bfloat16><<<ntasks, 256, 0, st>>>(
            s, tasks, P, toff, static_cast<__nv_bfloat16 *>(hi), static_cast<__nv_bfloat16 *>(lo));
    else
        panel_split_kernel<float><<<ntasks, 256, 0, st>>>(s, tasks, P, toff, static_cast<float *>(hi),
                                                          static_cast<float *>(lo));
}

// ---------------------------------------------------------------- GEMM-scatter

// maps[(side * 2 + part) * cblknbr + k]: side 0 L / 1 U, part 0 hi / 1 lo
template <int SPLIT, int BN, int OP>
__global__ void __launch_bounds__(TC_THREADS, 1) update_tc_kernel(DevSym s, const Upd *__restrict__ upds,
                                                                  const int2 *__restrict__ tmap, int ntiles,
                                                                  const CUtensorMap *__restrict__ maps,
                                                                  float *L, float *U, int *err) {
    using Cfg = TcCfg<SPLIT, BN>;
    using Fmt = OpFmt<OP>;
    constexpr int BK = Fmt::BK;  // K values per stage (one 128-byte operand row)
    constexpr int TC_B_BYTES = Cfg::B_BYTES;
    constexpr int TC_BN = BN;
    constexpr uint32_t TC_TMEM_COLS = Cfg::TMEM_COLS;
    constexpr int ECOLS = BN / 2;  // columns per epilogue warp
    constexpr int NST = Cfg::NST;
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[NST];
    __shared__ __align__(8) uint64_t empty_bar[NST];
    __shared__ __align__(8) uint64_t tfull_bar[2];
    __shared__ __align__(8) uint64_t tempty_bar[2];
    __shared__ __align__(8) uint64_t fin_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_sh;

    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int N = s.cblknbr;

    if (tid == 0) {
        for (int i = 0; i < NST; i++) {
            mbar_init(smem_addr(&full_bar[i]), 1);
            mbar_init(smem_addr(&empty_bar[i]), 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(smem_addr(&tfull_bar[i]), 1);
            mbar_init(smem_addr(&tempty_bar[i]), TC_EPI_WARPS);  // one arrival per epilogue warp
        }
        mbar_init(smem_addr(&fin_bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        abort_sh = 0;
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_addr(&tmem_base_sh)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            int it = 0;
            int last_ph[NST];
#pragma unroll
            for (int i = 0; i < NST; i++) last_ph[i] = -1;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                TcTile tt;
                tc_decode(upds, tmap, t, tt);
                const Upd &u = tt.u;
                const int side_a = (u.flags & UPD_A_U) ? 1 : 0, side_b = (u.flags & UPD_B_U) ? 1 : 0;
                const CUtensorMap *ma = maps + (size_t)(side_a * 2) * N + u.k;
                const CUtensorMap *mb = maps + (size_t)(side_b * 2) * N + u.k;
                const int nb = u.nb;  // this update's tile width: nb / 64 boxes of B rows
                const int ya = u.rowA0 + tt.mt * TC_BM, yb = u.rowB0 + tt.nt * nb;
                const int nk = (u.K + BK - 1) / BK;
                const uint32_t tx = (uint32_t)(TC_A_BYTES + nb * 128) * (SPLIT ? 2u : 1u);
                for (int kc = 0; kc < nk; kc++, it++) {
                    const int st = it % NST;
                    if (it >= NST && !mbar_wait(smem_addr(&empty_bar[st]), ((it / NST) - 1) & 1, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    const uint32_t bar = smem_addr(&full_bar[st]);
                    mbar_expect_tx(bar, tx);
                    last_ph[st] = (it / NST) & 1;
                    const uint32_t base = smem_addr(smem + (size_t)st * Cfg::STAGE);
                    const int x = kc * BK + u.colK0;
#pragma unroll
                    for (int g = 0; g < TC_BM / 64; g++) tma_load_2d(base + g * 8192, ma, x, ya + 64 * g, bar);
                    for (int g = 0; g < nb / 64; g++) tma_load_2d(base + TC_A_BYTES + g * 8192, mb, x, yb + 64 * g, bar);
                    if (SPLIT) {
                        const uint32_t lb = base + TC_A_BYTES + TC_B_BYTES;
#pragma unroll
                        for (int g = 0; g < TC_BM / 64; g++) tma_load_2d(lb + g * 8192, ma + N, x, ya + 64 * g, bar);
                        for (int g = 0; g < nb / 64; g++)
                            tma_load_2d(lb + TC_A_BYTES + g * 8192, mb + N, x, yb + 64 * g, bar);
                    }
                }
            }
            if (!ok) abort_sh = 1;
            // the loads still in flight land before the CTA exits
            for (int i = 0; i < NST; i++)
                if (last_ph[i] >= 0) mbar_wait(smem_addr(&full_bar[i]), (uint32_t)last_ph[i], nullptr);
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            int it = 0, tl = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                TcTile tt;
                tc_decode(upds, tmap, t, tt);
                const int a = tl & 1;
                if (tl >= 2 && !mbar_wait(smem_addr(&tempty_bar[a]), ((tl >> 1) - 1) & 1, &abort_sh)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(a * TC_BN);
                const int nk = (tt.u.K + BK - 1) / BK;
                const uint32_t idesc = tc_idesc(tt.u.nb, Fmt::FMT);
                for (int kc = 0; kc < nk; kc++, it++) {
                    const int st = it % NST;
                    if (!mbar_wait(smem_addr(&full_bar[st]), (it / NST) & 1, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const uint32_t base = smem_addr(smem + (size_t)st * Cfg::STAGE);
                    const uint32_t a_hi = base, b_hi = base + TC_A_BYTES;
                    const uint32_t a_lo = base + TC_A_BYTES + TC_B_BYTES, b_lo = a_lo + TC_A_BYTES;
                    // K steps holding data: the chunk's zero-filled tail (K past the
                    // cblk's columns, read as zeros by the TMA) contributes nothing
                    const int ksn = min(4, (tt.u.K - kc * BK + Fmt::KSTEP - 1) / Fmt::KSTEP);
#pragma unroll
                    for (int ks = 0; ks < 4; ks++) {
                        if (ks >= ksn) break;
                        // K step: 32 bytes into each row line (8 TF32 or 16 BF16 values)
                        const uint64_t dah = umma_desc(a_hi + 32 * ks), dbh = umma_desc(b_hi + 32 * ks);
                        umma_op<OP>(acc, dah, dbh, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
                        if (SPLIT) {
                            umma_op<OP>(acc, dah, umma_desc(b_lo + 32 * ks), idesc, 1u);
                            umma_op<OP>(acc, umma_desc(a_lo + 32 * ks), dbh, idesc, 1u);
                        }
                    }
                    umma_commit(smem_addr(&empty_bar[st]));
                }
                if (!ok) break;
                umma_commit(smem_addr(&tfull_bar[a]));
                tl++;
            }
            if (!ok) abort_sh = 1;
            // every MMA issued has completed before the TMEM is freed
            umma_commit(smem_addr(&fin_bar));
            mbar_wait(smem_addr(&fin_bar), 0, nullptr);
        }
    } else {
        // ------------------------------------------------ epilogue (warps 2-9)
        const int q = warp & 3;                 // TMEM lane quarter this warp may access
        const int c0 = ((warp - 2) >> 2) * ECOLS;  // its half of the BN columns
        const int row = q * 32 + lane;
        int tl = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            TcTile tt;
            tc_decode(upds, tmap, t, tt);
            const Upd &u = tt.u;
            const int a = tl & 1;
            const int lr = tt.mt * TC_BM + row;
            const int d = lr < u.M ? __ldg(s.rmap + u.rm0 + lr) : -1;  // destination row in f
            if (!mbar_wait(smem_addr(&tfull_bar[a]), (tl >> 1) & 1, &abort_sh)) {
                abort_sh = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            uint32_t v[ECOLS];
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * TC_BN + c0);
#pragma unroll
            for (int cb = 0; cb < ECOLS; cb += 16) {
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];\n"
                    : "=r"(v[cb + 0]), "=r"(v[cb + 1]), "=r"(v[cb + 2]), "=r"(v[cb + 3]), "=r"(v[cb + 4]),
                      "=r"(v[cb + 5]), "=r"(v[cb + 6]), "=r"(v[cb + 7]), "=r"(v[cb + 8]), "=r"(v[cb + 9]),
                      "=r"(v[cb + 10]), "=r"(v[cb + 11]), "=r"(v[cb + 12]), "=r"(v[cb + 13]), "=r"(v[cb + 14]),
                      "=r"(v[cb + 15])
                    : "r"(taddr + (uint32_t)cb)
                    : "memory");
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            // the accumulator may be overwritten by the next tile's MMAs
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&tempty_bar[a]));
            if (d >= 0) {
                // reductions without a returned value: no load latency on the SM, and
                // consecutive rows of a warp merge into one L2 transaction per column
                float *C = ((u.flags & UPD_C_U) ? U : L) + s.off[u.f];
                const size_t ldf = (size_t)s.ld[u.f];
                // columns of this warp's half inside the tile's nb (TMEM columns past nb
                // hold another tile's values and are never stored)
                const int cmax = min(u.nb, u.N - tt.nt * u.nb) - c0;
                const int csym = (u.flags & UPD_SYM) ? lr - tt.nt * u.nb - c0 : ECOLS - 1;  // last column kept
                const int cend = min(cmax, csym + 1);
                float *p = C + d + (size_t)(u.colbase + tt.nt * u.nb + c0) * ldf;
#pragma unroll
                for (int c = 0; c < ECOLS; c++)
                    if (c < cend) atomicAdd(p + (size_t)c * ldf, -__uint_as_float(v[c]));
            }
            tl++;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (tid == 0 && abort_sh) atomicOr(err, 2);
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_TMEM_COLS));
    }
}

static int g_num_sms = 0;

template <int SPLIT, int BN, int OP>
static void launch_tc(const DevSym &s, const Upd *upds, const int2 *tmap, int ntiles, const CUtensorMap *m, float *L,
                      float *U, int *err, cudaStream_t st) {
    const int grid = ntiles < g_num_sms ? ntiles : g_num_sms;
    update_tc_kernel<SPLIT, BN, OP><<<grid, TC_THREADS, TcCfg<SPLIT, BN>::SMEM, st>>>(s, upds, tmap, ntiles, m, L, U,
                                                                                    err);
}

void launch_update_tc(const DevSym &s, const Upd *upds, const int2 *tmap, int ntiles, const void *maps, float *L,
                      float *U, int split, int bn, int op, int *err, cudaStream_t st) {
    if (ntiles <= 0) return;
    const CUtensorMap *m = static_cast<const CUtensorMap *>(maps);
    if (op == OP_BF16) {
        // BF16 operands are always split (hi + lo): three products
        if (bn == 128) launch_tc<1, 128, OP_BF16>(s, upds, tmap, ntiles, m, L, U, err, st);
        else launch_tc<1, 64, OP_BF16>(s, upds, tmap, ntiles, m, L, U, err, st);
    } else if (bn == 128) {
        if (split) launch_tc<1, 128, OP_TF32>(s, upds, tmap, ntiles, m, L, U, err, st);
        else launch_tc<0, 128, OP_TF32>(s, upds, tmap, ntiles, m, L, U, err, st);
    } else {
        if (split) launch_tc<1, 64, OP_TF32>(s, upds, tmap, ntiles, m, L, U, err, st);
        else launch_tc<0, 64, OP_TF32>(s, upds, tmap, ntiles, m, L, U, err, st);
    }
}

template <int SPLIT, int BN, int OP>
static int tc_set_smem() {
    return (int)cudaFuncSetAttribute(update_tc_kernel<SPLIT, BN, OP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcCfg<SPLIT, BN>::SMEM);
}

int configure_tc_kernels() {
    int dev = 0, rc = 0;
    rc |= (int)cudaGetDevice(&dev);
    rc |= (int)cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    rc |= tc_set_smem<0, 64, OP_TF32>() | tc_set_smem<1, 64, OP_TF32>() | tc_set_smem<0, 128, OP_TF32>() |
          tc_set_smem<1, 128, OP_TF32>() | tc_set_smem<1, 64, OP_BF16>() | tc_set_smem<1, 128, OP_BF16>();
    return rc == 0 && g_num_sms > 0 ? 0 : -1;
}

// One 2D tensor map per operand copy (K innermost: ncols x stride with row pitch kp =
// ncols rounded up to 16 bytes), boxes of one 128-byte row (32 FP32 or 64 BF16 values)
// x 64 rows with 128-byte swizzle; elements past ncols or stride read as zero.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_operand_maps(const std::vector<int64_t> &toff, const std::vector<int> &stride,
                        const std::vector<int> &ncols, const std::vector<char> &wanted, void *arena, int op,
                        CUtensorMap *maps) {
    static EncodeTiledFn encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return -1;
        encode = reinterpret_cast<EncodeTiledFn>(fn);
    }
    const size_t n = toff.size();
    const int esz = op == OP_BF16 ? 2 : 4, pad = 16 / esz;
    for (size_t k = 0; k < n; k++) {
        maps[k] = CUtensorMap{};
        if (!wanted[k] || !arena) continue;
        const int kp = (ncols[k] + pad - 1) / pad * pad;
        cuuint64_t dims[2] = {(cuuint64_t)ncols[k], (cuuint64_t)stride[k]};
        cuuint64_t strides[1] = {(cuuint64_t)kp * esz};
        cuuint32_t box[2] = {(cuuint32_t)(128 / esz), 64};
        cuuint32_t estr[2] = {1, 1};
        CUresult r = encode(&maps[k], op == OP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                            2, static_cast<char *>(arena) + toff[k] * esz, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return -2;
    }
    return 0;
}

}  // namespace b200
