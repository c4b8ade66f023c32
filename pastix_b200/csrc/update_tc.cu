// GEMM + scatter-add update of FP32 factors on the 5th-generation tensor cores
// (sm_100a: TMA, tcgen05.mma kind::tf32, accumulator in tensor memory).
//
// Same operation as update_simt_f32_kernel (core_zgemmsp_2d2d,
// kernels/core_zgemmsp.c:396-465): C_f[rows, cols of block j] -= A_k[rows] B_k[j]^T
// with K = ncols_k, scattered into the facing cblk f through the block index map.
//
//  * Operands are read from the factor panels by TMA through one 2D tensor map per
//    cblk panel (rows x columns, leading dimension ld_k), boxes of 32 rows x 32
//    columns with 128-byte swizzle (rows of the panel contiguous).  A TMA row
//    coordinate must be a multiple of 4 FP32 elements, so a tile starts at the row
//    rounded down to 4 and the rows above the update's range are masked in the
//    epilogue.  3-stage TMA ring over K in chunks of 32.
//  * kind::tf32 reads its operands K-major (the MN-major form leaves the
//    accumulator untouched on sm_100a), so all threads transpose each chunk into
//    the K-major 128-byte-swizzled layout (one 128-byte line of 32 K values per
//    row) of a double-buffered operand area, splitting on the way for TF32X3:
//    x = hi + lo with hi = x with its 13 low mantissa bits cleared (exact in TF32)
//    and lo = x - hi (exact); D += hi_A hi_B + hi_A lo_B + lo_A hi_B keeps close
//    to FP32 accuracy.  TF32 stores x once and D += A B.
//  * One thread issues tcgen05.mma (M = 128, N = 64, K = 8 per instruction) into
//    a 128 x 64 FP32 accumulator in TMEM and commits each operand buffer to an
//    mbarrier; the transposition of chunk c + 1 overlaps the MMAs of chunk c.
//  * Epilogue: tcgen05.ld rows of TMEM (one row per thread), scatter-add into f.
//  * Every mbarrier wait is bounded; on expiry the kernel records an error
//    (bit 2 of err), skips its writes, frees its TMEM and returns.
#include <cuda.h>

#include "b200_internal.h"
#include "kernels.h"

namespace b200 {

constexpr int TC_BM = 128, TC_BN = 64, TC_BK = 32, TC_ST = 3;
constexpr int TC_A_BYTES = TC_BM * TC_BK * 4;           // 16 KB
constexpr int TC_B_BYTES = TC_BN * TC_BK * 4;           // 8 KB
constexpr int TC_RAW_BYTES = TC_A_BYTES + TC_B_BYTES;   // one TMA stage: [A][B], MN-major
constexpr int TC_OP_BYTES = 2 * TC_RAW_BYTES;           // one operand buffer: [A hi][A lo][B hi][B lo], K-major
constexpr int TC_SMEM = TC_ST * TC_RAW_BYTES + 2 * TC_OP_BYTES + 1024;  // + alignment slack
constexpr uint32_t TC_TMEM_COLS = 64;
constexpr long long TC_WAIT_CYCLES = 1000000000LL;  // about 0.5 s at the maximum SM clock

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait for the given phase parity; returns false if the limit expired.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (clock64() - t0 < TC_WAIT_CYCLES) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// UMMA shared-memory descriptor, 128-byte swizzle: K-major operand with one
// 128-byte line per row, SBO = stride between 8-row groups (bytes); LBO unused.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm100)
    d |= (uint64_t)2 << 61;  // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D F32, A/B TF32, both K-major, M = 128, N = 64.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                              ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(TC_IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ int tc_find_update(const Upd *__restrict__ upds, int nupd, int tile) {
    int lo = 0, hi = nupd - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (upds[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int tc_dest_row(const DevSym &s, int k, int f, int prow) {
    int lo = s.fblok[k], hi = s.fblok[k + 1] - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s.rowoff[mid] <= prow) lo = mid; else hi = mid - 1;
    }
    const int grow = s.frow[lo] + (prow - s.rowoff[lo]);
    int flo = s.fblok[f], fhi = s.fblok[f + 1] - 1;
    while (flo < fhi) {
        const int mid = (flo + fhi + 1) >> 1;
        if (s.frow[mid] <= grow) flo = mid; else fhi = mid - 1;
    }
    if (grow > s.lrow[flo]) return -1;
    return s.rowoff[flo] + (grow - s.frow[flo]);
}

// One 4-row x 4-K block: MN-major TMA tile (32-row boxes of 4 KB: K line of 128
// bytes, 16-byte chunk (r/4) ^ (K % 8)) -> K-major tile (row line of 128 bytes,
// 8-row groups of 1 KB, chunk (K/4) ^ (r % 8)).  Thread p of each group of 8 takes
// row group 8x + p and K group (p + c) % 8, which keeps both the 16-byte loads and
// the 16-byte stores of a group free of bank conflicts.
template <int SPLIT>
__device__ __forceinline__ void tc_transpose_block(const unsigned char *src, unsigned char *hi, unsigned char *lo,
                                                   int rg, int kg) {
    const int r0 = 4 * rg, kk0 = 4 * kg;
    float4 v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int kk = kk0 + j;
        v[j] = *reinterpret_cast<const float4 *>(src + (r0 >> 5) * 4096 + kk * 128 +
                                                  ((((r0 & 31) >> 2) ^ (kk & 7)) << 4));
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = r0 + i;
        const float4 w = i == 0 ? make_float4(v[0].x, v[1].x, v[2].x, v[3].x)
                       : i == 1 ? make_float4(v[0].y, v[1].y, v[2].y, v[3].y)
                       : i == 2 ? make_float4(v[0].z, v[1].z, v[2].z, v[3].z)
                                : make_float4(v[0].w, v[1].w, v[2].w, v[3].w);
        const int off = (r >> 3) * 1024 + (r & 7) * 128 + ((kg ^ (r & 7)) << 4);
        if (SPLIT) {
            const float4 wh = make_float4(__uint_as_float(__float_as_uint(w.x) & 0xFFFFE000u),
                                          __uint_as_float(__float_as_uint(w.y) & 0xFFFFE000u),
                                          __uint_as_float(__float_as_uint(w.z) & 0xFFFFE000u),
                                          __uint_as_float(__float_as_uint(w.w) & 0xFFFFE000u));
            *reinterpret_cast<float4 *>(hi + off) = wh;
            *reinterpret_cast<float4 *>(lo + off) = make_float4(w.x - wh.x, w.y - wh.y, w.z - wh.z, w.w - wh.w);
        } else {
            *reinterpret_cast<float4 *>(hi + off) = w;
        }
    }
}

template <int SPLIT>
__global__ void __launch_bounds__(128, 1) update_tc_kernel(DevSym s, const Upd *__restrict__ upds, int nupd,
                                                           const CUtensorMap *__restrict__ mapL,
                                                           const CUtensorMap *__restrict__ mapU, float *L, float *U,
                                                           int *err) {
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[TC_ST];
    __shared__ __align__(8) uint64_t mma_bar[2];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int drow[TC_BM];
    __shared__ volatile int abort_sh;

    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
    unsigned char *raw = smem;                          // TC_ST TMA stages
    unsigned char *opnd = smem + TC_ST * TC_RAW_BYTES;  // 2 operand buffers
    const int tid = threadIdx.x, warp = tid >> 5;

    const Upd u = upds[tc_find_update(upds, nupd, blockIdx.x)];
    const int lt = blockIdx.x - u.tile0;
    const int mt = lt % u.tiles_m, nt = lt / u.tiles_m;
    const int rA = u.rowA0 & 3, rB = u.rowB0 & 3;
    const int lm0 = mt * TC_BM - rA;  // first local row of the tile (may be negative)
    const int ln0 = nt * TC_BN - rB;
    const bool sym = (u.flags & UPD_SYM) != 0;
    // a tile entirely above the diagonal of a symmetric update has nothing to do
    if (sym && lm0 + TC_BM - 1 < ln0) return;
    // once a tile has timed out, the remaining tiles of the factorization do nothing
    if (*reinterpret_cast<volatile int *>(err) & 2) return;

    const int k = u.k;
    const CUtensorMap *ma = ((u.flags & UPD_A_U) ? mapU : mapL) + k;
    const CUtensorMap *mb = ((u.flags & UPD_B_U) ? mapU : mapL) + k;
    const int xa = u.rowA0 + lm0;  // multiple of 4
    const int xb = u.rowB0 + ln0;
    const int nk = (u.K + TC_BK - 1) / TC_BK;

    if (tid == 0) {
        for (int st = 0; st < TC_ST; st++) mbar_init(smem_addr(&full_bar[st]), 1);
        mbar_init(smem_addr(&mma_bar[0]), 1);
        mbar_init(smem_addr(&mma_bar[1]), 1);
        mbar_init(smem_addr(&done_bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        abort_sh = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_addr(&tmem_base_sh)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    {
        const int lr = lm0 + tid;
        drow[tid] = (lr >= 0 && lr < u.M) ? tc_dest_row(s, k, u.f, u.rowA0 + lr) : -1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    auto issue_loads = [&](int st, int kc) {
        const uint32_t bar = smem_addr(&full_bar[st]);
        mbar_expect_tx(bar, TC_RAW_BYTES);
        unsigned char *base = raw + (size_t)st * TC_RAW_BYTES;
        const int y = kc * TC_BK + u.colK0;
#pragma unroll
        for (int g = 0; g < TC_BM / 32; g++) tma_load_2d(smem_addr(base + g * 4096), ma, xa + 32 * g, y, bar);
#pragma unroll
        for (int g = 0; g < TC_BN / 32; g++)
            tma_load_2d(smem_addr(base + TC_A_BYTES + g * 4096), mb, xb + 32 * g, y, bar);
    };

    bool ok = true;
    if (tid == 0) {
        for (int st = 0; st < TC_ST && st < nk; st++) issue_loads(st, st);
    }
    const int p8 = tid & 7, w8 = tid >> 3;
    for (int kc = 0; kc < nk; kc++) {
        const int st = kc % TC_ST;
        const int b = kc & 1;
        // operands of chunk kc arrived; the MMAs of chunk kc - 2 released operand
        // buffer b.  A failed wait is published before the barrier, so every thread
        // leaves the loop together.
        if (ok && !mbar_wait(smem_addr(&full_bar[st]), (kc / TC_ST) & 1)) ok = false;
        if (ok && kc >= 2 && !mbar_wait(smem_addr(&mma_bar[b]), ((kc >> 1) - 1) & 1)) ok = false;
        if (!ok) abort_sh = 1;
        if (ok) {
            const unsigned char *src = raw + (size_t)st * TC_RAW_BYTES;
            unsigned char *ob = opnd + (size_t)b * TC_OP_BYTES;
#pragma unroll
            for (int it = 0; it < 2; it++) {
                const int combo = w8 + 16 * it;
                tc_transpose_block<SPLIT>(src, ob, ob + TC_A_BYTES, 8 * (combo & 3) + p8, (p8 + (combo >> 2)) & 7);
            }
            tc_transpose_block<SPLIT>(src + TC_A_BYTES, ob + 2 * TC_A_BYTES, ob + 2 * TC_A_BYTES + TC_B_BYTES,
                                      8 * (w8 & 1) + p8, (p8 + (w8 >> 1)) & 7);
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (abort_sh) break;
        if (tid == 0) {
            // stage st has been read by every thread: refill it with chunk kc + TC_ST
            if (kc + TC_ST < nk) issue_loads(st, kc + TC_ST);
            const uint32_t ob = smem_addr(opnd + (size_t)b * TC_OP_BYTES);
            const uint32_t a_hi = ob, a_lo = ob + TC_A_BYTES, b_hi = ob + 2 * TC_A_BYTES,
                           b_lo = ob + 2 * TC_A_BYTES + TC_B_BYTES;
#pragma unroll
            for (int t = 0; t < TC_BK / 8; t++) {
                // K step t: 8 values = 32 bytes into each row line
                const uint64_t dah = umma_desc(a_hi + 32 * t, 16, 1024);
                const uint64_t dbh = umma_desc(b_hi + 32 * t, 16, 1024);
                umma_tf32(tmem, dah, dbh, (kc > 0 || t > 0) ? 1u : 0u);
                if (SPLIT) {
                    umma_tf32(tmem, dah, umma_desc(b_lo + 32 * t, 16, 1024), 1u);
                    umma_tf32(tmem, umma_desc(a_lo + 32 * t, 16, 1024), dbh, 1u);
                }
            }
            umma_commit(smem_addr(&mma_bar[b]));
        }
    }
    if (tid == 0) umma_commit(smem_addr(&done_bar));
    if (!mbar_wait(smem_addr(&done_bar), 0)) abort_sh = 1;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    __syncthreads();
    const bool aborted = abort_sh != 0;
    if (!aborted) {
        // epilogue: thread = row (TMEM lane), 4 x 16 columns
        const int r = tid;
        const int d = drow[r];
        const int lr = lm0 + r;
        float *C = ((u.flags & UPD_C_U) ? U : L) + s.off[u.f];
        const int ldf = s.ld[u.f];
        const bool atomic = (u.flags & UPD_ATOMIC) != 0;
#pragma unroll
        for (int cb = 0; cb < TC_BN; cb += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                "tcgen05.wait::ld.sync.aligned;\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr)
                : "memory");
            if (d >= 0) {
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const int lc = ln0 + cb + q;
                    if (lc < 0 || lc >= u.N) continue;
                    if (sym && lr < lc) continue;
                    float *p = C + d + (size_t)(u.colbase + lc) * ldf;
                    const float val = __uint_as_float(v[q]);
                    if (atomic) atomicAdd(p, -val);
                    else *p -= val;
                }
            }
        }
    } else if (tid == 0) {
        atomicOr(err, 2);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_TMEM_COLS));
    }
}

void launch_update_tc(const DevSym &s, const Upd *upds, int nupd, int ntiles, const void *mapL, const void *mapU,
                      float *L, float *U, int split, int *err, cudaStream_t st) {
    if (ntiles <= 0) return;
    const CUtensorMap *ml = static_cast<const CUtensorMap *>(mapL);
    const CUtensorMap *mu = static_cast<const CUtensorMap *>(mapU);
    if (split)
        update_tc_kernel<1><<<ntiles, 128, TC_SMEM, st>>>(s, upds, nupd, ml, mu ? mu : ml, L, U, err);
    else
        update_tc_kernel<0><<<ntiles, 128, TC_SMEM, st>>>(s, upds, nupd, ml, mu ? mu : ml, L, U, err);
}

int configure_tc_kernels() {
    int rc = 0;
    rc |= (int)cudaFuncSetAttribute(update_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    rc |= (int)cudaFuncSetAttribute(update_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    return rc == 0 ? 0 : -1;
}

// One 2D tensor map per cblk panel (FP32, rows x columns, leading dimension ld),
// boxes of 32 x 32 with 128-byte swizzle, out-of-range elements read as zero.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_panel_maps(const std::vector<int64_t> &off, const std::vector<int> &ld, const std::vector<int> &ncols,
                      const std::vector<char> &wanted, float *arena, std::vector<CUtensorMap> &maps) {
    static EncodeTiledFn encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return -1;
        encode = reinterpret_cast<EncodeTiledFn>(fn);
    }
    const size_t n = off.size();
    maps.assign(n, CUtensorMap{});
    for (size_t k = 0; k < n; k++) {
        if (!wanted[k]) continue;
        cuuint64_t dims[2] = {(cuuint64_t)ld[k], (cuuint64_t)ncols[k]};
        cuuint64_t strides[1] = {(cuuint64_t)ld[k] * sizeof(float)};
        cuuint32_t box[2] = {32, 32};
        cuuint32_t estr[2] = {1, 1};
        CUresult r = encode(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, arena + off[k], dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return -2;
    }
    return 0;
}

}  // namespace b200
