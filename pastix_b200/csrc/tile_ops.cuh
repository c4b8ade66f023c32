// Warp-level operations on 32 x 32 tiles held in shared memory with the padded
// leading dimension TP (conflict-free column and row access).
#pragma once

#include <utility>

namespace b200 {

// f(std::integral_constant<int, I>) for I = 0 .. N-1, each index a compile-time
// constant: register arrays indexed by it stay in registers whatever the unroller
// decides (a loop that is not fully unrolled moves such arrays to local memory).
template <typename F, int... Is>
__device__ __forceinline__ void static_for_seq(F &&f, std::integer_sequence<int, Is...>) {
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F &&f) {
    static_for_seq(f, std::make_integer_sequence<int, N>{});
}

constexpr int TP = 33;  // padded leading dimension of 32x32 shared tiles

// Staging copy of N elements per thread: every load issued before the first store,
// so a thread waits for one memory latency instead of N (a loop that stores each
// loaded value into shared memory before the next load serialises the latencies).
template <int N, typename V, typename Load, typename Store>
__device__ __forceinline__ void stage_n(Load load, Store store) {
    V tmp[N];
#pragma unroll
    for (int u = 0; u < N; u++) tmp[u] = load(u);
#pragma unroll
    for (int u = 0; u < N; u++) store(u, tmp[u]);
}

// Inverse of the lower triangle of a pb x pb tile by one warp: lane j forms column
// j of W by forward substitution, W[m][j] = (delta_mj - sum_{p<m} T[m][p] W[p][j])
// / T[m][m] (T[m][m] = 1 if unit), with row m of T broadcast by warp shuffles and
// the reciprocals of the diagonal formed first.  trans = 1 inverts the lower
// triangle of T^T (the upper triangle of T read transposed).  Rows and columns
// >= pb of W are zero.  NB >= pb bounds the substitution (8, 16 or 32: narrow
// tiles skip the columns that are padding); T is read and W written in their first
// NB columns only (NB x TP elements each; W's rows 0..31).  Called by a whole warp.
template <typename T, int NB = 32>
__device__ void invert_lower_tile(const T *t, T *w, int pb, int lane, int unit, int trans) {
    T r[NB];  // row `lane` of the triangle to invert (lanes >= NB: padding, never read)
#pragma unroll
    for (int p = 0; p < NB; p++) r[p] = lane >= NB ? (T)0 : trans ? t[p + lane * TP] : t[lane + p * TP];
    // reciprocal of this lane's diagonal entry (the same entry, transposed or not)
    const T rd = (unit || lane >= pb) ? (T)1 : (T)1 / t[lane * (TP + 1)];
    T x[NB];
#pragma unroll
    for (int m = 0; m < NB; m++) {
        T acc = (lane == m) ? (T)1 : (T)0;
#pragma unroll
        for (int p = 0; p < m; p++) acc -= __shfl_sync(0xffffffffu, r[p], m) * x[p];
        const T rm = __shfl_sync(0xffffffffu, rd, m);
        x[m] = (m < pb && lane < pb) ? acc * rm : (T)0;
    }
    if (lane < NB) {  // W has NB columns (pitch TP), its rows >= NB zero
#pragma unroll
        for (int m = 0; m < NB; m++) w[m + lane * TP] = x[m];
#pragma unroll
        for (int m = NB; m < 32; m++) w[m + lane * TP] = (T)0;
    }
    __syncwarp();
}

}  // namespace b200
