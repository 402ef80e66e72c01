// k_chamfer.cu -- Chamfer 3-4 distance propagation (Borgefors), as the
// reference's Chamfer (DistanceOcclusionLib.cpp:916-1016) on int16 / int32
// fields, plus the integer InitDistancesFromBitMask overloads (:183-222).
//
// The reference makes one raster pass down the rows and one back up.  On the
// way down, row y first takes min(v, above-left + 4, above + 3, above-right + 4)
// per cell (fewer neighbours at the row ends), then a left-to-right pass takes
// min(v, left + 3).  The second step is a prefix min-plus scan:
//     r[x] = min over j <= x of (u[j] + 3 (x - j)) = 3x + min over j <= x of (u[j] - 3j)
// so a row is one block-wide prefix min.  Every step is a min of exact integer
// sums, so the order of evaluation cannot change the result: int16 sums are
// done in int (as the reference's promotion does) and never wrap; int32 sums
// are done in 64 bits, which equals the reference as long as its own int32
// sums do not wrap (every input at most INT32_MAX - 4).  The way up mirrors it
// (suffix min, right neighbour).
//
// A CTA walks a run of rows (each row needs the one before); a thread owns 4
// consecutive cells, so rows of up to 4096 cells.  The previous row sits in
// shared memory with "no value" sentinels at x = -1 and x = w; two barriers
// per row (warp totals, the next row's neighbours).  Fields of 64 rows or more
// run in blocks of 32 rows, all blocks at once (see below); smaller ones, or
// when the small boundary scratch cannot be had, in one CTA.
#include <type_traits>

#include "common.cuh"
#include "kernels.h"

namespace dolk {

constexpr int kChamferCells = 4;

template <typename T>
struct ChamferKey {
    using K = int;
    static constexpr int kInf = 1 << 29;
};
template <>
struct ChamferKey<int32_t> {
    using K = long long;
    static constexpr long long kInf = 1LL << 62;
};

template <typename K>
__device__ __forceinline__ K shfl_up_k(K v, int o)
{
    return __shfl_up_sync(0xFFFFFFFFu, v, o);
}
template <typename K>
__device__ __forceinline__ K shfl_down_k(K v, int o)
{
    return __shfl_down_sync(0xFFFFFFFFu, v, o);
}

// Block-wide scan of the per-thread totals: for kFwd the min over all earlier
// threads (exclusive prefix), else the min over all later threads (exclusive
// suffix).  wtot: one slot per warp; one barrier.
template <typename K, bool kFwd>
__device__ __forceinline__ K block_excl_min(K tot, K* wtot, K inf)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    K incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const K v = kFwd ? shfl_up_k(incl, o) : shfl_down_k(incl, o);
        if (kFwd ? lane >= o : lane + o < 32) incl = min(incl, v);
    }
    K excl = kFwd ? shfl_up_k(incl, 1) : shfl_down_k(incl, 1);
    if (kFwd ? lane == 0 : lane == 31) excl = inf;
    if (kFwd ? lane == 31 : lane == 0) wtot[wid] = incl;
    __syncthreads();
    // every warp scans the (at most 32) warp totals for itself
    K wv = lane < nw ? wtot[lane] : inf;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const K v = kFwd ? shfl_up_k(wv, o) : shfl_down_k(wv, o);
        if (kFwd ? lane >= o : lane + o < 32) wv = min(wv, v);
    }
    K wex = kFwd ? shfl_up_k(wv, 1) : shfl_down_k(wv, 1);
    if (kFwd ? lane == 0 : lane == 31) wex = inf;
    const K mine = __shfl_sync(0xFFFFFFFFu, wex, wid);
    return min(excl, mine);
}

// Rows ya, ya + dir, ..., yb of one pass (dir = +1 down, -1 up), the first of
// them with no row before it; one CTA, a thread per 4 consecutive cells.
template <typename T, bool kFwd>
__device__ __forceinline__ void chamfer_rows(T* __restrict__ dist, int w, int ya, int yb, unsigned char* smem_raw)
{
    using K = typename ChamferKey<T>::K;
    constexpr K kInf = ChamferKey<T>::kInf;
    constexpr int C = kChamferCells;
    K* prev = reinterpret_cast<K*>(smem_raw);   // [2][w + 2], cell x at index x + 1
    K* wtot = prev + 2 * (w + 2);               // [32]
    const int x0 = threadIdx.x * C;
    if (threadIdx.x == 0) {
        prev[0] = prev[w + 1] = kInf;
        prev[w + 2] = prev[2 * (w + 2) - 1] = kInf;
    }
    __syncthreads();
    int b = 0;
    const int dir = kFwd ? 1 : -1;
    for (int y = ya;; y += dir) {
        const K* pv = y == ya ? nullptr : prev + b * (w + 2);
        K* pn = prev + (b ^ 1) * (w + 2);
        K u[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const int x = x0 + c;
            u[c] = x < w ? (K)dist[(long long)y * w + x] : kInf;
            if (pv && x < w) u[c] = min(u[c], min(min(pv[x], pv[x + 2]) + 4, pv[x + 1] + 3));
        }
        K m[C];
        if (kFwd) {
#pragma unroll
            for (int c = 0; c < C; c++) {
                const K key = x0 + c < w ? u[c] - 3 * (K)(x0 + c) : kInf;
                m[c] = c ? min(m[c - 1], key) : key;
            }
        } else {
#pragma unroll
            for (int c = C - 1; c >= 0; c--) {
                const K key = x0 + c < w ? u[c] + 3 * (K)(x0 + c) : kInf;
                m[c] = c < C - 1 ? min(m[c + 1], key) : key;
            }
        }
        const K ex = block_excl_min<K, kFwd>(kFwd ? m[C - 1] : m[0], wtot, kInf);
#pragma unroll
        for (int c = 0; c < C; c++) {
            const int x = x0 + c;
            const K r = kFwd ? min(ex, m[c]) + 3 * (K)x : min(ex, m[c]) - 3 * (K)x;
            if (x < w) {
                dist[(long long)y * w + x] = (T)r;
                pn[x + 1] = r;
            }
        }
        __syncthreads();   // the next row reads pn; the next scan rewrites wtot
        b ^= 1;
        if (y == yb) break;
    }
}

// the whole field in one CTA: down the rows, then back up
template <typename T>
__global__ void __launch_bounds__(1024) k_chamfer2(T* __restrict__ dist, int w, int h)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    chamfer_rows<T, true>(dist, w, 0, h - 1, smem_raw);
    chamfer_rows<T, false>(dist, w, h - 1, 0, smem_raw);
}

// ---- the same passes over blocks of R rows ----
// A pass only takes mins of sums of exact integers, so it is min-plus linear:
// a block's result is the min of (a) the block run with nothing before its
// first row and (b) the boundary row before it carried through the block with
// every cell of the block "no value".  (b) has a closed form: a cell r rows
// past the boundary row gets min over j of T[j] + c(x - j, r), c the cheapest
// path of the pass's steps (3 straight, 4 diagonal, along the row only in the
// scan direction): c = 3 max(|dx|, r) + min(|dx|, r) where the path can reach,
// i.e. |dx| <= r, or any dx on the side the row scan moves towards.  So:
//   1. every block runs with nothing before it (parallel over blocks);
//   2. one CTA walks the blocks: a block's true last row is the min of its
//      row from step 1 and the previous true last row carried R rows;
//   3. every row of every block takes the min with the previous block's true
//      last row carried to it (parallel over rows).
constexpr int kChamferBlockRows = 32;

template <typename T, bool kFwd>
__global__ void __launch_bounds__(1024) k_chamfer_blocks(T* __restrict__ dist, int w, int h, int R)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int y0 = blockIdx.x * R, y1 = min(h, y0 + R);
    if (kFwd)
        chamfer_rows<T, true>(dist, w, y0, y1 - 1, smem_raw);
    else
        chamfer_rows<T, false>(dist, w, y1 - 1, y0, smem_raw);
}

// The boundary row bt carried r rows into the next block, at cell x: the window
// |x - j| <= r (cost 3r + |x - j|) and the far side the scan moves from (pre:
// prefix min of bt[j] - 3j going down, suffix min of bt[j] + 3j going up).
template <typename K, bool kFwd>
__device__ __forceinline__ K carried(const K* bt, const K* pre, int w, int x, int r, K inf)
{
    K best = inf;
    const int ja = max(0, x - r), jb = min(w - 1, x + r);
    for (int j = ja; j <= jb; j++) best = min(best, bt[j] + 3 * (K)r + (K)abs(x - j));
    if (kFwd) {
        if (x - r - 1 >= 0) best = min(best, pre[x - r - 1] + 3 * (K)x + (K)r);
    } else {
        if (x + r + 1 < w) best = min(best, pre[x + r + 1] - 3 * (K)x + (K)r);
    }
    return best;
}

// Step 2: one CTA walks the blocks in scan order and keeps each true boundary
// row (bt[blk]) with its prefix / suffix minima (pre[blk]) for step 3.
template <typename T, bool kFwd>
__global__ void __launch_bounds__(1024) k_chamfer_chain(T* __restrict__ dist, int w, int h, int R,
                                                        typename ChamferKey<T>::K* __restrict__ bt,
                                                        typename ChamferKey<T>::K* __restrict__ pre)
{
    using K = typename ChamferKey<T>::K;
    constexpr K kInf = ChamferKey<T>::kInf;
    constexpr int C = kChamferCells;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K* cur = reinterpret_cast<K*>(smem_raw);   // [w] boundary row
    K* cpre = cur + w;                          // [w] its prefix / suffix minima
    K* wtot = cpre + w;                         // [32]
    const int nb = (h + R - 1) / R;
    const int x0 = threadIdx.x * C;
    for (int s = 0; s < nb - 1; s++) {
        const int blk = kFwd ? s : nb - 1 - s;          // the block whose boundary row this is
        const int yb = kFwd ? min(h, (blk + 1) * R) - 1 : blk * R;   // its last row in scan order
        K v[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const int x = x0 + c;
            v[c] = x < w ? (K)dist[(long long)yb * w + x] : kInf;
            if (s > 0 && x < w) {
                const int rows = kFwd ? yb - (blk * R - 1) : (blk + 1) * R - yb;
                v[c] = min(v[c], carried<K, kFwd>(cur, cpre, w, x, rows, kInf));
            }
        }
        __syncthreads();   // every thread has read the previous boundary row
        K m[C];
        if (kFwd) {
#pragma unroll
            for (int c = 0; c < C; c++) {
                const K key = x0 + c < w ? v[c] - 3 * (K)(x0 + c) : kInf;
                m[c] = c ? min(m[c - 1], key) : key;
            }
        } else {
#pragma unroll
            for (int c = C - 1; c >= 0; c--) {
                const K key = x0 + c < w ? v[c] + 3 * (K)(x0 + c) : kInf;
                m[c] = c < C - 1 ? min(m[c + 1], key) : key;
            }
        }
        const K ex = block_excl_min<K, kFwd>(kFwd ? m[C - 1] : m[0], wtot, kInf);
#pragma unroll
        for (int c = 0; c < C; c++) {
            const int x = x0 + c;
            if (x < w) {
                const K pm = min(ex, m[c]);
                cur[x] = v[c];
                cpre[x] = pm;
                bt[(long long)blk * w + x] = v[c];
                pre[(long long)blk * w + x] = pm;
            }
        }
        __syncthreads();
    }
}

// Step 3: every row of a block after the first in scan order takes the min with
// the previous block's true boundary row carried to it.
template <typename T, bool kFwd>
__global__ void __launch_bounds__(256) k_chamfer_apply(T* __restrict__ dist, int w, int h, int R,
                                                       const typename ChamferKey<T>::K* __restrict__ bt,
                                                       const typename ChamferKey<T>::K* __restrict__ pre)
{
    using K = typename ChamferKey<T>::K;
    constexpr K kInf = ChamferKey<T>::kInf;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int blk = y / R, nb = (h + R - 1) / R;
    if (x >= w || (kFwd ? blk == 0 : blk == nb - 1)) return;
    const int src = kFwd ? blk - 1 : blk + 1;
    const int rows = kFwd ? y - (blk * R - 1) : (blk + 1) * R - y;
    const K c = carried<K, kFwd>(bt + (long long)src * w, pre + (long long)src * w, w, x, rows, kInf);
    T* p = dist + (long long)y * w + x;
    if (c < (K)*p) *p = (T)c;
}

template <typename T>
__global__ void __launch_bounds__(256) k_init_distances_int(const uint32_t* __restrict__ mask, T* __restrict__ dist,
                                                            int w, long long rows, T max_d)
{
    const int ws = words_per_row(w);
    const long long n = rows * w;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long y = i / w;
        const int x = (int)(i - y * w);
        dist[i] = ((__ldg(mask + y * ws + (x >> 5)) >> (x & 31)) & 1u) ? (T)0 : max_d;
    }
}

int chamfer_threads(int w)
{
    const int t = (w + kChamferCells - 1) / kChamferCells;
    return ((t + 31) / 32) * 32;
}

template <typename T>
void launch_chamfer_2d(T* dist, int w, int h, cudaStream_t st)
{
    using K = typename ChamferKey<T>::K;
    const size_t smem = (2 * (size_t)(w + 2) + 32) * sizeof(K);
    const int threads = chamfer_threads(w);
    ProfScope ps("chamfer_2d", st);
    const int R = kChamferBlockRows, nb = (h + R - 1) / R;
    void* scratch = nullptr;
    const size_t sb = 2 * (size_t)nb * w * sizeof(K);
    if (nb >= 2 && h <= 65535 && cudaMallocAsync(&scratch, sb, st) == cudaSuccess) {
        K* bt = static_cast<K*>(scratch);
        K* pre = bt + (size_t)nb * w;
        const size_t csmem = (2 * (size_t)w + 32) * sizeof(K);
        auto set = [](const void* f, size_t b) {
            if (b > 48 * 1024) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
        };
        set((const void*)k_chamfer_blocks<T, true>, smem);
        set((const void*)k_chamfer_blocks<T, false>, smem);
        set((const void*)k_chamfer_chain<T, true>, csmem);
        set((const void*)k_chamfer_chain<T, false>, csmem);
        const dim3 ag((w + 255) / 256, h);
        k_chamfer_blocks<T, true><<<nb, threads, smem, st>>>(dist, w, h, R);
        k_chamfer_chain<T, true><<<1, threads, csmem, st>>>(dist, w, h, R, bt, pre);
        k_chamfer_apply<T, true><<<ag, 256, 0, st>>>(dist, w, h, R, bt, pre);
        k_chamfer_blocks<T, false><<<nb, threads, smem, st>>>(dist, w, h, R);
        k_chamfer_chain<T, false><<<1, threads, csmem, st>>>(dist, w, h, R, bt, pre);
        k_chamfer_apply<T, false><<<ag, 256, 0, st>>>(dist, w, h, R, bt, pre);
        cudaFreeAsync(scratch, st);
        return;
    }
    cudaGetLastError();   // a failed scratch allocation: walk the whole field in one CTA
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_chamfer2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_chamfer2<T><<<1, threads, smem, st>>>(dist, w, h);
}

template <typename T>
void launch_init_distances_int(const uint32_t* mask, T* dist, int w, long long rows, T max_d, cudaStream_t st)
{
    long long n = rows * w;
    long long blocks = (n + 255) / 256;
    long long cap = (long long)g_num_sms * 32;
    k_init_distances_int<T><<<(int)(blocks < cap ? blocks : cap), 256, 0, st>>>(mask, dist, w, rows, max_d);
}

template void launch_chamfer_2d<int16_t>(int16_t*, int, int, cudaStream_t);
template void launch_chamfer_2d<int32_t>(int32_t*, int, int, cudaStream_t);
template void launch_init_distances_int<int16_t>(const uint32_t*, int16_t*, int, long long, int16_t, cudaStream_t);
template void launch_init_distances_int<int32_t>(const uint32_t*, int32_t*, int, long long, int32_t, cudaStream_t);

}  // namespace dolk
