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
// One CTA per field walks the rows (each row needs the one before); a thread
// owns 4 consecutive cells, so rows of up to 4096 cells.  The previous row
// sits in shared memory with "no value" sentinels at x = -1 and x = w; two
// barriers per row (warp totals, the next row's neighbours).
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

template <typename T>
__global__ void __launch_bounds__(1024) k_chamfer2(T* __restrict__ dist, int w, int h)
{
    using K = typename ChamferKey<T>::K;
    constexpr K kInf = ChamferKey<T>::kInf;
    constexpr int C = kChamferCells;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K* prev = reinterpret_cast<K*>(smem_raw);   // [2][w + 2], cell x at index x + 1
    K* wtot = prev + 2 * (w + 2);               // [32]
    const int x0 = threadIdx.x * C;
    if (threadIdx.x == 0) {
        prev[0] = prev[w + 1] = kInf;
        prev[w + 2] = prev[2 * (w + 2) - 1] = kInf;
    }

    K v[C], r[C];
    auto load_row = [&](int y) {
#pragma unroll
        for (int c = 0; c < C; c++) v[c] = x0 + c < w ? (K)dist[(long long)y * w + x0 + c] : kInf;
    };
    // one row: u from v and the previous row (if any), then the min-plus scan along dir
    auto row = [&](auto fwd_tag, int y, const K* pv, K* pn) {
        constexpr bool kFwd = decltype(fwd_tag)::value;
        K u[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            u[c] = v[c];
            if (pv && x0 + c < w) {
                const int i = x0 + c + 1;
                u[c] = min(u[c], min(min(pv[i - 1], pv[i + 1]) + 4, pv[i] + 3));
            }
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
            r[c] = kFwd ? min(ex, m[c]) + 3 * (K)x : min(ex, m[c]) - 3 * (K)x;
            if (x < w) {
                dist[(long long)y * w + x] = (T)r[c];
                pn[x + 1] = r[c];
            }
        }
        __syncthreads();   // the next row reads pn; the next scan rewrites wtot
    };
    using Fwd = std::true_type;
    using Bwd = std::false_type;

    __syncthreads();
    // down the rows
    int b = 0;
    load_row(0);
    row(Fwd{}, 0, (const K*)nullptr, prev + b * (w + 2));
    for (int y = 1; y < h; y++) {
        load_row(y);
        row(Fwd{}, y, prev + b * (w + 2), prev + (b ^ 1) * (w + 2));
        b ^= 1;
    }
    // back up: the last row starts from its result on the way down
#pragma unroll
    for (int c = 0; c < C; c++) v[c] = x0 + c < w ? r[c] : kInf;
    row(Bwd{}, h - 1, (const K*)nullptr, prev + (b ^ 1) * (w + 2));
    b ^= 1;
    for (int y = h - 2; y >= 0; y--) {
        load_row(y);
        row(Bwd{}, y, prev + b * (w + 2), prev + (b ^ 1) * (w + 2));
        b ^= 1;
    }
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
    ProfScope ps("chamfer_2d", st);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_chamfer2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_chamfer2<T><<<1, chamfer_threads(w), smem, st>>>(dist, w, h);
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
