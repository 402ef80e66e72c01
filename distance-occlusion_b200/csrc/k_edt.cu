// k_edt.cu -- exact Euclidean distance transform driven by a bitmask.
//
// The reference's Felzenszwalb transform (DistanceOcclusionLib.cpp:1026-1085,
// driven by DistanceOcclusionTool.cpp:741-782) starts from 0 / FLT_MAX, so every
// intermediate value is an integer squared distance below 2^24 and the float
// envelope returns the exact squared EDT (FLT_MAX where no set cell exists);
// any exact EDT gives identical floats.  This file computes it in integers,
// separably, as three (2D: two) passes over the field:
//
//   x pass  from the mask bits: per cell, the distance along its row to the
//           nearest cell of the opposite state, with the cell's own state in
//           bit 15 (uint16).  One warp per row, word-level bit scans.
//   y pass  per column: e(y) = min over y' of (y-y')^2 + f(y'), where f(y') is 0
//           for cells of the opposite state and v(y')^2 otherwise.  The search
//           walks outwards from y and stops once k^2 >= the best so far, which
//           is exact because f >= 0.  Whole columns of 16 adjacent x are
//           staged in shared memory by TMA.
//   z pass  the same along z on the y-pass output (uint32, state in bit 31),
//           which a volume of width 8k stores as [y][x/8][z][8] so that each
//           8-column z line is one contiguous tile.
//
// Keeping "distance to the opposite state" per cell serves both forms at once:
// for an empty cell it is the distance to the nearest set cell (the unsigned
// EDT), for a set cell the distance to the nearest empty cell, so the signed
// field (distance to set cells minus distance to empty cells) needs no second
// transform.
#include <float.h>

#include "common.cuh"
#include "hull.cuh"
#include "kernels.h"
#include "tma.cuh"

#ifndef DOL_EDT_SQUARED
#define DOL_EDT_SQUARED 0
#define DOL_EDT_DIST 1
#define DOL_EDT_SIGNED 2
#endif

namespace dolk {

constexpr uint32_t kInf16 = 0x7FFFu;        // "no opposite cell in this row"
constexpr uint32_t kInf32 = 0x7FFFFFFFu;    // "no opposite cell in this plane"
constexpr int kMaxChunks = 32;              // rows up to 32*32*32 = 32768 cells

// ---------------------------------------------------------------- x pass ----
// A row is split over the lanes of a warp segment, one mask word (32 cells) per
// lane: rows of up to 16 words share a warp (segments of 1..16 lanes), longer
// rows take the whole warp and loop over 32-word chunks.  Segment scans give
// each word the nearest clear / set cell before and after it (longer rows: a
// right-to-left pre-pass over the chunks gives the carries from the right).
// Inside the word a lane walks its 32 cells twice: forwards, the nearest
// cell of the other state on the left is the cell before the current run
// (runs change where m ^ (m << 1) has a bit), backwards the cell after it.
// The 32 results go out as four 16-byte stores.
__device__ __forceinline__ int pow2_at_least(int v)
{
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Cells H0 .. H0+15 of a word (me: states, cells past w continuing the last
// live run; tl / tr: run starts / ends; xb: the word's first cell).  runA is
// the nearest other-state cell left of cell H0's run; runB comes in as the one
// right of cell H0+15's run and leaves as the one right of cell H0's.  Each
// cell's value (distance to the nearer, at most kInf16, state in bit 15)
// goes out two per word.
template <int H0>
__device__ __forceinline__ void x_half(uint32_t me, uint32_t tl, uint32_t tr, int xb, int runA, int& runB,
                                       uint32_t packed[8])
{
    int dl[16];
#pragma unroll
    for (int u = 0; u < 16; u++) {
        const int t = H0 + u;
        if (t > 0 && ((tl >> t) & 1u)) runA = xb + t - 1;
        dl[u] = xb + t - runA;
    }
#pragma unroll
    for (int u = 15; u >= 0; u--) {
        const int t = H0 + u;
        if (t < 31 && ((tr >> t) & 1u)) runB = xb + t + 1;
        const int d = min(min(dl[u], runB - xb - t), (int)kInf16);
        const uint32_t v = (uint32_t)d | (((me >> t) & 1u) << 15);
        if (u & 1)
            packed[u >> 1] = v << 16;   // the odd cell comes first going down
        else
            packed[u >> 1] |= v;
    }
}

// 16 cells' packed values to o: two 16-byte stores, or per cell for the first
// `n` cells when the row end or alignment does not allow them
__device__ __forceinline__ void store_half(uint16_t* o, const uint32_t pk[8], bool whole, int n)
{
    if (whole) {
        uint4* o4 = reinterpret_cast<uint4*>(o);
        o4[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        o4[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    } else {
#pragma unroll
        for (int t = 0; t < 16; t++)
            if (t < n) o[t] = (uint16_t)(pk[t >> 1] >> (16 * (t & 1)));
    }
}

__global__ void __launch_bounds__(256) k_edt_x(const uint32_t* __restrict__ mask, uint16_t* __restrict__ out, int w,
                                               long long rows)
{
    __shared__ int right_carry[8][kMaxChunks][2];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int ws = words_per_row(w);
    const int SW = ws >= 32 ? 32 : pow2_at_least(ws);   // lanes per row
    const int seg = lane / SW, sl = lane % SW, rpw = 32 / SW;
    const int nchunks = (ws + 31) >> 5;
    const int NEG = -(1 << 30), POS = 1 << 30;
    const bool vec_ok = (w & 7) == 0;   // 16-byte aligned word outputs
    long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;

    for (long long row0 = warp * rpw; row0 < rows; row0 += nwarps * rpw) {
        const long long row = row0 + seg;
        const bool rowok = row < rows;
        const uint32_t* mrow = mask + (rowok ? row : 0) * ws;
        uint16_t* orow = out + (rowok ? row : 0) * (long long)w;

        // long rows: first clear / set cell right of each chunk (segments are whole warps here)
        if (nchunks > 1) {
            int carry0 = POS, carry1 = POS;
            for (int c = nchunks - 1; c >= 0; c--) {
                right_carry[wib][c][0] = carry0;
                right_carry[wib][c][1] = carry1;
                if (c == 0) break;
                const int k = 32 * c + lane;
                int f0 = POS, f1 = POS;
                if (k < ws) {
                    const uint32_t live = live_bits(w, k), m = mrow[k];
                    const uint32_t z0 = ~m & live, z1 = m & live;
                    if (z0) f0 = 32 * k + __ffs(z0) - 1;
                    if (z1) f1 = 32 * k + __ffs(z1) - 1;
                }
                for (int o = 16; o > 0; o >>= 1) {
                    f0 = min(f0, __shfl_xor_sync(0xFFFFFFFFu, f0, o));
                    f1 = min(f1, __shfl_xor_sync(0xFFFFFFFFu, f1, o));
                }
                carry0 = min(carry0, f0);
                carry1 = min(carry1, f1);
            }
            __syncwarp();
        }

        int left0 = NEG, left1 = NEG;   // last clear / set cell left of the chunk
        for (int c = 0; c < nchunks; c++) {
            const int k = 32 * c + sl;
            const bool on = rowok && sl < SW && k < ws && (nchunks > 1 || sl < ws);
            uint32_t m = 0, live = 0;
            int l0 = NEG, l1 = NEG, f0 = POS, f1 = POS;
            if (on) {
                m = mrow[k];
                live = live_bits(w, k);
                const uint32_t z0 = ~m & live, z1 = m & live;
                if (z0) { l0 = 32 * k + 31 - __clz(z0); f0 = 32 * k + __ffs(z0) - 1; }
                if (z1) { l1 = 32 * k + 31 - __clz(z1); f1 = 32 * k + __ffs(z1) - 1; }
            }
            // segment-exclusive prefix max of last positions, suffix min of first positions
            int p0 = l0, p1 = l1, s0 = f0, s1 = f1;
            for (int o = 1; o < SW; o <<= 1) {
                const int a0 = __shfl_up_sync(0xFFFFFFFFu, p0, o, SW), a1 = __shfl_up_sync(0xFFFFFFFFu, p1, o, SW);
                const int b0 = __shfl_down_sync(0xFFFFFFFFu, s0, o, SW), b1 = __shfl_down_sync(0xFFFFFFFFu, s1, o, SW);
                if (sl >= o) { p0 = max(p0, a0); p1 = max(p1, a1); }
                if (sl + o < SW) { s0 = min(s0, b0); s1 = min(s1, b1); }
            }
            int L0 = __shfl_up_sync(0xFFFFFFFFu, p0, 1, SW), L1 = __shfl_up_sync(0xFFFFFFFFu, p1, 1, SW);
            int R0 = __shfl_down_sync(0xFFFFFFFFu, s0, 1, SW), R1 = __shfl_down_sync(0xFFFFFFFFu, s1, 1, SW);
            if (sl == 0) { L0 = NEG; L1 = NEG; }
            if (sl == SW - 1) { R0 = POS; R1 = POS; }
            L0 = max(L0, left0); L1 = max(L1, left1);
            if (nchunks > 1) { R0 = min(R0, right_carry[wib][c][0]); R1 = min(R1, right_carry[wib][c][1]); }
            left0 = max(left0, __shfl_sync(0xFFFFFFFFu, p0, SW - 1, SW));
            left1 = max(left1, __shfl_sync(0xFFFFFFFFu, p1, SW - 1, SW));
            if (!on) continue;

            // cells past w continue the last live cell's run (no spurious run ends)
            const int nlive = min(32, w - 32 * k);
            const uint32_t lastbit = (m >> (nlive - 1)) & 1u;
            const uint32_t me = (m & live) | (lastbit ? ~live : 0u);
            const uint32_t tl = me ^ (me << 1);   // bit t: cell t starts a run (t >= 1)
            const uint32_t tr = me ^ (me >> 1);   // bit t: cell t ends a run (t <= 30)
            const int xb = 32 * k;
            // the word in two halves of 16 cells (half the registers of a
            // whole-word walk): first cells 16..31, whose walk back from the
            // right carry leaves the value the lower half starts from
            const int carry_l = (me & 1u) ? L0 : L1;   // nearest other-state cell left of cell 0's run
            const uint32_t st = tl & 0xFFFEu;          // run starts among cells 1..15
            int runB = (me >> 31) ? R0 : R1;           // nearest other-state cell right of cell 31's run
            uint32_t pk[8];
            uint16_t* o = orow + xb;
            const bool whole = vec_ok && nlive == 32;
            x_half<16>(me, tl, tr, xb, st ? xb + (30 - __clz(st)) : carry_l, runB, pk);
            store_half(o + 16, pk, whole, nlive - 16);
            x_half<0>(me, tl, tr, xb, carry_l, runB, pk);
            store_half(o, pk, whole, nlive);
        }
    }
}

// ------------------------------------------------------------ line passes ----
// A line runs along y (stride w) or z (stride w*h).  Each CTA owns 32 adjacent
// x of one "outer" index and the whole line.  TIn is uint16 (x-pass output)
// or uint32 (y-pass output).  kFinal writes the float field in the requested
// form; otherwise uint32 (state << 31) | squared distance.

template <typename TIn>
__device__ __forceinline__ void decode_in(TIn v, uint32_t* state, uint32_t* f)
{
    if (sizeof(TIn) == 2) {
        uint32_t u = (uint32_t)v;
        *state = u >> 15;
        uint32_t d = u & 0x7FFFu;
        *f = d == kInf16 ? 0xFFFFFFFFu : d * d;
    } else {
        uint32_t u = (uint32_t)v;
        *state = u >> 31;
        uint32_t e = u & 0x7FFFFFFFu;
        *f = e == kInf32 ? 0xFFFFFFFFu : e;
    }
}

// sqrtf of the integers 0 .. kSqrtTab - 1 as float bit patterns, built at
// compile time from an exact integer square root rounded to nearest (no tie
// is possible: (2m + 1)^2 is odd).  IEEE 754 square root is correctly
// rounded, so these are the values sqrtf returns; the distances of most cells
// are below 64, and one cached load replaces the square root there.
constexpr int kSqrtTab = 4096;

constexpr uint64_t isqrt64(uint64_t n)
{
    uint64_t r = 0, bit = 1ull << 62;
    while (bit > n) bit >>= 2;
    while (bit) {
        if (n >= r + bit) {
            n -= r + bit;
            r = (r >> 1) + bit;
        } else {
            r >>= 1;
        }
        bit >>= 2;
    }
    return r;   // floor(sqrt(n))
}

constexpr uint32_t sqrt_bits(uint32_t i)
{
    if (i == 0) return 0u;
    int k = 0;   // i * 4^k in [2^46, 2^48): its square root has 24 bits
    uint64_t v = i;
    while (v < (1ull << 46)) {
        v <<= 2;
        k++;
    }
    uint64_t m = isqrt64(v);
    if (4 * v > (2 * m + 1) * (2 * m + 1)) m++;   // round to nearest
    int e = 127 + 23 - k;
    if (m == (1ull << 24)) {
        m >>= 1;
        e++;
    }
    return ((uint32_t)e << 23) | (uint32_t)(m - (1ull << 23));
}
static_assert(sqrt_bits(4) == 0x40000000u && sqrt_bits(2) == 0x3FB504F3u && sqrt_bits(4095) == 0x427FF800u,
              "square-root table");

struct SqrtTable {
    uint32_t v[kSqrtTab];
};
constexpr SqrtTable make_sqrt_table()
{
    SqrtTable t{};
    for (int i = 0; i < kSqrtTab; i++) t.v[i] = sqrt_bits((uint32_t)i);
    return t;
}
static __device__ const SqrtTable g_sqrt_table = make_sqrt_table();

// sqrtf((float)e) for an integer squared distance e
__device__ __forceinline__ float sqrt_of_int(uint32_t e)
{
    return e < (uint32_t)kSqrtTab ? __uint_as_float(__ldg(&g_sqrt_table.v[e])) : sqrtf((float)e);
}

__device__ __forceinline__ float final_value(uint32_t state, uint32_t best, int form)
{
    // best == 0xFFFFFFFF: no cell of the other state anywhere on the lines searched
    if (form == DOL_EDT_SIGNED) {
        const float r = best == 0xFFFFFFFFu ? sqrtf(FLT_MAX) : sqrt_of_int(best);
        return state ? -r : r;
    }
    if (state) return 0.0f;   // unsigned forms: set cells are at distance 0
    if (best == 0xFFFFFFFFu) return form == DOL_EDT_DIST ? sqrtf(FLT_MAX) : FLT_MAX;
    return form == DOL_EDT_DIST ? sqrt_of_int(best) : (float)best;
}

// min over the line of (q-q')^2 + f(q') for the cell at q, walking outwards
// until k^2 reaches the best value found (f >= 0 makes that exact)
template <typename TIn, class At>
__device__ __forceinline__ uint32_t search_line(const At& at, int q, int n, uint32_t* state)
{
    uint32_t s, best;
    decode_in<TIn>(at(q), &s, &best);
    const int reach = max(q, n - 1 - q);
    for (int k = 1; k <= reach; k++) {
        const uint32_t k2 = (uint32_t)k * (uint32_t)k;
        if (k2 >= best) break;
        if (q - k >= 0) {
            uint32_t s2, f;
            decode_in<TIn>(at(q - k), &s2, &f);
            best = min(best, s2 != s ? k2 : (f == 0xFFFFFFFFu ? f : f + k2));
        }
        if (q + k < n) {
            uint32_t s2, f;
            decode_in<TIn>(at(q + k), &s2, &f);
            best = min(best, s2 != s ? k2 : (f == 0xFFFFFFFFu ? f : f + k2));
        }
    }
    *state = s;
    return best;
}

template <bool kFinal>
__device__ __forceinline__ void put_line_value(void* out, long long o, uint32_t s, uint32_t best, int form)
{
    if (kFinal) {
        static_cast<float*>(out)[o] = final_value(s, best, form);
    } else {
        uint32_t e = best == 0xFFFFFFFFu ? kInf32 : best;
        static_cast<uint32_t*>(out)[o] = e | (s << 31);
    }
}

// A walked cell's result: `none` -- no cell of the other state on the lines
// searched -- as kInf32 (uint32 field) or the float form's "no cell" value
template <bool kFinal>
__device__ __forceinline__ void put_walk_value(void* out, long long o, uint32_t s, uint32_t best, bool none, int form)
{
    if (kFinal) {
        float v;
        if (form == DOL_EDT_SIGNED) {
            const float r = none ? sqrtf(FLT_MAX) : sqrt_of_int(best);
            v = s ? -r : r;
        } else if (s) {
            v = 0.0f;   // unsigned forms: set cells are at distance 0
        } else if (form == DOL_EDT_DIST) {
            v = none ? sqrtf(FLT_MAX) : sqrt_of_int(best);
        } else {
            v = none ? FLT_MAX : (float)best;
        }
        static_cast<float*>(out)[o] = v;
    } else {
        static_cast<uint32_t*>(out)[o] = (none ? kInf32 : best) | (s << 31);
    }
}

// Plain-load form: 32 adjacent x per CTA, the line staged in shared memory when
// it fits (kStaged) or read from global memory otherwise.
template <typename TIn, bool kFinal, bool kStaged>
__global__ void __launch_bounds__(256) k_edt_line(const TIn* __restrict__ in, void* __restrict__ out, int w, int n,
                                                  long long stride, long long outer_stride, int form, int outer0)
{
    extern __shared__ unsigned char smem_raw[];
    TIn* tile = reinterpret_cast<TIn*>(smem_raw);   // [n][32]
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int x = blockIdx.x * 32 + lane;
    const long long base = (long long)(blockIdx.y + outer0) * outer_stride + x;
    const bool live = x < w;

    if (kStaged) {
        for (int q = wib; q < n; q += nw) tile[q * 32 + lane] = live ? in[base + q * stride] : (TIn)0;
        __syncthreads();
    }
    auto at = [&](int q) -> TIn { return kStaged ? tile[q * 32 + lane] : in[base + q * stride]; };
    for (int q = wib; q < n; q += nw) {
        if (!live) continue;
        uint32_t s;
        uint32_t best = search_line<TIn>(at, q, n, &s);
        put_line_value<kFinal>(out, base + q * stride, s, best, form);
    }
}

// TMA form.  A TX-column x full-line tile arrives in 256-position boxes
// (cp.async.bulk.tensor, one mbarrier).  It is then split in place, 16 bytes
// at a time, into two state-specific arrays: F_s[p] is the cell's value (v or
// e) when its state is s and 0 otherwise, so for a cell of state s every probe
// is one load and one multiply-add plus a share of a three-way min (uint16
// distances) or one fused add-min (uint32 squared distances) -- a cell of the
// other state at distance k contributes exactly k^2.  Each array carries
// kPadRows rows of "no cell" sentinels before and after the line (positions
// n .. rows-1 too), so the walk outwards from a cell runs on both sides with
// one test per two distances until it either ends or passes the nearer line
// end by the margin the sentinels allow; only then does it continue on the
// far side alone.  Each lane walks two cells of its column, 4 positions
// apart, in one loop; a warp covers 8 columns x 8 positions.
//
// Layouts (kMode): 0 reads and writes [z][y][x]; 1 (y pass of a volume) writes
// its uint32 output as [y][x/8][z][8], so that 2 (the z pass) reads every
// 8-column z line as one contiguous 32-byte-row tile.
constexpr int kPadRows = 32;

// sq_val(v) + k2: one multiply-add for the u16 (distance) form
template <typename TIn>
__device__ __forceinline__ uint32_t add_sq(TIn v, uint32_t k2)
{
    return sizeof(TIn) == 2 ? (uint32_t)v * (uint32_t)v + k2 : (uint32_t)v + k2;
}

// The rest of a walk on the far side of cell q once the near side is done:
// distances k.. with k2 = k^2, pl / pr at q - k / q + k; ends at the line end
// or when k^2 reaches the best value.
template <typename TIn, int TX>
__device__ __forceinline__ uint32_t far_side(uint32_t best, int q, int n, int k, uint32_t k2, const TIn* pl,
                                             const TIn* pr)
{
    if (q <= n - 1 - q) {
        for (; k <= n - 1 - q && k2 < best; k++) {
            best = min(best, add_sq<TIn>(*pr, k2));
            pr += TX;
            k2 += 2 * k + 1;
        }
    } else {
        for (; k <= q && k2 < best; k++) {
            best = min(best, add_sq<TIn>(*pl, k2));
            pl -= TX;
            k2 += 2 * k + 1;
        }
    }
    return best;
}

// Blocks of the pruned search (uint32 tiles): kPruneB cells, their minima kept
// per (state, column)
constexpr int kPruneB = 16;
// a uint32 tile takes the pruned search when far_pct percent of its sampled
// cells lie at least kFarDist cells from the other state in their plane (1024^3
// z passes: 2000 random points, ~90 % of the cells, 14.2 -> 11.7 ms; 20000
// points, ~37 %, stay on the windowed search, 8.2 against 9.5 ms pruned)
constexpr uint32_t kFarDist = 128;

// the two split line arrays with their sentinel rows, then the envelope
// path's hull words (two per column per 32-cell segment), then (uint32
// tiles) the pruned search's block minima (two per column per block)
template <typename TIn, int TX>
static size_t tma_tile_bytes(int n)
{
    constexpr int SB = 32;
    return 2 * (size_t)(((n + 255) / 256) * 256 + 2 * kPadRows) * TX * sizeof(TIn) +
           2 * (size_t)TX * ((n + SB - 1) / SB) * sizeof(uint32_t) +
           (sizeof(TIn) == 4 ? 2 * (size_t)TX * ((n + kPruneB - 1) / kPruneB) * sizeof(uint32_t) : 0);
}

// One 32-bit word of a staged tile split by state: its cells (two uint16 or
// one uint32, the state in each cell's top bit) go to *f0 when clear, *f1
// when set, 0 in the other; vmask holds every cell's value bits.
template <typename TIn>
__device__ __forceinline__ void split_word(uint32_t x, uint32_t vmask, uint32_t* f0, uint32_t* f1)
{
    const uint32_t v = x & vmask;
    const uint32_t st = x & ~vmask;                                                 // the state bits
    const uint32_t m = sizeof(TIn) == 2 ? (st >> 15) * 0xFFFFu : 0u - (st >> 31);   // all of a set cell's bits
    *f0 = v & ~m;
    *f1 = v & m;
}

// Envelope path (hull.cuh): the windowed search costs a cell about sqrt(its
// own value) probes, and a cell with no cell of the other state on its row
// (or plane) walks to the line end, so sparse or nearly empty volumes make it
// O(n) per cell.  Tiles holding such values take the lower-envelope path,
// O(n) per line whatever the data.

// The envelope path of one staged tile (hull.cuh), out of line so that the
// windowed search's code is laid out and register-allocated as if it were
// alone in the kernel (inlined, the dense tiles' passes measured 1-3 % slower).
template <typename TIn, bool kFinal, int TX, int kMode>
__device__ __noinline__ void edt_tile_envelope(const TIn* F0, TIn* F1, int rows, int n, int w, int x0, int outer,
                                               void* out, long long stride, long long outer_stride, int form)
{
    // envelope path: units (column, 32-cell segment); hull words after the tile
    // cells per segment (16-cell segments, which keep every thread of an
    // 8-column tile busy, measured slower: more words to scan and merge)
    constexpr int SB = 32;
    const int nseg = (n + SB - 1) / SB;
    uint32_t* HM = reinterpret_cast<uint32_t*>(F1 + (rows + 2 * kPadRows) * TX - kPadRows * TX);
    const int units = TX * nseg;
    for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int col = u % TX, seg = u / TX;
        if (x0 + col < w) hull_build<TIn, SB>(F0, F1, HM, TX, nseg, n, col, seg);
    }
    __syncthreads();
    for (int half = 1; half < nseg; half <<= 1) {
        const int groups = (nseg + 2 * half - 1) / (2 * half);
        for (int j = threadIdx.x; j < 2 * TX * groups; j += blockDim.x) {
            const int g = j % groups, sc = j / groups;   // sc = s * TX + col
            const int col = sc % TX, s = sc / TX;
            const int lo = g * 2 * half, mid = lo + half, hi = min(mid + half, nseg);
            if (mid < nseg && x0 + col < w)
                hull_merge<TIn, SB>(s ? F1 : F0, HM + (size_t)sc * nseg, TX, col, lo, mid, hi);
        }
        __syncthreads();
    }
    const uint32_t kNoneH = sizeof(TIn) == 2 ? kInf16 * kInf16 : kInf32;
    for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int col = u % TX, seg = u / TX;
        const int x = x0 + col;
        if (x >= w) continue;
        const long long base = kMode == 1 ? ((long long)(x >> 3) * outer_stride + outer) * 8 + (x & 7)
                                          : (long long)outer * outer_stride + x;
        hull_query<TIn, SB>(F0, F1, HM, TX, nseg, n, col, seg, [&](int p, int s, uint32_t best, bool none) {
            put_walk_value<kFinal>(out, base + (long long)p * stride, (uint32_t)s, best, none || best >= kNoneH,
                                   form);
        });
    }
}

// Pruned search (uint32 tiles whose cells mostly lie far from the other
// state in their plane: the z pass of a sparse volume, whose cells see a
// candidate in most planes but far away).  The line is cut into blocks of
// kPruneB cells with each block's smallest F_s value; a cell scans its own
// block, then visits blocks outwards on both sides, skipping a block when its
// minimum plus the squared distance to its nearest cell is not below the best
// value, and stops when the nearer unvisited block is at least sqrt(best)
// away.  Every skipped candidate is bounded below by the block's bound, so the
// result is the exact minimum over the line, the windowed search's.
template <typename TIn, bool kFinal, int TX, int kMode>
__device__ __noinline__ void edt_tile_pruned(const TIn* F0, const TIn* F1, int rows, int n, int w, int x0, int outer,
                                             void* out, long long stride, long long outer_stride, int form)
{
    if (sizeof(TIn) != 4) return;   // uint32 tiles only (the launcher never asks otherwise)
    constexpr int B = kPruneB;
    const int nseg = (n + 31) / 32, nb = (n + B - 1) / B;
    uint32_t* MB = reinterpret_cast<uint32_t*>(const_cast<TIn*>(F1) + (rows + 2 * kPadRows) * TX - kPadRows * TX) +
                   2 * TX * nseg;   // [state][block][column]
    // block minima; the rows of a block are read rotated by the block so that
    // a warp's lanes (8 columns x 4 blocks) hit different banks
    for (int jb = threadIdx.x; jb < 2 * nb * TX; jb += blockDim.x) {
        const int col = jb % TX, j = (jb / TX) % nb, st = jb / (TX * nb);
        const TIn* A = (st ? F1 : F0) + (size_t)j * B * TX + col;
        uint32_t m = 0xFFFFFFFFu;
        for (int i = 0; i < B; i++) m = min(m, (uint32_t)A[((i + j) & (B - 1)) * TX]);
        MB[jb] = m;
    }
    __syncthreads();
    constexpr int kGroups = TX / 8;
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5, wi = threadIdx.x >> 5;
    const int col = (wi % kGroups) * 8 + (lane & 7), sub = lane >> 3;
    const int qstep = 8 * (nw / kGroups);
    const int x = x0 + col;
    if (x >= w) return;
    const long long base = kMode == 1 ? ((long long)(x >> 3) * outer_stride + outer) * 8 + (x & 7)
                                      : (long long)outer * outer_stride + x;
    const uint32_t kNone = kInf32;
    for (int qa = 8 * (wi / kGroups) + sub; qa < n; qa += qstep) {
        for (int h = 0; h < 2; h++) {   // the lane's two cells, 4 positions apart (the windowed path's cells)
            const int q = qa + 4 * h;
            if (q >= n) break;
            const uint32_t c0 = F0[q * TX + col], c1 = F1[q * TX + col];
            const uint32_t s = c1 != 0;
            const TIn* A = (s ? F1 : F0) + col;
            const uint32_t* M = MB + (size_t)s * nb * TX + col;
            uint32_t best = c0 | c1;
            const int j0 = q / B;
            {   // the own block: distances j0 * B - q .. j0 * B + B - 1 - q
                int dd = j0 * B - q;
                const TIn* pa = A + (size_t)j0 * B * TX;
#pragma unroll
                for (int i = 0; i < B; i++, dd++) best = __viaddmin_u32((uint32_t)pa[i * TX], (uint32_t)(dd * dd), best);
            }
            for (int r = 1;; r++) {
                const int jl = j0 - r, jr = j0 + r;
                const uint32_t dl = (uint32_t)(q - jl * B - (B - 1)), dr = (uint32_t)(jr * B - q);
                const uint32_t dl2 = dl * dl, dr2 = dr * dr;
                const bool okl = jl >= 0 && dl2 < best, okr = jr < nb && dr2 < best;
                if (!okl && !okr) break;
                if (okl && M[(size_t)jl * TX] + dl2 < best) {   // leftwards from the block's last cell
                    const TIn* pa = A + ((size_t)jl * B + B - 1) * TX;
                    uint32_t d = dl;
#pragma unroll
                    for (int i = 0; i < B; i++, d++) best = __viaddmin_u32((uint32_t)pa[-i * TX], d * d, best);
                }
                if (okr && M[(size_t)jr * TX] + dr2 < best) {
                    const TIn* pa = A + (size_t)jr * B * TX;
                    uint32_t d = dr;
#pragma unroll
                    for (int i = 0; i < B; i++, d++) best = __viaddmin_u32((uint32_t)pa[i * TX], d * d, best);
                }
            }
            put_walk_value<kFinal>(out, base + (long long)q * stride, s, best, best >= kNone, form);
        }
    }
}

template <typename TIn, bool kFinal, int TX, int kMode>
__global__ void __launch_bounds__(512) k_edt_line_tma(const __grid_constant__ CUtensorMap map, void* __restrict__ out,
                                                      int w, int n, long long stride, long long outer_stride,
                                                      int along_z, int form, int* err, int outer0, uint32_t hull_pct,
                                                      uint32_t far_pct)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int nbox = (n + 255) >> 8;
    const int rows = nbox * 256;
    TIn* F0 = reinterpret_cast<TIn*>(smem_raw) + kPadRows * TX;   // rows -kPadRows .. rows+kPadRows-1, first the raw tile
    TIn* F1 = F0 + (rows + 2 * kPadRows) * TX;                      // the same for state 1
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned s_score;   // far cells of the tile (envelope-path test)
    int x0, outer, line = 0;
    if (kMode == 2) {
        // one block per (y, 8-column group) of the [y][x/8][z][8] array
        const int wb = w >> 3;
        line = blockIdx.x + outer0 * wb;
        outer = line / wb;
        x0 = (line - outer * wb) * 8;
    } else {
        x0 = blockIdx.x * TX;
        outer = blockIdx.y + outer0;
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        s_score = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, (uint32_t)(rows * TX * sizeof(TIn)));
        for (int b = 0; b < nbox; b++) {
            if (kMode == 2)
                tma_load_3d(F0 + b * 256 * TX, &map, 0, b * 256, line, &bar);
            else if (along_z)
                tma_load_3d(F0 + b * 256 * TX, &map, x0, outer, b * 256, &bar);
            else
                tma_load_3d(F0 + b * 256 * TX, &map, x0, b * 256, outer, &bar);
        }
    }
    // every thread polls; the block leaves together if the tile never arrived
    const bool arrived = mbar_wait(&bar, 0, 1u << 22);
    if (!__syncthreads_and(arrived)) {
        if (threadIdx.x == 0) atomicExch(err, 2);
        return;
    }
    // split by state (the top bit is the state, the rest the value), 16 bytes
    // at a time; positions n .. rows + kPadRows - 1 and the kPadRows rows
    // before 0 become sentinels.  A row is TX * sizeof(TIn) = 32 bytes.
    constexpr int kVecRow = TX * (int)sizeof(TIn) / 16;
    uint4* V0 = reinterpret_cast<uint4*>(F0);
    uint4* V1 = reinterpret_cast<uint4*>(F1);
    const uint32_t sw = sizeof(TIn) == 2 ? 0x7FFF7FFFu : 0x7FFFFFFFu;   // a word of sentinels / value bits
    const uint4 sent = make_uint4(sw, sw, sw, sw);
    // while splitting, count the cells with no cell of the other state on
    // their lower-dimension lines ("none"): their windowed walk runs to the
    // line end.  When they make up hull_pct percent of the tile (sparse or
    // empty volumes), the tile takes the envelope path.  The count looks at
    // the first word of every 16 bytes -- a quarter of the cells, a fixed
    // set of columns -- which is enough to tell the tiles apart and keeps the
    // dense tiles' split loop within a percent of its cost without the test.
    uint32_t score = 0;
    for (int i = threadIdx.x; i < n * kVecRow; i += blockDim.x) {
        const uint4 x = V0[i];
        uint4 a, b;
        split_word<TIn>(x.x, sw, &a.x, &b.x);
        split_word<TIn>(x.y, sw, &a.y, &b.y);
        split_word<TIn>(x.z, sw, &a.z, &b.z);
        split_word<TIn>(x.w, sw, &a.w, &b.w);
        V0[i] = a;
        V1[i] = b;
        if (hull_pct <= 100u || far_pct <= 100u) {   // uniform; skipped when both other paths are off
            if (sizeof(TIn) == 2) {
                score += __vcmpeq2(x.x & sw, sw) & 0x00010001u;   // one per "none" half, summed per half
            } else {
                // low half: "none" cells; high half: cells at least kFarDist
                // from the other state in their plane ("none" included)
                const uint32_t v = x.x & sw;
                score += (uint32_t)(v == sw) + ((uint32_t)(v >= kFarDist * kFarDist) << 16);
            }
        }
    }
    for (int i = n * kVecRow + threadIdx.x; i < (rows + kPadRows) * kVecRow; i += blockDim.x) {
        V0[i] = sent;
        V1[i] = sent;
    }
    for (int i = threadIdx.x; i < kPadRows * kVecRow; i += blockDim.x) {
        V0[i - kPadRows * kVecRow] = sent;
        V1[i - kPadRows * kVecRow] = sent;
    }
    if (sizeof(TIn) == 2) score = (score & 0xFFFFu) + (score >> 16);
    score = __reduce_add_sync(0xFFFFFFFFu, score);
    if ((threadIdx.x & 31) == 0 && score) atomicAdd(&s_score, score);
    __syncthreads();
    const long long sampled = (long long)n * min(TX, w - x0) / 4;
    const uint32_t n_none = sizeof(TIn) == 2 ? s_score : (s_score & 0xFFFFu), n_far = s_score >> 16;
    const bool use_hull = hull_pct <= 100u && 100LL * n_none >= (long long)hull_pct * sampled;

    if (use_hull) {
        edt_tile_envelope<TIn, kFinal, TX, kMode>(F0, F1, rows, n, w, x0, outer, out, stride, outer_stride, form);
        return;
    }
    if (sizeof(TIn) == 4 && far_pct <= 100u && 100LL * n_far >= (long long)far_pct * sampled) {
        edt_tile_pruned<TIn, kFinal, TX, kMode>(F0, F1, rows, n, w, x0, outer, out, stride, outer_stride, form);
        return;
    }

    // a warp covers 8 columns x 8 positions, each lane two cells of its
    // column 4 apart, both walked in one loop (a compact footprint:
    // neighbouring cells have similar search lengths; the probes of each half
    // of a step, 8 columns x 4 adjacent positions, fall in distinct
    // shared-memory banks); TX / 8 column groups per CTA
    constexpr int kGroups = TX / 8;
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5, wi = threadIdx.x >> 5;
    const int col = (wi % kGroups) * 8 + (lane & 7), sub = lane >> 3;
    const int qstep = 8 * (nw / kGroups);
    const int x = x0 + col;
    if (x >= w) return;
    const long long base = kMode == 1 ? ((long long)(x >> 3) * outer_stride + outer) * 8 + (x & 7)
                                      : (long long)outer * outer_stride + x;
    // "no cell of the other state reachable": INF (0x7FFF) squared for u16 input, 0x7FFFFFFF for u32
    const uint32_t kNone = sizeof(TIn) == 2 ? kInf16 * kInf16 : kInf32;
    const int q0 = 8 * (wi / kGroups) + sub;
    long long o = base + (long long)q0 * stride;   // output index of the lane's first cell
    const long long ostep = (long long)qstep * stride, o4 = 4 * stride;
    for (int qa = q0; qa < n; qa += qstep, o += ostep) {
        const bool has_b = qa + 4 < n;
        const int qb = has_b ? qa + 4 : qa;   // without a second cell the lane walks the first twice
        // a cell's value sits in its own state's array, 0 in the other (every own value is >= 1)
        const uint32_t a0 = F0[qa * TX + col], a1 = F1[qa * TX + col];
        const uint32_t b0 = F0[qb * TX + col], b1 = F1[qb * TX + col];
        const uint32_t sa = a1 != 0, sb = b1 != 0;
        const TIn* Aa = (sa ? F1 : F0) + col;
        const TIn* Ab = (sb ? F1 : F0) + col;
        uint32_t besta = sq_val<TIn>((TIn)(a0 | a1)), bestb = sq_val<TIn>((TIn)(b0 | b1));
        // both sides, two distances per trip, while k^2 < best for either cell
        // and k stays below kcap: within kPadRows - 4 of the nearer line end
        // of either cell (they are 4 positions apart, so neither walks past
        // the sentinels)
        const uint32_t kcap = (uint32_t)(min(qa, n - 1 - qb) + kPadRows - 4);
        const uint32_t cap2 = kcap * kcap;
        uint32_t k2 = 1, t = 3;   // k^2 and 2k + 1 for the next distance k
        uint32_t lim = min(max(besta, bestb), cap2);
        const TIn* pla = Aa + (qa - 1) * TX;
        const TIn* pra = Aa + (qa + 1) * TX;
        const TIn* plb = Ab + (qb - 1) * TX;
        const TIn* prb = Ab + (qb + 1) * TX;
        while (k2 < lim) {
            const uint32_t k2b = k2 + t;   // (k+1)^2
            // three-way minimum (u16) and fused add-min (u32): the DPX integer intrinsics
            if (sizeof(TIn) == 2) {
                besta = __vimin3_u32(besta, add_sq<TIn>(pla[0], k2), add_sq<TIn>(pra[0], k2));
                bestb = __vimin3_u32(bestb, add_sq<TIn>(plb[0], k2), add_sq<TIn>(prb[0], k2));
                besta = __vimin3_u32(besta, add_sq<TIn>(pla[-TX], k2b), add_sq<TIn>(pra[TX], k2b));
                bestb = __vimin3_u32(bestb, add_sq<TIn>(plb[-TX], k2b), add_sq<TIn>(prb[TX], k2b));
            } else {
                besta = __viaddmin_u32((uint32_t)pla[0], k2, besta);
                bestb = __viaddmin_u32((uint32_t)plb[0], k2, bestb);
                besta = __viaddmin_u32((uint32_t)pra[0], k2, besta);
                bestb = __viaddmin_u32((uint32_t)prb[0], k2, bestb);
                besta = __viaddmin_u32((uint32_t)pla[-TX], k2b, besta);
                bestb = __viaddmin_u32((uint32_t)plb[-TX], k2b, bestb);
                besta = __viaddmin_u32((uint32_t)pra[TX], k2b, besta);
                bestb = __viaddmin_u32((uint32_t)prb[TX], k2b, bestb);
            }
            pla -= 2 * TX;
            pra += 2 * TX;
            plb -= 2 * TX;
            prb += 2 * TX;
            k2 = k2b + t + 2;   // (k+2)^2
            t += 4;
            lim = min(max(besta, bestb), cap2);
        }
        // a cell whose walk stopped at the cap (past its nearer line end: kcap
        // is at least its distance to that end + kPadRows - 8) goes on along
        // the far side alone
        if (k2 < max(besta, bestb)) {   // rare: one test for both cells
            const int k = (int)(t >> 1);
            if (k2 < besta) besta = far_side<TIn, TX>(besta, qa, n, k, k2, pla, pra);
            if (k2 < bestb) bestb = far_side<TIn, TX>(bestb, qb, n, k, k2, plb, prb);
        }
        put_walk_value<kFinal>(out, o, sa, besta, besta >= kNone, form);
        if (has_b) put_walk_value<kFinal>(out, o + o4, sb, bestb, bestb >= kNone, form);
    }
}

constexpr size_t kStageLimit = 200 * 1024;   // largest staged line tile of the plain form

// set_attr = false: the caller raised the staged kernel's shared-memory limit
// to kStageLimit beforehand (prepare_edt_mask_2d_plain)
template <typename TIn, bool kFinal>
static void line_pass_plain(const TIn* in, void* out, int w, int n, long long stride, long long outer,
                            long long outer_stride, int form, cudaStream_t st, int outer0 = 0, bool set_attr = true)
{
    size_t bytes = (size_t)n * 32 * sizeof(TIn);
    dim3 grid((w + 31) / 32, (unsigned)outer);
    if (bytes <= kStageLimit) {
        auto kern = k_edt_line<TIn, kFinal, true>;
        if (set_attr && bytes > 48 * 1024)
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        kern<<<grid, 256, bytes, st>>>(in, out, w, n, stride, outer_stride, form, outer0);
    } else {
        k_edt_line<TIn, kFinal, false><<<grid, 256, 0, st>>>(in, out, w, n, stride, outer_stride, form, outer0);
    }
}

__global__ void k_flag_error(int* err)
{
    atomicExch(err, 2);
}

// Tensor map of the TMA line kernels: lines along y (along_z = 0) or z of a
// w x h x d array, TX columns per box row; mode 2: the [y][x/8][z][8] array.
template <typename TIn, int TX>
static bool line_map(CUtensorMap* map, const TIn* in, int w, int h, int d, int along_z, int mode)
{
    const CUtensorMapDataType type = sizeof(TIn) == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT32;
    if (mode == 2) {
        const uint64_t dims[3] = {8, (uint64_t)d, (uint64_t)(w / 8) * h};
        const uint64_t strides[2] = {8 * sizeof(TIn), (uint64_t)d * 8 * sizeof(TIn)};
        const uint32_t box[3] = {8, 256, 1};
        return encode_map_3d(map, in, type, dims, strides, box);
    }
    const uint64_t plane = (uint64_t)w * h;
    const uint64_t dims[3] = {(uint64_t)w, (uint64_t)h, (uint64_t)d};
    const uint64_t strides[2] = {(uint64_t)w * sizeof(TIn), plane * sizeof(TIn)};
    const uint32_t box[3] = {(uint32_t)TX, along_z ? 1u : 256u, along_z ? 256u : 1u};
    return encode_map_3d(map, in, type, dims, strides, box);
}

// True when a volume's y pass can write, and its z pass read, the
// [y][x/8][z][8] array: 8 | w, both line tiles fit, both maps encode.
static bool blocked_layout_ok(const uint16_t* vx, const uint32_t* ey, int w, int h, int d)
{
    if (w % 8 != 0 || d > 65535) return false;
    if (tma_tile_bytes<uint16_t, 16>(h) > 200 * 1024 || tma_tile_bytes<uint32_t, 8>(d) > 200 * 1024) return false;
    if ((long long)(w / 8) * h > 0x7FFFFFFFLL) return false;
    if (((uintptr_t)vx % 16) != 0 || ((uintptr_t)ey % 16) != 0) return false;
    CUtensorMap m;
    return line_map<uint16_t, 16>(&m, vx, w, h, d, 0, 1) && line_map<uint32_t, 8>(&m, ey, w, h, d, 1, 2);
}

// Share of "none" cells (percent) at which a line-pass tile takes the
// envelope path; above 100: never.  The tuned value (DOL_TUNE_EDT_HULL, by
// line length): 1 = windowed search only, 2 = envelope only, 3..100 = that
// percentage, 101 / 102 = no envelope path / the default share without the
// pruned search; 0 = 50 (the tiles of sparse and empty volumes; dense fields
// keep the windowed search, and uint32 tiles whose far cells still see a
// candidate take the pruned search, both faster there).
static uint32_t edt_hull_share(int n)
{
    const int v = tune_get(kTuneEdtHull, n);
    if (v == 1 || v == 101) return 0xFFFFFFFFu;
    if (v == 2) return 0u;
    return v >= 3 && v <= 100 ? (uint32_t)v : 50u;
}

// Share of far cells (percent) at which a uint32 tile that does not take the
// envelope path takes the pruned search; above 100: never.  DOL_TUNE_EDT_HULL
// 101 sends every such tile there, 102 keeps the windowed search.
static uint32_t edt_far_share(int n)
{
    const int v = tune_get(kTuneEdtHull, n);
    if (v == 101) return 0u;
    if (v == 1 || v == 102) return 0xFFFFFFFFu;
    return 50u;
}

// Lines along y (along_z = 0, outer index = z) or z (along_z = 1, outer = y)
// of a w x h x d array; outer indices outer0 .. outer0 + nouter - 1 (nouter < 0:
// all).  TMA needs 16-byte row pitches and a tile that fits in shared memory;
// otherwise the plain form runs.  mode 1 / 2 (blocked y-pass output / z-pass
// input) only after blocked_layout_ok.
template <typename TIn, bool kFinal>
static void line_pass(const TIn* in, void* out, int w, int h, int d, int along_z, int form, int* err, cudaStream_t st,
                      int outer0 = 0, int nouter = -1, int mode = 0)
{
    const int n = along_z ? d : h;
    const long long plane = (long long)w * h;
    const long long stride = along_z ? plane : w;
    const long long outer = nouter >= 0 ? nouter : (along_z ? h : d);
    const long long outer_stride = along_z ? w : plane;
    constexpr int TX = sizeof(TIn) == 2 ? 16 : 8;   // 32-byte box rows either way
    const size_t tile_bytes = tma_tile_bytes<TIn, TX>(n);
    const bool aligned = ((size_t)w * sizeof(TIn)) % 16 == 0 && ((uintptr_t)in % 16) == 0;
    const int tv = tune_get(kTuneEdt, w);
    const int threads = tv == 256 ? 256 : 512;
    const uint32_t hthr = edt_hull_share(n), fthr = edt_far_share(n);
    CUtensorMap map;
    if (mode == 1) {
        if (!line_map<TIn, TX>(&map, in, w, h, d, along_z, 0)) return;   // blocked_layout_ok encoded it already
        auto kern = k_edt_line_tma<TIn, kFinal, TX, 1>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_bytes);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        dim3 grid((w + TX - 1) / TX, (unsigned)outer);
        kern<<<grid, threads, tile_bytes, st>>>(map, out, w, n, (long long)w * d, d, along_z, form, err, outer0, hthr,
                                                fthr);
        return;
    }
    if (mode == 2) {
        if (!line_map<TIn, TX>(&map, in, w, h, d, along_z, 2)) {
            // blocked_layout_ok encoded this map; should the driver refuse it
            // now, the call reports failure rather than leave the field unwritten
            k_flag_error<<<1, 1, 0, st>>>(err);
            return;
        }
        auto kern = k_edt_line_tma<TIn, kFinal, 8, 2>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_bytes);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        const unsigned blocks = (unsigned)(outer * (w / 8));
        kern<<<blocks, threads, tile_bytes, st>>>(map, out, w, n, plane, w, along_z, form, err, outer0, hthr, fthr);
        return;
    }
    if (aligned && tile_bytes <= 200 * 1024 && outer <= 65535) {
        if (line_map<TIn, TX>(&map, in, w, h, d, along_z, 0)) {
            auto kern = k_edt_line_tma<TIn, kFinal, TX, 0>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_bytes);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            dim3 grid((w + TX - 1) / TX, (unsigned)outer);
            kern<<<grid, threads, tile_bytes, st>>>(map, out, w, n, stride, outer_stride, along_z, form, err, outer0,
                                                    hthr, fthr);
            return;
        }
    }
    line_pass_plain<TIn, kFinal>(in, out, w, n, stride, outer, outer_stride, form, st, outer0);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

bool encode_map_3d(CUtensorMap* map, const void* base, CUtensorMapDataType type, const uint64_t dims[3],
                   const uint64_t strides_bytes[2], const uint32_t box[3])
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p) {
            cudaGetLastError();
            return false;
        }
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    const cuuint32_t elem_strides[3] = {1, 1, 1};
    CUresult r = fn(map, type, 3, const_cast<void*>(base), dims, strides_bytes, box, elem_strides,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

size_t edt_workspace_bytes(int dim, int w, int h, int d)
{
    size_t cells = (size_t)w * h * (dim == 3 ? d : 1);
    size_t b = cells * sizeof(uint16_t);
    b = (b + 255) & ~(size_t)255;
    if (dim == 3) b += cells * sizeof(uint32_t);
    return b;
}

void launch_edt_mask(int dim, const uint32_t* mask, float* out, int w, int h, int d, int form, void* ws, int* err,
                     cudaStream_t st)
{
    long long rows = (long long)h * (dim == 3 ? d : 1);
    size_t cells = (size_t)w * rows;
    uint16_t* vx = static_cast<uint16_t*>(ws);
    long long blocks = (rows * 32 + 255) / 256;
    long long cap = (long long)g_num_sms * 16;
    {
        ProfScope ps("edt_x", st);
        k_edt_x<<<(int)(blocks < cap ? blocks : cap), 256, 0, st>>>(mask, vx, w, rows);
    }
    if (dim == 2) {
        ProfScope ps("edt_y_final", st);
        line_pass<uint16_t, true>(vx, out, w, h, 1, 0, form, err, st);
    } else {
        size_t off = (cells * sizeof(uint16_t) + 255) & ~(size_t)255;
        uint32_t* ey = reinterpret_cast<uint32_t*>(static_cast<char*>(ws) + off);
        const bool blk = blocked_layout_ok(vx, ey, w, h, d);
        {
            ProfScope ps("edt_y", st);
            line_pass<uint16_t, false>(vx, ey, w, h, d, 0, form, err, st, 0, -1, blk ? 1 : 0);   // y lines
        }
        ProfScope ps("edt_z_final", st);
        line_pass<uint32_t, true>(ey, out, w, h, d, 1, form, err, st, 0, -1, blk ? 2 : 0);   // z lines
    }
}

// The 3D mask EDT in pieces, for a caller that overlaps copies with it: the x
// and y passes run over `slabs` ranges of z, each after `ready(ctx, z0, z1)`
// (the caller makes the stream wait for those slices of the mask), and the
// last (z) pass over `chunks` ranges of y, each followed by `done(ctx, y0, y1)`
// (the caller queues work on rows y0..y1-1 of every slice, e.g. their copy
// back to the host).  Both hooks run on the host after / before the launches.
void launch_edt_mask_3d_chunked(const uint32_t* mask, float* out, int w, int h, int d, int form, void* ws, int* err,
                                cudaStream_t st, int slabs, void (*ready)(void*, int, int), int chunks,
                                void (*done)(void*, int, int), void* ctx)
{
    const size_t cells = (size_t)w * h * d;
    const int words = words_per_row(w);
    uint16_t* vx = static_cast<uint16_t*>(ws);
    const size_t off = (cells * sizeof(uint16_t) + 255) & ~(size_t)255;
    uint32_t* ey = reinterpret_cast<uint32_t*>(static_cast<char*>(ws) + off);
    const bool blk = blocked_layout_ok(vx, ey, w, h, d);
    slabs = slabs < 1 ? 1 : (slabs > d ? d : slabs);
    for (int s = 0; s < slabs; s++) {
        const int z0 = (int)((long long)d * s / slabs), z1 = (int)((long long)d * (s + 1) / slabs);
        if (z1 <= z0) continue;
        if (ready) ready(ctx, z0, z1);
        const long long rows = (long long)(z1 - z0) * h;
        const long long blocks = (rows * 32 + 255) / 256, cap = (long long)g_num_sms * 16;
        k_edt_x<<<(int)(blocks < cap ? blocks : cap), 256, 0, st>>>(mask + (size_t)z0 * h * words,
                                                                    vx + (size_t)z0 * h * w, w, rows);
        line_pass<uint16_t, false>(vx, ey, w, h, d, 0, form, err, st, z0, z1 - z0, blk ? 1 : 0);
    }
    chunks = chunks < 1 ? 1 : (chunks > h ? h : chunks);
    for (int c = 0; c < chunks; c++) {
        const int y0 = (int)((long long)h * c / chunks), y1 = (int)((long long)h * (c + 1) / chunks);
        if (y1 <= y0) continue;
        line_pass<uint32_t, true>(ey, out, w, h, d, 1, form, err, st, y0, y1 - y0, blk ? 2 : 0);
        if (done) done(ctx, y0, y1);
    }
}

// 2D mask EDT on caller-provided scratch (w*h uint16), plain loads only: no
// tensor maps, no bounded waits, nothing allocated.  The staged column
// kernel's shared-memory limit comes from prepare_edt_mask_2d_plain.
void launch_edt_mask_2d_plain(const uint32_t* mask, float* out, int w, int h, int form, uint16_t* scratch, int sms,
                              cudaStream_t st)
{
    long long blocks = ((long long)h * 32 + 255) / 256;
    long long cap = (long long)sms * 16;
    k_edt_x<<<(int)(blocks < cap ? blocks : cap), 256, 0, st>>>(mask, scratch, w, h);
    line_pass_plain<uint16_t, true>(scratch, out, w, h, w, 1, 0, form, st, 0, false);
}

cudaError_t prepare_edt_mask_2d_plain()
{
    return cudaFuncSetAttribute(k_edt_line<uint16_t, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kStageLimit);
}

// ------------------------------------------------ faithful float Felzenszwalb ----
// DOL::Felzenszwalb(w, h, float[]) on arbitrary input: the same 1D lower
// envelope in the same float operations (DistanceOcclusionLib.cpp:1026-1062),
// one thread per line.  Column pass into a scratch field, then row pass back.
// Envelope stacks live in the workspace, interleaved by line for coalescing.

__device__ void felz_line_dev(int n, const float* f, long long fstride, float* out, long long ostride, int* v, float* z,
                              long long sstride)
{
    int k = 0;
    v[0] = 0;
    z[0] = -FLT_MAX;
    z[sstride] = FLT_MAX;
    for (int q = 1; q < n; q++) {
        float hq = f[q * fstride] + (float)(q * q);
        float s;
        for (;;) {
            int p = v[k * sstride];
            float hp = f[p * fstride] + (float)(p * p);
            s = __fdiv_rn(hq - hp, (float)(2 * (q - p)));
            if (s > z[k * sstride]) break;
            k--;
        }
        k++;
        v[k * sstride] = q;
        z[k * sstride] = s;
        z[(k + 1) * sstride] = FLT_MAX;
    }
    k = 0;
    for (int q = 0; q < n; q++) {
        while (z[(k + 1) * sstride] < (float)q) k++;
        int p = v[k * sstride];
        out[q * ostride] = __fadd_rn((float)((q - p) * (q - p)), f[p * fstride]);
    }
}

__global__ void k_felz_cols(const float* __restrict__ in, float* __restrict__ td, int w, int h, int* v, float* z)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= w) return;
    // column x (stride w) -> td[x*h + q] (the reference's transposed scratch)
    felz_line_dev(h, in + x, w, td + (long long)x * h, 1, v + x, z + x, w);
}

__global__ void k_felz_rows(const float* __restrict__ td, float* __restrict__ out, int w, int h, int* v, float* z)
{
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= h) return;
    felz_line_dev(w, td + y, h, out + (long long)y * w, 1, v + y, z + y, h);
}

size_t felz_float_workspace_bytes(int w, int h)
{
    size_t n = (size_t)(w > h ? w : h);
    size_t lines = (size_t)(w > h ? w : h);
    size_t td = ((size_t)w * h * sizeof(float) + 255) & ~(size_t)255;
    size_t vb = (n * lines * sizeof(int) + 255) & ~(size_t)255;
    size_t zb = (n + 1) * lines * sizeof(float);
    return td + vb + zb;
}

void launch_felz_float_2d(float* dist, int w, int h, void* ws, cudaStream_t st)
{
    size_t n = (size_t)(w > h ? w : h);
    size_t lines = n;
    char* p = static_cast<char*>(ws);
    float* td = reinterpret_cast<float*>(p);
    p += ((size_t)w * h * sizeof(float) + 255) & ~(size_t)255;
    int* v = reinterpret_cast<int*>(p);
    p += (n * lines * sizeof(int) + 255) & ~(size_t)255;
    float* z = reinterpret_cast<float*>(p);
    (void)lines;
    // stacks are indexed [position * lines_in_pass + line]; each pass uses its own line count as the stride
    k_felz_cols<<<(w + 127) / 128, 128, 0, st>>>(dist, td, w, h, v, z);
    k_felz_rows<<<(h + 127) / 128, 128, 0, st>>>(td, dist, w, h, v, z);
}

}  // namespace dolk
