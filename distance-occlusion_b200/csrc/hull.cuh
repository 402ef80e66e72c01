// hull.cuh -- the lower-envelope form of the EDT line passes (k_edt.cu),
// __host__ __device__ so the CPU tests run the same code (tests/edt_hull_host.cpp).
//
// A line pass gives each cell of state s the 1D transform
//     min over p' of G_s(p') + (p - p')^2,
// where G_s(p') is 0 for a cell of the other state and the cell's own value
// squared (u16 input: v^2; u32 input: e) for a cell of state s; in the split
// tile that is F_s[p'] "squared" (sq_val), with the sentinel (0x7FFF /
// 0x7FFFFFFF) meaning "no cell of the other state on the lower-dimension
// lines" -- not a candidate.  The minimum is attained at a vertex of the lower
// convex hull of the points (p', G_s(p') + p'^2): Felzenszwalb's lower
// envelope of parabolas (DistanceOcclusionLib.cpp:1026-1062) seen as a hull,
// and as p grows the minimising vertex moves right.
//
// Candidates for transform s: state-s cells with a finite value, and
// other-state cells next to a state-s cell (a zero farther away is never the
// nearest for a state-s cell, the adjacent one is closer).
//
// Representation: per column and transform, a bitmask over positions (one
// 32-bit word per segment of SB cells, only the low SB bits used; the kernel
// uses SB = 32, the CPU tests 16 as well).  A (column, segment) unit builds its
// segment's hull as a stack of set bits; segments merge pairwise in a tree
// (the lower bridge of two x-separated hulls, walked from their facing ends,
// clearing the vertices it passes); each unit then walks its cells left to
// right with one pointer per state.  Arithmetic is exact: points in 64 bits,
// orientation by cross products of 32-bit differences (at most ~2^45).
//
// Arrays: Fs points at position 0 of one state's split array, rows of TXv
// elements (column col at offset col); positions up to the segment-rounded
// line end must be readable (the tile pads them with sentinels).  W points at
// one (state, column)'s hull words, nseg of them.
#pragma once

#include "common.cuh"

namespace dolk {

#if defined(__CUDA_ARCH__)
DOL_HD int ffs32(uint32_t x) { return __ffs(x) - 1; }            // lowest set bit (x != 0)
DOL_HD int hibit32(uint32_t x) { return 31 - __clz(x); }          // highest set bit (x != 0)
#else
DOL_HD int ffs32(uint32_t x) { return __builtin_ctz(x); }
DOL_HD int hibit32(uint32_t x) { return 31 - __builtin_clz(x); }
#endif

// squared own value of a split-tile entry: u16 entries hold a distance, u32
// entries a squared distance
template <typename TIn>
DOL_HD uint32_t sq_val(TIn v)
{
    return sizeof(TIn) == 2 ? (uint32_t)v * (uint32_t)v : (uint32_t)v;
}

// hull y of position p in transform s: G_s(p) + p^2.  Below 2^31 for every
// supported size: a candidate's G is at most (16383^2) * 2 < 2^29 and
// p^2 < 2^28, so points and their differences fit 32 bits.
template <typename TIn>
DOL_HD int hull_y(const TIn* Fs, int p, int TXv, int col)
{
    return (int)(sq_val<TIn>(Fs[p * TXv + col]) + (uint32_t)(p * p));
}

// true iff (xb, yb) lies strictly below the segment from (xa, ya) to (xc, yc),
// xa < xb < xc: two 32 x 32 -> 64-bit products, exact
DOL_HD bool hull_keep(int xa, int ya, int xb, int yb, int xc, int yc)
{
    return (long long)(xb - xa) * (long long)(yc - ya) - (long long)(xc - xa) * (long long)(yb - ya) > 0;
}

// Positions map to hull words SB cells each: word v / SB, bit v % SB.  Nearest vertex after v in words [.., hi) / before v in words
// [lo, ..); -1 if none.
template <int SB>
DOL_HD int hull_next(const uint32_t* W, int v, int hi)
{
    int wi = v / SB;
    uint32_t m = W[wi] & ~((2u << (v % SB)) - 1u);
    while (!m) {
        if (++wi >= hi) return -1;
        m = W[wi];
    }
    return wi * SB + ffs32(m);
}

template <int SB>
DOL_HD int hull_prev(const uint32_t* W, int v, int lo)
{
    int wi = v / SB;
    uint32_t m = W[wi] & ((1u << (v % SB)) - 1u);
    while (!m) {
        if (--wi < lo) return -1;
        m = W[wi];
    }
    return wi * SB + hibit32(m);
}

// Segment hulls of both transforms for unit (col, seg) of a line of n cells,
// written to HM[(s * TXv + col) * nseg + seg].
template <typename TIn, int SB = 32>
DOL_HD void hull_build(const TIn* F0, const TIn* F1, uint32_t* HM, int TXv, int nseg, int n, int col, int seg)
{
    const int p0 = seg * SB;
    const uint32_t sent = sizeof(TIn) == 2 ? 0x7FFFu : 0x7FFFFFFFu;
    uint32_t S = 0, inf = 0;   // state bits; own value "none"
    for (int i = 0; i < SB; i++) {
        // rotated by the segment: the units of a warp, in consecutive
        // segments, then read rows in different shared-memory banks
        const int t = (i + seg) & (SB - 1), p = p0 + t;
        const uint32_t r0 = F0[p * TXv + col], r1 = F1[p * TXv + col];
        S |= (uint32_t)(r1 != 0) << t;
        inf |= (uint32_t)((r0 | r1) == sent) << t;
    }
    const uint32_t full = SB == 32 ? 0xFFFFFFFFu : ((1u << SB) - 1u);
    const uint32_t live = n - p0 >= SB ? full : ((1u << (n - p0)) - 1u);
    // the states just outside the segment (outside the line: neither)
    const bool pv = p0 > 0, nx = p0 + SB < n;
    const uint32_t s_prev = pv ? (uint32_t)(F1[(p0 - 1) * TXv + col] != 0) : 0u;
    const uint32_t s_next = nx ? (uint32_t)(F1[(p0 + SB) * TXv + col] != 0) : 0u;
    for (int s = 0; s < 2; s++) {
        const TIn* Fs = s ? F1 : F0;
        const uint32_t own = (s ? S : ~S) & live;
        const uint32_t other = (s ? ~S : S) & live;
        const uint32_t own_prev = pv && (s ? s_prev : !s_prev) ? 1u : 0u;
        const uint32_t own_next = nx && (s ? s_next : !s_next) ? 1u : 0u;
        const uint32_t near_own = (own << 1) | (own >> 1) | own_prev | (own_next << (SB - 1));
        uint32_t cand = (own & ~inf) | (other & near_own);
        uint32_t M = 0;
        int xa = -1, xb = -1;
        int ya = 0, yb = 0;
        while (cand) {
            const int t = ffs32(cand);
            cand &= cand - 1;
            const int p = p0 + t;
            const int yc = hull_y<TIn>(Fs, p, TXv, col);
            while (xa >= 0 && !hull_keep(xa, ya, xb, yb, p, yc)) {
                M &= ~(1u << (xb - p0));   // pop the top
                xb = xa;
                yb = ya;
                const uint32_t below = M & ((1u << (xb - p0)) - 1u);
                if (below) {
                    xa = p0 + hibit32(below);
                    ya = hull_y<TIn>(Fs, xa, TXv, col);
                } else {
                    xa = -1;
                }
            }
            M |= 1u << t;
            xa = xb;
            ya = yb;
            xb = p;
            yb = yc;
        }
        HM[(s * TXv + col) * nseg + seg] = M;
    }
}

// Merges the hulls of segments [lo, mid) and [mid, hi) of one (state, column).
template <typename TIn, int SB = 32>
DOL_HD void hull_merge(const TIn* Fs, uint32_t* W, int TXv, int col, int lo, int mid, int hi)
{
    int a = -1, b = -1;
    for (int i = mid - 1; i >= lo && a < 0; i--)
        if (W[i]) a = i * SB + hibit32(W[i]);
    if (a < 0) return;
    for (int i = mid; i < hi && b < 0; i++)
        if (W[i]) b = i * SB + ffs32(W[i]);
    if (b < 0) return;
    int ya = hull_y<TIn>(Fs, a, TXv, col), yb = hull_y<TIn>(Fs, b, TXv, col);
    for (;;) {
        const int ap = hull_prev<SB>(W, a, lo);
        if (ap >= 0) {
            const int yp = hull_y<TIn>(Fs, ap, TXv, col);
            if (!hull_keep(ap, yp, a, ya, b, yb)) {
                W[a / SB] &= ~(1u << (a % SB));
                a = ap;
                ya = yp;
                continue;
            }
        }
        const int bn = hull_next<SB>(W, b, hi);
        if (bn >= 0) {
            const int yn = hull_y<TIn>(Fs, bn, TXv, col);
            if (!hull_keep(a, ya, b, yb, bn, yn)) {
                W[b / SB] &= ~(1u << (b % SB));
                b = bn;
                yb = yn;
                continue;
            }
        }
        break;
    }
}

// value of hull vertex v at position p: G(v) + (p - v)^2
template <typename TIn>
DOL_HD uint32_t hull_at(const TIn* Fs, int v, int p, int TXv, int col)
{
    const int d = p - v;
    return sq_val<TIn>(Fs[v * TXv + col]) + (uint32_t)(d * d);
}

// The cells of unit (col, seg) against the merged hulls: emit(p, s, best,
// none) per cell p < n, best = the transform's value (meaningless if none).
template <typename TIn, int SB = 32, class Emit>
DOL_HD void hull_query(const TIn* F0, const TIn* F1, const uint32_t* HM, int TXv, int nseg, int n, int col, int seg,
                       Emit&& emit)
{
    // per state: the current vertex c (-2 = not placed yet, -1 = empty hull)
    // and the vertex after it r (-2 = not looked up, -1 = none): c only moves
    // right, so r stays valid until c moves, and the scan over empty hull
    // words to find it is done once per move, not once per cell
    int c0 = -2, c1 = -2, r0 = -2, r1 = -2;
    const int p0 = seg * SB, p1 = n < p0 + SB ? n : p0 + SB;
    for (int p = p0; p < p1; p++) {
        const int s = F1[p * TXv + col] != 0;
        const TIn* Fs = s ? F1 : F0;
        const uint32_t* W = HM + (s * TXv + col) * nseg;
        int c = s ? c1 : c0, r = s ? r1 : r0;
        if (c == -2) {   // first cell of this state in the unit: place the pointer
            // the first vertex at or after p, else the last one before it
            if (p == 0)
                c = (W[0] & 1u) ? 0 : hull_next<SB>(W, 0, nseg);
            else
                c = hull_next<SB>(W, p - 1, nseg);
            if (c < 0 && p > 0) c = hull_prev<SB>(W, p, 0);
            if (c >= 0) {
                uint32_t cv = hull_at<TIn>(Fs, c, p, TXv, col);
                for (;;) {   // the values along the hull are convex: walk down to the left
                    const int l = hull_prev<SB>(W, c, 0);
                    if (l < 0) break;
                    const uint32_t lv = hull_at<TIn>(Fs, l, p, TXv, col);
                    if (lv > cv) break;
                    c = l;
                    cv = lv;
                }
            }
            r = -2;
        }
        uint32_t best = 0xFFFFFFFFu;
        if (c >= 0) {
            best = hull_at<TIn>(Fs, c, p, TXv, col);
            if (r == -2) r = hull_next<SB>(W, c, nseg);
            while (r >= 0) {   // and to the right, as p advances
                const uint32_t rv = hull_at<TIn>(Fs, r, p, TXv, col);
                if (rv > best) break;
                c = r;
                best = rv;
                r = hull_next<SB>(W, c, nseg);
            }
        }
        if (s) {
            c1 = c;
            r1 = r;
        } else {
            c0 = c;
            r0 = r;
        }
        emit(p, s, best, c < 0);
    }
}

}  // namespace dolk
