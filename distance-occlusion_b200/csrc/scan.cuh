// scan.cuh -- exact parallel form of the reference's serial x passes.
//
// Every delta sweep in the reference ends each row with one or two serial
// passes along x (Danielsson :722-738, FastSweep :669-693, :2245-2255):
//
//     v[i] = closer(v[i], v[i-dir] shifted by -dir*cw in x)      (+ a fixed
//            candidate D[i] from the previous row in FastSweep 2D)
//
// `closer` keeps the incumbent on ties, and which of two deltas is closer can
// change along the row, so this is not an associative scan: the result depends
// on the exact chain of replacements.  It is still a composition of per-cell
// functions v -> f_i(v), so a row split into segments (S cells per thread) can
// be solved by iterating segment inputs to the unique fixed point:
//
//   round 0   each segment takes as input its predecessor's boundary cell as
//             it was before the pass (published during the previous pass);
//   round r   each segment takes the output of the nearest segment before it
//             that did NOT pass its input through unchanged ("transparent":
//             output == input shifted by the segment length), shifted across
//             the transparent segments in between;
//   stop      when every segment's input equals its predecessor's output.
//
// At the stop every input is what the serial pass would feed that segment, so
// the result is bit-identical to the serial pass.  It terminates: if segments
// 0..k are right after round r, segment k+1 is right after round r+1 (its
// jump source is right and everything between passed the right value on), so
// at most one round per segment; measured rows take 1-3 rounds, the jump rule
// keeping long chains (a seed's influence crossing an empty row) short.
//
// One barrier per round: a thread can tell by itself whether its successor's
// input was right, because that input is either the thread's own output (the
// thread was not transparent) or its own input shifted by its length (it
// was); so each thread checks its successor and a single __syncthreads_or
// both publishes the round's outputs and decides whether another round runs.
#pragma once

#include "common.cuh"

namespace dolk {

constexpr int kMaxScanThreads = 512;

template <class Cell, int N = kMaxScanThreads>
struct ScanShared {
    Cell out[2][N];     // segment outputs, by round parity
    uint32_t nt[2][32]; // per warp: ballot of non-transparent segments, by round parity
    Cell guess[2][N];   // boundary cells published for the next pass, by pass parity
    Cell edge[2][N];    // FastSweep 2D: each segment's boundary cell of the previous row
};

// Load/store helpers for row cells.  2D cells are one uint32; 3D cells three int16.
DOL_HD C2 cell_load(const uint32_t* p, long long i) { return unpack2(p[i]); }
DOL_HD void cell_store(uint32_t* p, long long i, C2 c) { p[i] = pack2(c); }
DOL_HD C3 cell_load(const int16_t* p, long long i)
{
    const int16_t* c = p + 3 * i;
    return C3{c[0], c[1], c[2]};
}
DOL_HD void cell_store(int16_t* p, long long i, C3 c)
{
    int16_t* o = p + 3 * i;
    o[0] = (int16_t)c.x;
    o[1] = (int16_t)c.y;
    o[2] = (int16_t)c.z;
}

// The boundary cell of a segment on the side its successor sees in scan
// direction dir: the last live cell for dir > 0, the first for dir < 0.
// (Unrolled select, so the register array is never indexed dynamically.)
template <class Cell, int S, int dir>
__device__ __forceinline__ Cell seg_edge(const Cell (&A)[S], int n)
{
    Cell e = A[0];
    if (dir > 0) {
#pragma unroll
        for (int s = 1; s < S; s++)
            if (s < n) e = A[s];
    }
    return e;
}

// Segment-local serial pass.  dir = +1: cells 0..n-1, chain shift -cw;
// dir = -1: cells n-1..0, chain shift +cw (a template argument, so the
// register arrays stay in registers).  D (FastSweep 2D) holds the
// previous-row diagonal candidate of each cell; like the chain candidate it
// exists for every cell but the first of the row in scan order.
template <class Cell, int S, bool kDiag, int dir>
__device__ __forceinline__ Cell seg_pass(Cell (&R)[S], const Cell (&V)[S], int n, int cw, Cell in, bool has_in,
                                         const Cell (&D)[S])
{
    Cell cur = in;
    bool have = has_in;
#pragma unroll
    for (int u = 0; u < S; u++) {
        const int s = dir > 0 ? u : S - 1 - u;
        if (s < n) {
            Cell v = V[s];
            if (have) {
                v = closer(v, addx(cur, -dir * cw));
                if (kDiag) v = closer(v, D[s]);
            }
            R[s] = v;
            cur = v;
            have = true;
        }
    }
    return cur;
}

// The row pass over the whole CTA.  t: thread index; nseg: threads holding
// cells; n: cells of this thread (0 if none); in0: this segment's round-0
// input (its predecessor's boundary cell before the pass).  `publish(R)` runs
// after every round, before the round's barrier: the caller uses it to post
// what the NEXT pass needs from this thread, so the final round's post is
// visible to all threads when this function returns.
template <class Cell, int S, bool kDiag, int dir, class Pub, int N>
__device__ __forceinline__ void row_pass(Cell (&R)[S], const Cell (&V)[S], int t, int nseg, int n, int cw,
                                         ScanShared<Cell, N>& sh, const Cell (&D)[S], Cell in0, Pub&& publish)
{
    const int lane = t & 31, wi = t >> 5;
    const bool active = t < nseg;
    const int sigma = dir > 0 ? t : nseg - 1 - t;   // position in scan order
    const bool has_pred = active && sigma > 0;
    const bool has_succ = active && sigma < nseg - 1;

    Cell in = in0;
    Cell succ_in = seg_edge<Cell, S, dir>(V, n);   // what my successor takes in round 0
    for (int r = 0;; r++) {
        const int b = r & 1;
        const Cell out = seg_pass<Cell, S, kDiag, dir>(R, V, n, cw, in, has_pred, D);
        publish(R);
        const bool trans = has_pred && same(out, addx(in, -dir * cw * n));
        if (active) sh.out[b][t] = out;
        const uint32_t nt = __ballot_sync(0xFFFFFFFFu, active && !trans);
        if (lane == 0) sh.nt[b][wi] = nt;
        const bool bad = has_succ && !same(succ_in, out);
        // the cap only keeps a logic error from looping on the device; the
        // fixed point is reached within nseg rounds
        if (!__syncthreads_or(bad) || r > nseg + 2) break;

        // round r+1 input: nearest non-transparent segment before us in scan order
        if (has_pred) {
            int j = -1;
            if (dir > 0) {
                const uint32_t below = nt & ((1u << lane) - 1u);
                if (below) {
                    j = (wi << 5) + 31 - __clz(below);
                } else {
                    for (int ww = wi - 1; ww >= 0; ww--) {
                        const uint32_t m = sh.nt[b][ww];
                        if (m) { j = (ww << 5) + 31 - __clz(m); break; }
                    }
                }
            } else {
                const uint32_t above = lane == 31 ? 0u : (nt & ~((2u << lane) - 1u));
                if (above) {
                    j = (wi << 5) + __ffs(above) - 1;
                } else {
                    const int nwarps = (nseg + 31) >> 5;
                    for (int ww = wi + 1; ww < nwarps; ww++) {
                        const uint32_t m = sh.nt[b][ww];
                        if (m) { j = (ww << 5) + __ffs(m) - 1; break; }
                    }
                }
            }
            // j exists: the first segment in scan order is never transparent
            const int gap = (dir > 0 ? t - j : j - t) - 1;   // full segments in between
            in = addx(sh.out[b][j], -dir * cw * S * gap);
        }
        // my successor's round r+1 input, by the same rule: my output, or (if I
        // passed my input through) my new input carried across my cells
        succ_in = trans ? addx(in, -dir * cw * n) : out;
    }
}

}  // namespace dolk

namespace dolk {

// ---- single-warp form -----------------------------------------------------------
// For rows of at most 32*S cells one warp holds the whole row and every
// exchange is a shuffle: no shared memory, no CTA barrier.  Same rounds, same
// jump rule, same exactness argument as row_pass; convergence is a warp vote.

DOL_HD C2 shfl_cell(unsigned m, C2 c, int src)
{
#if defined(__CUDA_ARCH__)
    return C2{__shfl_sync(m, c.x, src), __shfl_sync(m, c.y, src)};
#else
    (void)m; (void)src;
    return c;
#endif
}
DOL_HD C3 shfl_cell(unsigned m, C3 c, int src)
{
#if defined(__CUDA_ARCH__)
    return C3{__shfl_sync(m, c.x, src), __shfl_sync(m, c.y, src), __shfl_sync(m, c.z, src)};
#else
    (void)m; (void)src;
    return c;
#endif
}

// The predecessor's boundary cell before the pass (round-0 input), from the
// lane before (dir > 0) or after (dir < 0) in scan order.
template <class Cell, int S, int dir>
__device__ __forceinline__ Cell warp_round0_input(const Cell (&V)[S], int n, int lane)
{
    const Cell e = seg_edge<Cell, S, dir>(V, n);
    return shfl_cell(0xFFFFFFFFu, e, dir > 0 ? (lane > 0 ? lane - 1 : 0) : (lane < 31 ? lane + 1 : 31));
}

template <class Cell, int S, bool kDiag, int dir>
__device__ __forceinline__ void row_pass_warp(Cell (&R)[S], const Cell (&V)[S], int lane, int nseg, int n, int cw,
                                              const Cell (&D)[S], Cell in0)
{
    const bool active = lane < nseg;
    const int sigma = dir > 0 ? lane : nseg - 1 - lane;
    const bool has_pred = active && sigma > 0;
    const bool has_succ = active && sigma < nseg - 1;
    Cell in = in0;
    Cell succ_in = seg_edge<Cell, S, dir>(V, n);
    for (int r = 0;; r++) {
        const Cell out = seg_pass<Cell, S, kDiag, dir>(R, V, n, cw, in, has_pred, D);
        const bool trans = has_pred && same(out, addx(in, -dir * cw * n));
        const uint32_t nt = __ballot_sync(0xFFFFFFFFu, active && !trans);
        const bool bad = has_succ && !same(succ_in, out);
        if (!__any_sync(0xFFFFFFFFu, bad) || r > nseg + 2) break;
        // nearest non-transparent lane before me in scan order (exists for has_pred)
        int j = lane;
        if (dir > 0) {
            const uint32_t below = nt & ((1u << lane) - 1u);
            if (below) j = 31 - __clz(below);
        } else {
            const uint32_t above = lane == 31 ? 0u : (nt & ~((2u << lane) - 1u));
            if (above) j = __ffs(above) - 1;
        }
        const Cell src = shfl_cell(0xFFFFFFFFu, out, j);
        if (has_pred) {
            const int gap = (dir > 0 ? lane - j : j - lane) - 1;
            in = addx(src, -dir * cw * S * gap);
        }
        succ_in = trans ? addx(in, -dir * cw * n) : out;
    }
}

}  // namespace dolk
