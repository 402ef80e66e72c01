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
// be solved by iterating to the unique fixed point:
//
//   round 0   each segment guesses its input (the neighbour's value before the
//             pass) and runs its cells serially;
//   round r   each segment takes as input the output of the nearest segment
//             before it that did NOT simply pass its input through (a segment
//             whose output equals its input shifted by its length is
//             "transparent"), shifted across the transparent segments between;
//   stop      when every segment's input equals its predecessor's output.
//
// At the stop every segment's input is exactly what the serial pass would feed
// it, so the result is bit-identical to the serial pass.  Termination: if
// segments 0..k are correct after round r, segment k+1 is correct after round
// r+1 (its jump source is correct and everything between passed the correct
// value through), so at most (segments) rounds; on real rows it is 1-3 rounds,
// and the transparent-jump rule is what keeps long chains (a seed's influence
// crossing an empty row) to a few rounds instead of one round per segment.
#pragma once

#include "common.cuh"

namespace dolk {

template <class Cell>
struct ScanShared {
    // per round parity: each thread's segment output, and per warp a ballot of
    // the threads whose segment was not transparent
    Cell out[2][1024];
    uint32_t nt[2][32];
    Cell guess[1024];
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
            // both the chain and the diagonal candidate exist iff a cell precedes
            // this one in the row's scan order
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
// cells; n: cells of this thread (0 if none).  Exact; see the file comment.
template <class Cell, int S, bool kDiag, int dir>
__device__ __forceinline__ void row_pass(Cell (&R)[S], const Cell (&V)[S], int t, int nseg, int n, int cw,
                                         ScanShared<Cell>& sh, const Cell (&D)[S], bool row_first_diag_ok)
{
    const int lane = t & 31, wi = t >> 5;
    const bool active = t < nseg;
    // scan-order index of this segment and of its predecessor's thread
    const int sigma = dir > 0 ? t : nseg - 1 - t;
    const int pred = t - dir;
    const bool has_pred = active && sigma > 0;
    (void)row_first_diag_ok;

    // round 0 guess: the predecessor's boundary cell before the pass
    Cell edge = V[0];
    if (dir > 0) {
#pragma unroll
        for (int s = 1; s < S; s++)
            if (s < n) edge = V[s];
    }
    if (active) sh.guess[t] = edge;
    __syncthreads();
    Cell in = has_pred ? sh.guess[pred] : V[0];
    bool has_in = has_pred;

    for (int r = 0;; r++) {
        const int b = r & 1;
        Cell out = seg_pass<Cell, S, kDiag, dir>(R, V, n, cw, in, has_in, D);
        const bool trans = has_in && same(out, addx(in, -dir * cw * n));
        if (active) sh.out[b][t] = out;
        const uint32_t nt = __ballot_sync(0xFFFFFFFFu, active && !trans);
        if (lane == 0) sh.nt[b][wi] = nt;
        __syncthreads();

        bool bad = has_pred && !same(in, sh.out[b][pred]);
        // next input: the nearest non-transparent segment before us in scan order
        Cell nin = in;
        if (has_pred) {
            int j = -1;
            if (dir > 0) {
                uint32_t below = nt & ((1u << lane) - 1u);
                if (below) {
                    j = (wi << 5) + 31 - __clz(below);
                } else {
                    for (int ww = wi - 1; ww >= 0; ww--) {
                        uint32_t m = sh.nt[b][ww];
                        if (m) { j = (ww << 5) + 31 - __clz(m); break; }
                    }
                }
            } else {
                uint32_t above = lane == 31 ? 0u : (nt & ~((2u << lane) - 1u));
                if (above) {
                    j = (wi << 5) + __ffs(above) - 1;
                } else {
                    const int nwarps = (nseg + 31) >> 5;
                    for (int ww = wi + 1; ww < nwarps; ww++) {
                        uint32_t m = sh.nt[b][ww];
                        if (m) { j = (ww << 5) + __ffs(m) - 1; break; }
                    }
                }
            }
            // j exists: the first segment in scan order is never transparent
            const int gap = (dir > 0 ? t - j : j - t) - 1;   // full segments in between
            nin = addx(sh.out[b][j], -dir * cw * S * gap);
        }
        // the fixed point is reached within nseg rounds; the cap only guards
        // against a logic error turning into an endless loop on the device
        if (!__syncthreads_or(bad) || r > nseg + 2) break;
        in = nin;
    }
}

}  // namespace dolk
