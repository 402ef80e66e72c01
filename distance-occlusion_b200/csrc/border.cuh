// border.cuh -- signed border initialisation as a per-word gather.
//
// The reference (SetBorderCellsCombo, DistanceOcclusionLib.cpp:504-599 for 2D,
// :1820-2150 for 3D) walks the mask once and writes half-cell deltas in a fixed
// program order; later writes win, and diagonal writes only land in cells that
// are still at max (or, in 3D, that hold a diagonal).  The result therefore
// depends on that order, including writes that cross a word boundary: the
// x-edge / diagonal writes of bit 0 of word k+1 land in cell 31 of word k
// AFTER all of word k's writes of the same row pair.
//
// Here one thread owns the 32 cells of one (row, word) and replays, in the
// reference's order, every write that can land in them: the row pairs (and in
// 3D slice pairs) that contain the row, and words k and k+1.  The 32 cells are
// held as bit planes (one bit per cell): "still at max" and, per axis, "non-zero"
// and "negative" -- every value the reference writes has components in
// {-1, 0, +1}.  A group of writes from the reference becomes a masked select on
// the planes, so a word costs a few hundred bit operations and no memory
// traffic beyond the 3x3(x3) neighbouring mask words.
//
// Everything is __host__ __device__ so the CPU test build can check it against
// the oracle without a GPU.
#pragma once

#include "common.cuh"

namespace dolk {

// ---------------------------------------------------------------- 2D ----

struct Planes2 {
    uint32_t mx, xn, xs, yn, ys;
};

DOL_HD void put2(Planes2& p, uint32_t sel, int vx, int vy)
{
    p.mx &= ~sel;
    p.xn = vx ? (p.xn | sel) : (p.xn & ~sel);
    p.xs = vx < 0 ? (p.xs | sel) : (p.xs & ~sel);
    p.yn = vy ? (p.yn | sel) : (p.yn & ~sel);
    p.ys = vy < 0 ? (p.ys | sel) : (p.ys & ~sel);
}

// Bit vectors of one word for the row pair (top, bottom) -- names follow the
// roles, not the reference's variables.
struct Pair2 {
    uint32_t yedge;    // top and bottom differ at x                  (writes y deltas)
    uint32_t xedge;    // top row differs between x-1 and x          (writes x deltas)
    uint32_t yedgel;   // top and bottom differ at x-1
    uint32_t diag;     // corner case: yedge != yedgel
};

DOL_HD Pair2 pair2(int w, const uint32_t* top, const uint32_t* bot, int k)
{
    uint32_t live = live_bits(w, k);
    uint32_t t = top[k], tl = left_word(top, k);
    Pair2 q;
    q.xedge = (t ^ tl) & live;
    if (bot) {
        uint32_t b = bot[k], bl = left_word(bot, k);
        q.yedge = (t ^ b) & live;
        q.yedgel = tl ^ bl;
        q.diag = (q.yedge ^ q.yedgel) & live;
    } else {
        q.yedge = q.yedgel = q.diag = 0;
    }
    return q;
}

// Apply the writes of one row pair that land in this row.  s = 0: the row is
// the top of the pair; s = 1: the bottom.  bot == nullptr means the reference's
// last-row loop (x edges only, :573-597).
DOL_HD void row_pair2(Planes2& p, int w, const uint32_t* top, const uint32_t* bot, int k, int s)
{
    const int vy = 1 - 2 * s;
    Pair2 q = pair2(w, top, bot, k);
    // diagonals whose row (xedge bit) is ours: sx=1 -> cell b, sx=0 -> cell b-1
    uint32_t mine = q.diag & (s ? q.xedge : ~q.xedge);
    put2(p, mine & q.yedgel & p.mx, -1, vy);
    put2(p, ((mine & ~q.yedgel) >> 1) & p.mx, +1, vy);
    if (s == 0) {   // x edges land in the top row: b gets (-1,0), then b-1 gets (+1,0)
        put2(p, q.xedge, -1, 0);
        put2(p, q.xedge >> 1, +1, 0);
    }
    put2(p, q.yedge, 0, s ? -1 : +1);

    // word k+1, bit 0: its writes to "cell -1" are our cell 31, after all of ours
    if (32 * (k + 1) < w) {
        Pair2 r = pair2(w, top, bot, k + 1);
        const uint32_t c31 = 0x80000000u;
        if ((r.diag & 1u) && !(r.yedgel & 1u) && (int)(r.xedge & 1u) == s && (p.mx & c31)) put2(p, c31, +1, vy);
        if (s == 0 && (r.xedge & 1u)) put2(p, c31, +1, 0);
    }
}

// Final border-init planes of word k of row y.
DOL_HD Planes2 border2_word(int w, int h, const uint32_t* mask, int y, int k)
{
    const int ws = words_per_row(w);
    Planes2 p{0xFFFFFFFFu, 0, 0, 0, 0};
    const uint32_t* row = mask + (size_t)y * ws;
    if (y >= 1) row_pair2(p, w, row - ws, row, k, 1);
    if (y + 1 < h)
        row_pair2(p, w, row, row + ws, k, 0);
    else
        row_pair2(p, w, row, nullptr, k, 0);
    return p;
}

DOL_HD C2 decode2(const Planes2& p, int b)
{
    if (p.mx >> b & 1u) return C2{kMax2, kMax2};
    int x = (p.xn >> b & 1u) ? ((p.xs >> b & 1u) ? -1 : 1) : 0;
    int y = (p.yn >> b & 1u) ? ((p.ys >> b & 1u) ? -1 : 1) : 0;
    return C2{x, y};
}

// ---------------------------------------------------------------- 3D ----

struct Planes3 {
    uint32_t mx, xn, xs, yn, ys, zn, zs;
};

DOL_HD void put3(Planes3& p, uint32_t sel, int vx, int vy, int vz)
{
    p.mx &= ~sel;
    p.xn = vx ? (p.xn | sel) : (p.xn & ~sel);
    p.xs = vx < 0 ? (p.xs | sel) : (p.xs & ~sel);
    p.yn = vy ? (p.yn | sel) : (p.yn & ~sel);
    p.ys = vy < 0 ? (p.ys | sel) : (p.ys & ~sel);
    p.zn = vz ? (p.zn | sel) : (p.zn & ~sel);
    p.zs = vz < 0 ? (p.zs | sel) : (p.zs & ~sel);
}

// cells that a face/edge diagonal may overwrite: at max or already diagonal
DOL_HD uint32_t diag_ok(const Planes3& p) { return p.mx | (p.xn & p.yn) | (p.xn & p.zn) | (p.yn & p.zn); }

// Which groups of writes a step of the reference performs.
enum StepKind : int {
    kFull = 0,       // slice pair x row pair, all seven groups   (:1852-2003)
    kLastRowOfPair,  // last row of a slice pair: fy, ex, ez      (:2005-2065)
    kLastSlice,      // row pair of the last slice: fz, ex, ey    (:2068-2131)
    kLastRow,        // last row of the last slice: ex            (:2133-2150)
};

// Bit vectors of one word of a 2x2x2 (or degenerate) cube: "L" is cell x-1
// and "R" is cell x; rows r0/r1 and slices s0/s1.
struct Cube3 {
    uint32_t ex, ey, ez, ezR, eyR;
    uint32_t fx, fy, fz, fxx, corner;
};

DOL_HD Cube3 cube3(int w, int kind, const uint32_t* r00, const uint32_t* r01, const uint32_t* r10,
                   const uint32_t* r11, int k)
{
    // r00: slice s0 row r0, r01: s0 row r1, r10: s1 row r0, r11: s1 row r1
    uint32_t live = live_bits(w, k);
    Cube3 c{};
    uint32_t R000 = r00[k], L000 = left_word(r00, k);
    c.ex = L000 ^ R000;
    if (kind == kFull || kind == kLastSlice) {
        uint32_t R010 = r01[k], L010 = left_word(r01, k);
        c.ey = L000 ^ L010;
        c.eyR = R000 ^ R010;
        c.fz = (c.ey ^ c.eyR) & live;     // == ex ^ (x change of row r1)
    }
    if (kind == kFull || kind == kLastRowOfPair) {
        uint32_t R100 = r10[k], L100 = left_word(r10, k);
        c.ez = L000 ^ L100;
        c.ezR = R000 ^ R100;
        c.fy = (c.ez ^ c.ezR) & live;
        if (kind == kFull) {
            uint32_t R110 = r11[k], L110 = left_word(r11, k);
            uint32_t eyL1 = L100 ^ L110, eyR1 = R100 ^ R110;
            c.fx = c.ey ^ eyL1;
            c.fxx = (c.eyR ^ eyR1) & live;
            c.corner = (c.fz ^ eyL1 ^ eyR1) & live;
        }
    }
    c.ex &= live;
    c.eyR &= live;
    c.ezR &= live;
    return c;
}

// Apply one step's writes landing in our row: oz / oy say whether our row is
// the second slice / second row of the step.  `tail` selects the bit-0-of-
// word-k+1 pass (writes to our cell 31 only).
DOL_HD void apply3(Planes3& p, const Cube3& c, int kind, int oz, int oy, bool tail)
{
    const int vy = 1 - 2 * oy, vz = 1 - 2 * oz;
    const uint32_t selz_all = 0xFFFFFFFFu;
    auto selz = [&](uint32_t bits) { return oz ? bits : ~bits; };
    auto sely = [&](uint32_t bits) { return oy ? bits : ~bits; };
    // R-type writes hit cell b, L-type cell b-1 (shift right by one).  In the
    // tail pass only L-type writes from bit 0 matter; they land in cell 31.
    auto R = [&](uint32_t sel) { return tail ? 0u : sel; };
    auto L = [&](uint32_t sel) { return tail ? ((sel & 1u) << 31) : (sel >> 1); };
    (void)selz_all;

    if (kind == kFull) {
        uint32_t mine = c.corner & selz(c.fz) & sely(c.fy);
        put3(p, R(mine & c.fx) & p.mx, -1, vy, vz);
        put3(p, L(mine & ~c.fx) & p.mx, +1, vy, vz);
        uint32_t m2 = c.fxx & selz(c.eyR) & sely(c.ezR);
        put3(p, R(m2) & diag_ok(p), 0, vy, vz);
    }
    if ((kind == kFull || kind == kLastRowOfPair) && oy == 0) {
        uint32_t m = c.fy & selz(c.ex);
        put3(p, R(m & c.ez) & diag_ok(p), -1, 0, vz);
        put3(p, L(m & ~c.ez) & diag_ok(p), +1, 0, vz);
    }
    if ((kind == kFull || kind == kLastSlice) && oz == 0) {
        uint32_t m = c.fz & sely(c.ex);
        put3(p, R(m & c.ey) & diag_ok(p), -1, vy, 0);
        put3(p, L(m & ~c.ey) & diag_ok(p), +1, vy, 0);
    }
    if (oz == 0 && oy == 0) {   // x edges, every kind
        put3(p, R(c.ex), -1, 0, 0);
        put3(p, L(c.ex), +1, 0, 0);
    }
    if ((kind == kFull || kind == kLastSlice) && oz == 0) put3(p, R(c.eyR), 0, vy, 0);
    if ((kind == kFull || kind == kLastRowOfPair) && oy == 0) put3(p, R(c.ezR), 0, 0, vz);
}

DOL_HD void step3(Planes3& p, int w, int kind, const uint32_t* r00, const uint32_t* r01, const uint32_t* r10,
                  const uint32_t* r11, int k, int oz, int oy)
{
    apply3(p, cube3(w, kind, r00, r01, r10, r11, k), kind, oz, oy, false);
    if (32 * (k + 1) < w) apply3(p, cube3(w, kind, r00, r01, r10, r11, k + 1), kind, oz, oy, true);
}

// Final border-init planes of word k of row y of slice z.
DOL_HD Planes3 border3_word(int w, int h, int d, const uint32_t* mask, int z, int y, int k)
{
    const int ws = words_per_row(w);
    const size_t ss = (size_t)ws * h;
    Planes3 p{0xFFFFFFFFu, 0, 0, 0, 0, 0, 0};
    auto row = [&](int zz, int yy) { return mask + (size_t)zz * ss + (size_t)yy * ws; };

    // slice pairs (z-1, z) then (z, z+1): rows pairs (y-1, y) then (y, y+1) or the pair's last row
    for (int oz = 1; oz >= 0; oz--) {
        int z0 = z - oz;
        if (z0 < 0) continue;
        if (z0 + 1 < d) {
            for (int oy = 1; oy >= 0; oy--) {
                int y0 = y - oy;
                if (y0 < 0) continue;
                if (y0 + 1 < h)
                    step3(p, w, kFull, row(z0, y0), row(z0, y0 + 1), row(z0 + 1, y0), row(z0 + 1, y0 + 1), k, oz, oy);
                else
                    step3(p, w, kLastRowOfPair, row(z0, y0), nullptr, row(z0 + 1, y0), nullptr, k, oz, 0);
            }
        } else if (oz == 0) {
            // the last slice, after every slice pair
            for (int oy = 1; oy >= 0; oy--) {
                int y0 = y - oy;
                if (y0 < 0) continue;
                if (y0 + 1 < h)
                    step3(p, w, kLastSlice, row(z0, y0), row(z0, y0 + 1), nullptr, nullptr, k, 0, oy);
                else
                    step3(p, w, kLastRow, row(z0, y0), nullptr, nullptr, nullptr, k, 0, 0);
            }
        }
    }
    return p;
}

DOL_HD C3 decode3(const Planes3& p, int b)
{
    if (p.mx >> b & 1u) return C3{kMax3, kMax3, kMax3};
    int x = (p.xn >> b & 1u) ? ((p.xs >> b & 1u) ? -1 : 1) : 0;
    int y = (p.yn >> b & 1u) ? ((p.ys >> b & 1u) ? -1 : 1) : 0;
    int z = (p.zn >> b & 1u) ? ((p.zs >> b & 1u) ? -1 : 1) : 0;
    return C3{x, y, z};
}

}  // namespace dolk
