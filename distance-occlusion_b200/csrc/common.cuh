// common.cuh -- cell types and the comparison rule shared by every kernel.
//
// A 2D cell is the reference's cCellDelta2 (int16 x, y; 4 bytes) and a 3D cell
// its cCellDelta3 (int16 x, y, z; 6 bytes).  In registers a cell is kept as
// sign-extended ints.  Arithmetic on a component is stored back through int16
// truncation, and squared lengths are summed in 32-bit two's complement, which
// is what the reference's `Closer` (DistanceOcclusionLib.cpp:624-630,
// :2177-2183) compiles to; the wrap matters only for the max sentinel
// (32767 + cw wraps to -32768), and reproducing it keeps results bit-exact.
#pragma once

#include <stddef.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define DOL_HD __host__ __device__ __forceinline__
#else
#define DOL_HD inline
#endif

namespace dolk {

constexpr int kMax2 = 32767;   // kMaxDelta2
constexpr int kMax3 = 25000;   // kMaxDelta3

DOL_HD int trunc16(int v) { return (int)(int16_t)v; }

struct C2 {
    int x, y;
};
struct C3 {
    int x, y, z;
};

DOL_HD int32_t len(C2 c) { return (int32_t)((uint32_t)(c.x * c.x) + (uint32_t)(c.y * c.y)); }
DOL_HD int32_t len(C3 c)
{
    return (int32_t)((uint32_t)(c.x * c.x) + (uint32_t)(c.y * c.y) + (uint32_t)(c.z * c.z));
}

// offsets with int16 truncation
DOL_HD C2 add(C2 c, int dx, int dy) { return C2{trunc16(c.x + dx), trunc16(c.y + dy)}; }
DOL_HD C3 add(C3 c, int dx, int dy, int dz) { return C3{trunc16(c.x + dx), trunc16(c.y + dy), trunc16(c.z + dz)}; }
DOL_HD C2 addx(C2 c, int dx) { return C2{trunc16(c.x + dx), c.y}; }
DOL_HD C3 addx(C3 c, int dx) { return C3{trunc16(c.x + dx), c.y, c.z}; }

// the incumbent keeps ties: cand wins only when strictly shorter
DOL_HD C2 closer(C2 cur, C2 cand) { return len(cur) > len(cand) ? cand : cur; }
DOL_HD C3 closer(C3 cur, C3 cand) { return len(cur) > len(cand) ? cand : cur; }

DOL_HD bool same(C2 a, C2 b) { return a.x == b.x && a.y == b.y; }
DOL_HD bool same(C3 a, C3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// packed 2D cell: low half x, high half y (little-endian cCellDelta2)
DOL_HD C2 unpack2(uint32_t u) { return C2{(int)(int16_t)(u & 0xFFFFu), (int)(int16_t)(u >> 16)}; }
DOL_HD uint32_t pack2(C2 c) { return ((uint32_t)(uint16_t)c.x) | ((uint32_t)(uint16_t)c.y << 16); }

DOL_HD int words_per_row(int w) { return (w + 31) >> 5; }

// bits of mask word k that address cells < w
DOL_HD uint32_t live_bits(int w, int k)
{
    int n = w - 32 * k;
    return n >= 32 ? 0xFFFFFFFFu : (n <= 0 ? 0u : ((1u << n) - 1u));
}

// the word seen one cell to the left: bit b holds cell 32k+b-1; at x = 0 the
// cell repeats itself (the reference's "lastBit" seeding)
DOL_HD uint32_t left_word(const uint32_t* row, int k)
{
    uint32_t cur = row[k];
    uint32_t carry = k > 0 ? (row[k - 1] >> 31) : (cur & 1u);
    return (cur << 1) | carry;
}

}  // namespace dolk
