/*
 * dol_oracle.c -- CPU restatement of DistanceOcclusionLib's distance path.
 *
 * TEST INFRASTRUCTURE ONLY (see dol_oracle.h): the checker for the CUDA
 * library, never part of it.
 *
 * Integer edge behaviour follows what the reference compiles to: a delta
 * component is stored through int16 truncation (so 32767 + 1 wraps to -32768)
 * and squared lengths are summed in 32-bit two's complement.  The sums are
 * done in uint32 here so that the wrap is defined behaviour in C.
 */
#include "dol_oracle.h"

#include <float.h>
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

typedef int16_t i16;

/* ---- small helpers ----------------------------------------------------- */

static int words_per_row(int w) { return (w + 31) / 32; }

int dolo_mask_words(int w, int h, int d) { return words_per_row(w) * h * (d > 0 ? d : 1); }

/* squared length as the reference's Closer() sees it (int, wrapping) */
static inline int32_t len2(int x, int y) { return (int32_t)((uint32_t)(x * x) + (uint32_t)(y * y)); }
static inline int32_t len3(int x, int y, int z)
{
    return (int32_t)((uint32_t)(x * x) + (uint32_t)(y * y) + (uint32_t)(z * z));
}

/* candidate (cx,cy) replaces *c when strictly shorter: Closer(), :624-630 */
static inline void offer2(i16* c, int cx, int cy)
{
    i16 nx = (i16)cx, ny = (i16)cy;
    if (len2(c[0], c[1]) > len2(nx, ny)) { c[0] = nx; c[1] = ny; }
}
/* 3D Closer(), :2177-2183 */
static inline void offer3(i16* c, int cx, int cy, int cz)
{
    i16 nx = (i16)cx, ny = (i16)cy, nz = (i16)cz;
    if (len3(c[0], c[1], c[2]) > len3(nx, ny, nz)) { c[0] = nx; c[1] = ny; c[2] = nz; }
}

static inline void set2(i16* c, int x, int y) { c[0] = (i16)x; c[1] = (i16)y; }
static inline void set3(i16* c, int x, int y, int z) { c[0] = (i16)x; c[1] = (i16)y; c[2] = (i16)z; }

/* LCG of DistanceOcclusionLib.cpp:28-32: returns floor(seed' * limit / 2^32) */
static int lcg_pick(uint32_t* s, int limit)
{
    *s = *s * 1103515245u + 12345u;
    return (int)(((uint64_t)(*s) * (uint64_t)(int64_t)limit) >> 32);
}

/* ---- generators ---------------------------------------------------------- */

void dolo_add_points_2d(int w, int h, int n, uint32_t seed, uint32_t* mask)
{
    /* DistanceOcclusionLib.cpp:95-113: x then y from the LCG */
    int ws = words_per_row(w);
    for (int k = 0; k < n; k++) {
        int x = lcg_pick(&seed, w);
        int y = lcg_pick(&seed, h);
        mask[y * ws + (x >> 5)] |= 1u << (x & 31);
    }
}

void dolo_add_points_3d(int w, int h, int d, int n, uint32_t seed, uint32_t* mask)
{
    /* DistanceOcclusionLib.cpp:1224-1244: x, y, z */
    int ws = words_per_row(w);
    for (int k = 0; k < n; k++) {
        int x = lcg_pick(&seed, w);
        int y = lcg_pick(&seed, h);
        int z = lcg_pick(&seed, d);
        mask[((size_t)z * h + y) * ws + (x >> 5)] |= 1u << (x & 31);
    }
}

/* fill cells [x0,x1] x [y0,y1] of one slice: FillMaskBlock, :131-156 */
static void fill_rect(int ws, int x0, int x1, int y0, int y1, uint32_t* slice)
{
    int wa = x0 / 32, wb = x1 / 32;
    uint32_t lo = ~((1u << (x0 - wa * 32)) - 1u);            /* bits >= x0 */
    uint32_t hb = 1u << (x1 - wb * 32);
    uint32_t hi = hb | (hb - 1u);                              /* bits <= x1 */
    if (wa == wb) { lo &= hi; hi = 0; }
    for (int y = y0; y <= y1; y++) {
        uint32_t* row = slice + (size_t)y * ws;
        row[wa] |= lo;
        for (int k = wa + 1; k < wb; k++) row[k] = ~0u;
        row[wb] |= hi;
    }
}

void dolo_add_block_2d(int w, int h, int sides, uint32_t* mask)
{
    /* :159-179 */
    int x0 = w / 4, x1 = x0 + w / 2 - 1, y0 = h / 3, y1 = y0 + h / 3 - 1;
    int ws = words_per_row(w);
    if (sides > 4) { fill_rect(ws, x0, x1, y0, y1, mask); return; }
    if (sides > 0) fill_rect(ws, x0, x1, y0, y0, mask);
    if (sides > 1) fill_rect(ws, x0, x0, y0, y1, mask);
    if (sides > 2) fill_rect(ws, x0, x1, y1, y1, mask);
    if (sides > 3) fill_rect(ws, x1, x1, y0, y1, mask);
}

static void fill_box(int ws, int h, int x0, int x1, int y0, int y1, int z0, int z1, uint32_t* mask)
{
    for (int z = z0; z <= z1; z++) fill_rect(ws, x0, x1, y0, y1, mask + (size_t)z * ws * h);
}

void dolo_add_block_3d(int w, int h, int d, int sides, uint32_t* mask)
{
    /* :1259-1287 */
    int ws = words_per_row(w);
    int x0 = w / 4, x1 = x0 + w / 2 - 1;
    int y0 = h / 3, y1 = y0 + h / 3 - 1;
    int z0 = d / 3, z1 = z0 + d / 3 - 1;
    if (sides > 6) { fill_box(ws, h, x0, x1, y0, y1, z0, z1, mask); return; }
    if (sides > 0) fill_box(ws, h, x0, x1, y0, y1, z0, z0, mask);
    if (sides > 1) fill_box(ws, h, x0, x0, y0, y1, z0, z1, mask);
    if (sides > 2) fill_box(ws, h, x0, x1, y0, y0, z0, z1, mask);
    if (sides > 3) fill_box(ws, h, x1, x1, y0, y1, z0, z1, mask);
    if (sides > 4) fill_box(ws, h, x0, x1, y1, y1, z0, z1, mask);
    if (sides > 5) fill_box(ws, h, x0, x1, y0, y1, z1, z1, mask);
}

void dolo_pack_bytes(int w, int h, const uint8_t* img, int threshold, int less_than, uint32_t* mask)
{
    /* DistanceOcclusionTool.cpp:646-665: bit set iff (v >= threshold) ^ lessThan */
    int ws = words_per_row(w);
    for (int y = 0; y < h; y++)
        for (int k = 0; k < ws; k++) {
            uint32_t word = 0;
            for (int b = 0; b < 32 && 32 * k + b < w; b++) {
                int v = img[(size_t)y * w + 32 * k + b];
                if ((v >= threshold) != (less_than != 0)) word |= 1u << b;
            }
            mask[(size_t)y * ws + k] = word;
        }
}

/* ---- plain initialisation ---------------------------------------------- */

static inline int mask_bit(const uint32_t* row, int x) { return (row[x >> 5] >> (x & 31)) & 1; }

void dolo_init_distances_2d(int w, int h, const uint32_t* mask, float* dist, float max_d)
{
    /* InitFromBitMask<float>, :183-222 */
    int ws = words_per_row(w);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++)
            dist[(size_t)y * w + x] = mask_bit(mask + (size_t)y * ws, x) ? 0.0f : max_d;
}

void dolo_init_distances_2d_i16(int w, int h, const uint32_t* mask, i16* dist, i16 max_d)
{
    /* InitFromBitMask<int16_t>, :183-222 */
    int ws = words_per_row(w);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++)
            dist[(size_t)y * w + x] = mask_bit(mask + (size_t)y * ws, x) ? 0 : max_d;
}

void dolo_init_distances_2d_i32(int w, int h, const uint32_t* mask, int32_t* dist, int32_t max_d)
{
    /* InitFromBitMask<int32_t>, :183-222 */
    int ws = words_per_row(w);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++)
            dist[(size_t)y * w + x] = mask_bit(mask + (size_t)y * ws, x) ? 0 : max_d;
}

/* Chamfer 3-4 (Borgefors), :916-1004.  One raster pass down the rows (row 0:
 * left neighbour only; other rows: the three cells above, then the left
 * neighbour) and one pass up (mirrored).  A cell takes a neighbour's value plus
 * 3 (edge) or 4 (diagonal) when that is smaller.  Sums are int (int16 values
 * are promoted, so they never wrap); int32 sums wrap as two's complement, which
 * is what the reference's build does past INT32_MAX (done here in uint32 to
 * stay defined).  Rows of one cell are not handled (the reference reads
 * outside the row there).  Returns the multiplier 3. */
#define CHAMFER_BODY(T, ADD)                                                               \
    const int d0 = 3, d1 = 4;                                                              \
    T* row0 = dist;                                                                        \
    for (int x = 1; x < w; x++)                                                            \
        if (row0[x] > ADD(row0[x - 1], d0)) row0[x] = (T)ADD(row0[x - 1], d0);             \
    for (int y = 1; y < h; y++) {                                                          \
        T* row1 = row0 + w;                                                                \
        if (row1[0] > ADD(row0[0], d0)) row1[0] = (T)ADD(row0[0], d0);                     \
        if (row1[0] > ADD(row0[1], d1)) row1[0] = (T)ADD(row0[1], d1);                     \
        for (int x = 1; x < w - 1; x++) {                                                  \
            if (row1[x] > ADD(row0[x - 1], d1)) row1[x] = (T)ADD(row0[x - 1], d1);         \
            if (row1[x] > ADD(row0[x], d0)) row1[x] = (T)ADD(row0[x], d0);                 \
            if (row1[x] > ADD(row0[x + 1], d1)) row1[x] = (T)ADD(row0[x + 1], d1);         \
            if (row1[x] > ADD(row1[x - 1], d0)) row1[x] = (T)ADD(row1[x - 1], d0);         \
        }                                                                                  \
        if (row1[w - 1] > ADD(row0[w - 2], d1)) row1[w - 1] = (T)ADD(row0[w - 2], d1);     \
        if (row1[w - 1] > ADD(row0[w - 1], d0)) row1[w - 1] = (T)ADD(row0[w - 1], d0);     \
        if (row1[w - 1] > ADD(row1[w - 2], d0)) row1[w - 1] = (T)ADD(row1[w - 2], d0);     \
        row0 = row1;                                                                       \
    }                                                                                      \
    row0 = dist + (size_t)h * w - w;                                                       \
    for (int x = w - 2; x >= 0; x--)                                                       \
        if (row0[x] > ADD(row0[x + 1], d0)) row0[x] = (T)ADD(row0[x + 1], d0);             \
    for (int y = h - 2; y >= 0; y--) {                                                     \
        T* row1 = row0 - w;                                                                \
        if (row1[w - 1] > ADD(row0[w - 1], d0)) row1[w - 1] = (T)ADD(row0[w - 1], d0);     \
        if (row1[w - 1] > ADD(row0[w - 2], d1)) row1[w - 1] = (T)ADD(row0[w - 2], d1);     \
        for (int x = w - 2; x > 0; x--) {                                                  \
            if (row1[x] > ADD(row0[x + 1], d1)) row1[x] = (T)ADD(row0[x + 1], d1);         \
            if (row1[x] > ADD(row0[x], d0)) row1[x] = (T)ADD(row0[x], d0);                 \
            if (row1[x] > ADD(row0[x - 1], d1)) row1[x] = (T)ADD(row0[x - 1], d1);         \
            if (row1[x] > ADD(row1[x + 1], d0)) row1[x] = (T)ADD(row1[x + 1], d0);         \
        }                                                                                  \
        if (row1[0] > ADD(row0[1], d1)) row1[0] = (T)ADD(row0[1], d1);                     \
        if (row1[0] > ADD(row0[0], d0)) row1[0] = (T)ADD(row0[0], d0);                     \
        if (row1[0] > ADD(row1[1], d0)) row1[0] = (T)ADD(row1[1], d0);                     \
        row0 = row1;                                                                       \
    }                                                                                      \
    return d0;

#define ADD16(a, b) ((int)(a) + (b))
#define ADD32(a, b) ((int32_t)((uint32_t)(a) + (uint32_t)(b)))

int dolo_chamfer_2d_i16(int w, int h, i16* dist) { CHAMFER_BODY(i16, ADD16) }
int dolo_chamfer_2d_i32(int w, int h, int32_t* dist) { CHAMFER_BODY(int32_t, ADD32) }

void dolo_init_deltas_2d(int w, int h, const uint32_t* mask, i16* deltas, int invert)
{
    /* :224-254 -- zero where (bit ^ invert), kMaxDelta2 elsewhere */
    int ws = words_per_row(w);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int on = mask_bit(mask + (size_t)y * ws, x) ^ (invert ? 1 : 0);
            i16 v = on ? 0 : DOLO_MAX2;
            set2(deltas + 2 * ((size_t)y * w + x), v, v);
        }
}

void dolo_init_deltas_3d(int w, int h, int d, const uint32_t* mask, i16* deltas, int invert)
{
    /* :1289-1321 */
    int ws = words_per_row(w);
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                int on = mask_bit(mask + ((size_t)z * h + y) * ws, x) ^ (invert ? 1 : 0);
                i16 v = on ? 0 : DOLO_MAX3;
                set3(deltas + 3 * (((size_t)z * h + y) * w + x), v, v, v);
            }
}

/* ---- signed border initialisation, 2D ------------------------------------
 * SetBorderCellsCombo, DistanceOcclusionLib.cpp:504-599.  The result depends
 * on the order of the writes (later writes win; diagonals only land in cells
 * still at max), so the walk below keeps the reference's order exactly:
 * row pairs top to bottom, words left to right, and in each word the diagonal
 * writes, then the x-edge writes, then the y-edge writes, each in ascending
 * bit order.  Bits at x >= w are ignored.  The shifted word carries the
 * previous cell's bit; at x = 0 it repeats cell 0, so no edge is seen there.
 */

/* bits of word k that address cells < w */
static uint32_t live_bits(int w, int k)
{
    int n = w - 32 * k;
    return n >= 32 ? ~0u : ((1u << n) - 1u);
}

/* the x-edge writes of one word of one row: a change between cells x-1 and
 * x gives x-1 the delta (+1,0) and x the delta (-1,0) (:557-561, :585-590) */
static void x_edges_2d(uint32_t bits, int base, i16* row)
{
    for (int b = 0; b < 32; b++)
        if (bits >> b & 1) {
            set2(row + 2 * (base + b - 1), +1, 0);
            set2(row + 2 * (base + b), -1, 0);
        }
}

void dolo_border_init_2d(int w, int h, const uint32_t* mask, i16* deltas)
{
    for (size_t c = 0; c < (size_t)w * h; c++) set2(deltas + 2 * c, DOLO_MAX2, DOLO_MAX2);

    int ws = words_per_row(w);
    for (int y = 0; y + 1 < h; y++) {
        const uint32_t* top = mask + (size_t)y * ws;
        const uint32_t* bot = top + ws;
        i16* dtop = deltas + 2 * (size_t)y * w;
        i16* dbot = dtop + 2 * (size_t)w;
        uint32_t ct = top[0] & 1u, cb = bot[0] & 1u;          /* carried bit of cell x-1 */
        for (int k = 0; k < ws; k++) {
            uint32_t t = top[k], b = bot[k];
            uint32_t tl = (t << 1) | ct, bl = (b << 1) | cb;   /* cell x-1 */
            ct = t >> 31; cb = b >> 31;
            uint32_t live = live_bits(w, k);
            uint32_t yedge = (t ^ b) & live;                   /* change between rows at x   */
            uint32_t xedge = (t ^ tl) & live;                  /* change along the top row   */
            uint32_t yedgel = tl ^ bl;                         /* change between rows at x-1 */
            uint32_t diag = (yedge ^ yedgel) & live;
            int base = 32 * k;

            for (int bi = 0; bi < 32; bi++)
                if (diag >> bi & 1) {
                    int sx = (int)(yedgel >> bi & 1), sy = (int)(xedge >> bi & 1);
                    i16* c = (sy ? dbot : dtop) + 2 * (base + bi + sx - 1);
                    if (c[0] == DOLO_MAX2) set2(c, 1 - 2 * sx, 1 - 2 * sy);
                }
            x_edges_2d(xedge, base, dtop);
            for (int bi = 0; bi < 32; bi++)
                if (yedge >> bi & 1) {
                    set2(dtop + 2 * (base + bi), 0, +1);
                    set2(dbot + 2 * (base + bi), 0, -1);
                }
        }
    }
    /* last row: x edges only (:573-597) */
    {
        const uint32_t* row = mask + (size_t)(h - 1) * ws;
        i16* drow = deltas + 2 * (size_t)(h - 1) * w;
        uint32_t cr = row[0] & 1u;
        for (int k = 0; k < ws; k++) {
            uint32_t r = row[k];
            uint32_t rl = (r << 1) | cr;
            cr = r >> 31;
            x_edges_2d((r ^ rl) & live_bits(w, k), 32 * k, drow);
        }
    }
}

/* ---- signed border initialisation, 3D ------------------------------------
 * SetBorderCellsCombo, DistanceOcclusionLib.cpp:1820-2150.  Same ordering rule
 * as 2D.  For each slice pair (z,z+1) and row pair (y,y+1) a word is looked at
 * as a 2x2x2 cube of cells: x-1 ("L") and x ("R"), rows y/y+1, slices z/z+1.
 * Within a word the groups run: box corners, x-face diagonals, y-face
 * diagonals, z-face diagonals, x edges, y edges, z edges.  Diagonal groups
 * only overwrite cells at max or cells already holding a diagonal
 * (|x|+|y|+|z| > 1); box corners only cells at max.  Then the last row of each
 * slice pair (y-face diagonals, x edges, z edges), then the last slice (z-face
 * diagonals, x edges, y edges per row pair, and x edges on its last row).
 */

typedef struct {
    i16* row[2][2];   /* [slice offset][row offset] -> first cell of that row */
} cube_rows;

static inline i16* cell3(i16* row, int x) { return row + 3 * (size_t)x; }

static inline int may_take_diagonal(const i16* c)
{
    return c[0] == DOLO_MAX3 || (abs(c[0]) + abs(c[1]) + abs(c[2]) > 1);
}

/* x edges, :1967-1972 etc.: L gets (+1,0,0), R gets (-1,0,0) */
static void x_edges_3d(uint32_t bits, int base, i16* row)
{
    for (int b = 0; b < 32; b++)
        if (bits >> b & 1) {
            set3(cell3(row, base + b - 1), +1, 0, 0);
            set3(cell3(row, base + b), -1, 0, 0);
        }
}

/* y-face diagonals (corner in the x/z plane of row r), :1923-1936 */
static void yface_diagonals(uint32_t fy, uint32_t ez, uint32_t ex, int base, i16* r_z0, i16* r_z1)
{
    for (int b = 0; b < 32; b++)
        if (fy >> b & 1) {
            int sx = (int)(ez >> b & 1), sz = (int)(ex >> b & 1);
            i16* c = cell3(sz ? r_z1 : r_z0, base + b + sx - 1);
            if (may_take_diagonal(c)) set3(c, 1 - 2 * sx, 0, 1 - 2 * sz);
        }
}

/* z-face diagonals (corner in the x/y plane of slice s), :1938-1951 */
static void zface_diagonals(uint32_t fz, uint32_t ey, uint32_t ex, int base, i16* r_y0, i16* r_y1)
{
    for (int b = 0; b < 32; b++)
        if (fz >> b & 1) {
            int sx = (int)(ey >> b & 1), sy = (int)(ex >> b & 1);
            i16* c = cell3(sy ? r_y1 : r_y0, base + b + sx - 1);
            if (may_take_diagonal(c)) set3(c, 1 - 2 * sx, 1 - 2 * sy, 0);
        }
}

void dolo_border_init_3d(int w, int h, int d, const uint32_t* mask, i16* deltas)
{
    size_t n = (size_t)w * h * d;
    for (size_t c = 0; c < n; c++) set3(deltas + 3 * c, DOLO_MAX3, DOLO_MAX3, DOLO_MAX3);

    int ws = words_per_row(w);
    size_t mslice = (size_t)ws * h, dslice = (size_t)w * h;

    for (int z = 0; z + 1 < d; z++) {
        for (int y = 0; y + 1 < h; y++) {
            const uint32_t* m00 = mask + z * mslice + (size_t)y * ws;   /* slice z,   row y   */
            const uint32_t* m01 = m00 + ws;                             /* slice z,   row y+1 */
            const uint32_t* m10 = m00 + mslice;                         /* slice z+1, row y   */
            const uint32_t* m11 = m10 + ws;                             /* slice z+1, row y+1 */
            i16* r00 = deltas + 3 * (z * dslice + (size_t)y * w);
            i16* r01 = r00 + 3 * (size_t)w;
            i16* r10 = r00 + 3 * dslice;
            i16* r11 = r10 + 3 * (size_t)w;
            uint32_t c00 = m00[0] & 1u, c01 = m01[0] & 1u, c10 = m10[0] & 1u, c11 = m11[0] & 1u;

            for (int k = 0; k < ws; k++) {
                /* cube corners: L = cell x-1, R = cell x */
                uint32_t R000 = m00[k], R010 = m01[k], R100 = m10[k], R110 = m11[k];
                uint32_t L000 = (R000 << 1) | c00, L010 = (R010 << 1) | c01;
                uint32_t L100 = (R100 << 1) | c10, L110 = (R110 << 1) | c11;
                c00 = R000 >> 31; c01 = R010 >> 31; c10 = R100 >> 31; c11 = R110 >> 31;
                uint32_t live = live_bits(w, k);

                uint32_t ex = L000 ^ R000;       /* x change, row y, slice z     */
                uint32_t ey = L000 ^ L010;       /* y change at L, slice z       */
                uint32_t ez = L000 ^ L100;       /* z change at L, row y         */
                uint32_t ezR = R000 ^ R100;      /* z change at R, row y         */
                uint32_t eyL1 = L100 ^ L110;     /* y change at L, slice z+1     */
                uint32_t exY1 = L010 ^ R010;     /* x change, row y+1, slice z   */
                uint32_t eyR = R000 ^ R010;      /* y change at R, slice z       */
                uint32_t eyR1 = R100 ^ R110;     /* y change at R, slice z+1     */

                uint32_t fx = ey ^ eyL1;
                uint32_t fy = (ez ^ ezR) & live;
                uint32_t fz = (ex ^ exY1) & live;
                uint32_t fxx = (eyR ^ eyR1) & live;
                uint32_t corner = (fz ^ (eyL1 ^ eyR1)) & live;
                ex &= live; eyR &= live; ezR &= live;
                int base = 32 * k;

                for (int b = 0; b < 32; b++)
                    if (corner >> b & 1) {
                        int sx = (int)(fx >> b & 1), sy = (int)(fy >> b & 1), sz = (int)(fz >> b & 1);
                        i16* row = sz ? (sy ? r11 : r10) : (sy ? r01 : r00);
                        i16* c = cell3(row, base + b + sx - 1);
                        if (c[0] == DOLO_MAX3) set3(c, 1 - 2 * sx, 1 - 2 * sy, 1 - 2 * sz);
                    }
                for (int b = 0; b < 32; b++)
                    if (fxx >> b & 1) {
                        int sy = (int)(ezR >> b & 1), sz = (int)(eyR >> b & 1);
                        i16* row = sz ? (sy ? r11 : r10) : (sy ? r01 : r00);
                        i16* c = cell3(row, base + b);
                        if (may_take_diagonal(c)) set3(c, 0, 1 - 2 * sy, 1 - 2 * sz);
                    }
                yface_diagonals(fy, ez, ex, base, r00, r10);
                zface_diagonals(fz, ey, ex, base, r00, r01);
                x_edges_3d(ex, base, r00);
                for (int b = 0; b < 32; b++)
                    if (eyR >> b & 1) {
                        set3(cell3(r00, base + b), 0, +1, 0);
                        set3(cell3(r01, base + b), 0, -1, 0);
                    }
                for (int b = 0; b < 32; b++)
                    if (ezR >> b & 1) {
                        set3(cell3(r00, base + b), 0, 0, +1);
                        set3(cell3(r10, base + b), 0, 0, -1);
                    }
            }
        }
        /* last row of the slice pair: y-face diagonals, x edges, z edges (:2005-2065) */
        {
            int y = h - 1;
            const uint32_t* m00 = mask + z * mslice + (size_t)y * ws;
            const uint32_t* m10 = m00 + mslice;
            i16* r00 = deltas + 3 * (z * dslice + (size_t)y * w);
            i16* r10 = r00 + 3 * dslice;
            uint32_t c00 = m00[0] & 1u, c10 = m10[0] & 1u;
            for (int k = 0; k < ws; k++) {
                uint32_t R000 = m00[k], R100 = m10[k];
                uint32_t L000 = (R000 << 1) | c00, L100 = (R100 << 1) | c10;
                c00 = R000 >> 31; c10 = R100 >> 31;
                uint32_t live = live_bits(w, k);
                uint32_t ex = L000 ^ R000, ez = L000 ^ L100, ezR = R000 ^ R100;
                uint32_t fy = (ez ^ ezR) & live;
                ex &= live; ezR &= live;
                int base = 32 * k;
                yface_diagonals(fy, ez, ex, base, r00, r10);
                x_edges_3d(ex, base, r00);
                for (int b = 0; b < 32; b++)
                    if (ezR >> b & 1) {
                        set3(cell3(r00, base + b), 0, 0, +1);
                        set3(cell3(r10, base + b), 0, 0, -1);
                    }
            }
        }
    }

    /* last slice: z-face diagonals, x edges, y edges; then its last row (:2068-2150) */
    {
        int z = d - 1;
        for (int y = 0; y + 1 < h; y++) {
            const uint32_t* m00 = mask + z * mslice + (size_t)y * ws;
            const uint32_t* m01 = m00 + ws;
            i16* r00 = deltas + 3 * (z * dslice + (size_t)y * w);
            i16* r01 = r00 + 3 * (size_t)w;
            uint32_t c00 = m00[0] & 1u, c01 = m01[0] & 1u;
            for (int k = 0; k < ws; k++) {
                uint32_t R000 = m00[k], R010 = m01[k];
                uint32_t L000 = (R000 << 1) | c00, L010 = (R010 << 1) | c01;
                c00 = R000 >> 31; c01 = R010 >> 31;
                uint32_t live = live_bits(w, k);
                uint32_t ex = L000 ^ R000, ey = L000 ^ L010, eyR = R000 ^ R010;
                uint32_t fz = (ey ^ eyR) & live;
                ex &= live; eyR &= live;
                int base = 32 * k;
                zface_diagonals(fz, ey, ex, base, r00, r01);
                x_edges_3d(ex, base, r00);
                for (int b = 0; b < 32; b++)
                    if (eyR >> b & 1) {
                        set3(cell3(r00, base + b), 0, +1, 0);
                        set3(cell3(r01, base + b), 0, -1, 0);
                    }
            }
        }
        {
            int y = h - 1;
            const uint32_t* m00 = mask + z * mslice + (size_t)y * ws;
            i16* r00 = deltas + 3 * (z * dslice + (size_t)y * w);
            uint32_t c00 = m00[0] & 1u;
            for (int k = 0; k < ws; k++) {
                uint32_t R000 = m00[k];
                uint32_t L000 = (R000 << 1) | c00;
                c00 = R000 >> 31;
                x_edges_3d((L000 ^ R000) & live_bits(w, k), 32 * k, r00);
            }
        }
    }
}

/* ---- Danielsson ----------------------------------------------------------
 * 2D: DistanceOcclusionLib.cpp:702-778.  Down sweep over rows 1..h-1, then up
 * sweep over rows h-2..0; each row takes the neighbour row's delta with the
 * y offset, then a left-to-right x pass, then a right-to-left x pass.
 */

static void row_pull_2d(i16* cur, const i16* nb, int w, int dy)
{
    for (int i = 0; i < w; i++) offer2(cur + 2 * i, nb[2 * i], nb[2 * i + 1] + dy);
}

static void row_xpasses_2d(i16* r, int w, int cw)
{
    for (int i = 1; i < w; i++) offer2(r + 2 * i, r[2 * (i - 1)] - cw, r[2 * (i - 1) + 1]);
    for (int i = w - 2; i >= 0; i--) offer2(r + 2 * i, r[2 * (i + 1)] + cw, r[2 * (i + 1) + 1]);
}

void dolo_danielsson_2d(int w, int h, i16* deltas, int cw)
{
    for (int y = 1; y < h; y++) {
        i16* r = deltas + 2 * (size_t)y * w;
        row_pull_2d(r, r - 2 * (size_t)w, w, -cw);
        row_xpasses_2d(r, w, cw);
    }
    for (int y = h - 2; y >= 0; y--) {
        i16* r = deltas + 2 * (size_t)y * w;
        row_pull_2d(r, r + 2 * (size_t)w, w, +cw);
        row_xpasses_2d(r, w, cw);
    }
}

/* 3D: DanielssonSlice :2264-2345 and Danielsson :2348-2394 */
static void row_pull_3d(i16* cur, const i16* nb, int n, int dy, int dz)
{
    for (int i = 0; i < n; i++) offer3(cur + 3 * i, nb[3 * i], nb[3 * i + 1] + dy, nb[3 * i + 2] + dz);
}

static void row_xpasses_3d(i16* r, int w, int cw)
{
    for (int i = 1; i < w; i++) {
        const i16* p = r + 3 * (i - 1);
        offer3(r + 3 * i, p[0] - cw, p[1], p[2]);
    }
    for (int i = w - 2; i >= 0; i--) {
        const i16* p = r + 3 * (i + 1);
        offer3(r + 3 * i, p[0] + cw, p[1], p[2]);
    }
}

static void slice_danielsson_3d(i16* s, int w, int h, int cw)
{
    for (int y = 1; y < h; y++) {
        i16* r = s + 3 * (size_t)y * w;
        row_pull_3d(r, r - 3 * (size_t)w, w, -cw, 0);
        row_xpasses_3d(r, w, cw);
    }
    for (int y = h - 2; y >= 0; y--) {
        i16* r = s + 3 * (size_t)y * w;
        row_pull_3d(r, r + 3 * (size_t)w, w, +cw, 0);
        row_xpasses_3d(r, w, cw);
    }
}

void dolo_danielsson_3d(int w, int h, int d, i16* deltas, int cw)
{
    size_t ss = (size_t)w * h;
    for (int z = 1; z < d; z++) {
        i16* s = deltas + 3 * z * ss;
        row_pull_3d(s, s - 3 * ss, (int)ss, 0, -cw);
        slice_danielsson_3d(s, w, h, cw);
    }
    for (int z = d - 2; z >= 0; z--) {
        i16* s = deltas + 3 * z * ss;
        row_pull_3d(s, s + 3 * ss, (int)ss, 0, +cw);
        slice_danielsson_3d(s, w, h, cw);
    }
}

/* ---- FastSweep -------------------------------------------------------------
 * 2D: DistanceOcclusionLib.cpp:633-697.  Four quadrant sweeps (x direction
 * bit 0, y direction bit 1 of the sweep index).  The first row of each sweep
 * is left as is.  Each later row first takes the previous row's delta, then
 * walks along x taking the previous cell of this row and then the diagonal
 * cell of the previous row.
 */
void dolo_fastsweep_2d(int w, int h, i16* deltas, int cw)
{
    for (int s = 0; s < 4; s++) {
        int dx = (s & 1) ? -1 : 1, dy = (s & 2) ? -1 : 1;
        int ox = -cw * dx, oy = -cw * dy;
        int x0 = (dx > 0) ? 0 : w - 1;
        int y0 = (dy > 0) ? 0 : h - 1;
        for (int t = 1; t < h; t++) {
            i16* prev = deltas + 2 * (size_t)(y0 + (t - 1) * dy) * w;
            i16* cur = deltas + 2 * (size_t)(y0 + t * dy) * w;
            for (int u = 0; u < w; u++) {
                int x = x0 + u * dx;
                offer2(cur + 2 * x, prev[2 * x], prev[2 * x + 1] + oy);
            }
            for (int u = 1; u < w; u++) {
                int x = x0 + u * dx, xp = x - dx;
                offer2(cur + 2 * x, cur[2 * xp] + ox, cur[2 * xp + 1]);
                offer2(cur + 2 * x, prev[2 * xp] + ox, prev[2 * xp + 1] + oy);
            }
        }
    }
}

/* 3D: :2186-2260.  Eight octant sweeps (x bit 0, y bit 1, z bit 2).  The first
 * slice and the first row of every slice are left as is; each later row
 * takes the previous slice's cell, then the previous row's cell, then walks
 * along x taking the previous cell. */
void dolo_fastsweep_3d(int w, int h, int d, i16* deltas, int cw)
{
    size_t ss = (size_t)w * h;
    for (int s = 0; s < 8; s++) {
        int dx = (s & 1) ? -1 : 1, dy = (s & 2) ? -1 : 1, dz = (s & 4) ? -1 : 1;
        int ox = -cw * dx, oy = -cw * dy, oz = -cw * dz;
        int x0 = (dx > 0) ? 0 : w - 1, y0 = (dy > 0) ? 0 : h - 1, z0 = (dz > 0) ? 0 : d - 1;
        for (int tz = 1; tz < d; tz++) {
            i16* sprev = deltas + 3 * (size_t)(z0 + (tz - 1) * dz) * ss;
            i16* scur = deltas + 3 * (size_t)(z0 + tz * dz) * ss;
            for (int ty = 1; ty < h; ty++) {
                size_t ry = (size_t)(y0 + ty * dy) * w, rp = (size_t)(y0 + (ty - 1) * dy) * w;
                i16* cur = scur + 3 * ry;
                const i16* zprev = sprev + 3 * ry;
                const i16* yprev = scur + 3 * rp;
                for (int u = 0; u < w; u++) {
                    int x = x0 + u * dx;
                    offer3(cur + 3 * x, zprev[3 * x], zprev[3 * x + 1], zprev[3 * x + 2] + oz);
                    offer3(cur + 3 * x, yprev[3 * x], yprev[3 * x + 1] + oy, yprev[3 * x + 2]);
                }
                for (int u = 1; u < w; u++) {
                    int x = x0 + u * dx, xp = x - dx;
                    offer3(cur + 3 * x, cur[3 * xp] + ox, cur[3 * xp + 1], cur[3 * xp + 2]);
                }
            }
        }
    }
}

/* ---- JumpFlood --------------------------------------------------------------
 * 2D pass :782-873 with the fixed neighbour order (x-s, x-s/y-s, x-s/y+s, x+s,
 * x+s/y-s, x+s/y+s, y-s, y+s); no skip of max cells.  Driver :887-908: steps
 * from FloorPow2(max dim - 1) down to 1, ping-pong, then one more step-1 pass
 * back into the caller's buffer if the last result sits in the temporary.
 */
static int floor_pow2(int v)
{
    /* FloorPow2, :875-884 */
    v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    return (v + 1) >> 1;
}

static void jfa_pass_2d(int s, int w, int h, const i16* in, i16* out, int cw)
{
    int o = cw * s;
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            i16 best[2];
            const i16* self = in + 2 * ((size_t)y * w + x);
            best[0] = self[0]; best[1] = self[1];
#define AT(xx, yy) (in + 2 * ((size_t)(yy) * w + (xx)))
            if (x - s >= 0) {
                offer2(best, AT(x - s, y)[0] - o, AT(x - s, y)[1]);
                if (y - s >= 0) offer2(best, AT(x - s, y - s)[0] - o, AT(x - s, y - s)[1] - o);
                if (y + s < h) offer2(best, AT(x - s, y + s)[0] - o, AT(x - s, y + s)[1] + o);
            }
            if (x + s < w) {
                offer2(best, AT(x + s, y)[0] + o, AT(x + s, y)[1]);
                if (y - s >= 0) offer2(best, AT(x + s, y - s)[0] + o, AT(x + s, y - s)[1] - o);
                if (y + s < h) offer2(best, AT(x + s, y + s)[0] + o, AT(x + s, y + s)[1] + o);
            }
            if (y - s >= 0) offer2(best, AT(x, y - s)[0], AT(x, y - s)[1] - o);
            if (y + s < h) offer2(best, AT(x, y + s)[0], AT(x, y + s)[1] + o);
#undef AT
            i16* dst = out + 2 * ((size_t)y * w + x);
            dst[0] = best[0]; dst[1] = best[1];
        }
}

void dolo_jumpflood_2d(int w, int h, i16* deltas, int cw, i16* temp)
{
    i16* a = deltas;
    i16* b = temp;
    for (int s = floor_pow2((w >= h ? w : h) - 1); s > 0; s /= 2) {
        jfa_pass_2d(s, w, h, a, b, cw);
        i16* t = a; a = b; b = t;
    }
    if (a != deltas) jfa_pass_2d(1, w, h, a, deltas, cw);
}

/* 3D pass :2398-2447: all 27 offsets (z outer, then y, then x; each -s, 0, +s
 * where in range), skipping neighbours whose stored x is kMaxDelta3.
 * Driver :2450-2472. */
static void jfa_pass_3d(int s, int w, int h, int d, const i16* in, i16* out, int cw)
{
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                size_t idx = ((size_t)z * h + y) * w + x;
                i16 best[3];
                best[0] = in[3 * idx]; best[1] = in[3 * idx + 1]; best[2] = in[3 * idx + 2];
                for (int kz = (z - s >= 0 ? -s : 0); kz <= (z + s < d ? s : 0); kz += s)
                    for (int ky = (y - s >= 0 ? -s : 0); ky <= (y + s < h ? s : 0); ky += s)
                        for (int kx = (x - s >= 0 ? -s : 0); kx <= (x + s < w ? s : 0); kx += s) {
                            const i16* c = in + 3 * (((size_t)(z + kz) * h + (y + ky)) * w + (x + kx));
                            if (c[0] == DOLO_MAX3) continue;
                            offer3(best, c[0] + cw * kx, c[1] + cw * ky, c[2] + cw * kz);
                        }
                out[3 * idx] = best[0]; out[3 * idx + 1] = best[1]; out[3 * idx + 2] = best[2];
            }
}

void dolo_jumpflood_3d(int w, int h, int d, i16* deltas, int cw, i16* temp)
{
    int m = w >= h ? w : h;
    m = m >= d ? m : d;
    i16* a = deltas;
    i16* b = temp;
    for (int s = floor_pow2(m - 1); s > 0; s /= 2) {
        jfa_pass_3d(s, w, h, d, a, b, cw);
        i16* t = a; a = b; b = t;
    }
    if (a != deltas) jfa_pass_3d(1, w, h, d, a, deltas, cw);
}

/* ---- BruteForce ------------------------------------------------------------ */

void dolo_bruteforce_2d(int w, int h, i16* deltas, int cw)
{
    /* :1088-1110: every cell with |x| < cw and |y| < cw, in row-major order
       and with its current value, is offered to every cell */
    for (int i = 0; i < h; i++)
        for (int j = 0; j < w; j++) {
            i16* src = deltas + 2 * ((size_t)i * w + j);
            if (abs(src[0]) >= cw || abs(src[1]) >= cw) continue;
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++)
                    offer2(deltas + 2 * ((size_t)y * w + x), (j - x) * cw + src[0], (i - y) * cw + src[1]);
        }
}

void dolo_bruteforce_3d(int w, int h, int d, i16* deltas, int cw, int exact)
{
    for (int k = 0; k < d; k++)
        for (int j = 0; j < h; j++)
            for (int i = 0; i < w; i++) {
                i16* src = deltas + 3 * (((size_t)k * h + j) * w + i);
                if (abs(src[0]) >= cw || abs(src[1]) >= cw || abs(src[2]) >= cw) continue;
                for (int z = 0; z < d; z++)
                    for (int y = 0; y < h; y++)
                        for (int x = 0; x < w; x++) {
                            i16* c = deltas + 3 * (((size_t)z * h + y) * w + x);
                            if (exact) {
                                offer3(c, (i - x) * cw + src[0], (j - y) * cw + src[1], (k - z) * cw + src[2]);
                            } else {
                                /* :2487-2500: plain offsets, strict < on the int lengths */
                                int dx = i - x, dy = j - y, dz = k - z;
                                if (len3(dx, dy, dz) < len3(c[0], c[1], c[2])) set3(c, dx, dy, dz);
                            }
                        }
            }
}

/* ---- Felzenszwalb ----------------------------------------------------------
 * 1D lower envelope of parabolas, DistanceOcclusionLib.cpp:1026-1062, in the
 * same float arithmetic: n samples at stride m in f, n outputs contiguous in
 * out.  v holds n ints, z n+1 floats.
 */
static void felz_line(int n, int m, const float* f, float* out, int* v, float* z)
{
    int k = 0;
    v[0] = 0;
    z[0] = -FLT_MAX;
    z[1] = +FLT_MAX;
    for (int q = 1; q < n; q++) {
        float hq = f[(size_t)m * q] + (float)(q * q);
        float s;
        for (;;) {
            int p = v[k];
            float hp = f[(size_t)m * p] + (float)(p * p);
            s = (hq - hp) / (float)(2 * (q - p));
            if (s > z[k]) break;
            k--;
        }
        k++;
        v[k] = q;
        z[k] = s;
        z[k + 1] = +FLT_MAX;
    }
    k = 0;
    for (int q = 0; q < n; q++) {
        while (z[k + 1] < (float)q) k++;
        int p = v[k];
        out[q] = (float)((q - p) * (q - p)) + f[(size_t)m * p];
    }
}

void dolo_felzenszwalb_2d(int w, int h, float* dist, float* td, int* v, float* z)
{
    /* :1065-1085: columns into the transposed scratch, then rows back */
    for (int x = 0; x < w; x++) felz_line(h, w, dist + x, td + (size_t)x * h, v, z);
    for (int y = 0; y < h; y++) felz_line(w, h, td + y, dist + (size_t)y * w, v, z);
}

void dolo_felzenszwalb_3d(int w, int h, int d, float* dist, float* td, int* v, float* z)
{
    /* restatement: the 1D routine along z, y, x in turn (separable EDT) */
    size_t ss = (size_t)w * h;
    float* line = td;   /* one line of scratch is enough per 1D call */
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            float* col = dist + (size_t)y * w + x;
            felz_line(d, (int)ss, col, line, v, z);
            for (int q = 0; q < d; q++) col[(size_t)q * ss] = line[q];
        }
    for (int k = 0; k < d; k++)
        for (int x = 0; x < w; x++) {
            float* col = dist + k * ss + x;
            felz_line(h, w, col, line, v, z);
            for (int q = 0; q < h; q++) col[(size_t)q * w] = line[q];
        }
    for (int k = 0; k < d; k++)
        for (int y = 0; y < h; y++) {
            float* row = dist + k * ss + (size_t)y * w;
            felz_line(w, 1, row, line, v, z);
            memcpy(row, line, sizeof(float) * (size_t)w);
        }
}

/* One pass of the 3D restatement over a rectangle of its lines (a0 <= a < a1,
 * b0 <= b < b1): pass 0 z lines (a = y, b = x), 1 y lines (a = z, b = x), 2 x
 * rows (a = z, b = y); src -> dst, both whole volumes (dst may be src).  v, z
 * and line are scratch for one line (max(w,h,d) ints, one more float, and
 * max(w,h,d) floats). */
void dolo_felzenszwalb_3d_pass(int w, int h, int d, const float* src, float* dst, int pass, int a0, int a1, int b0,
                               int b1, int* v, float* z, float* line)
{
    size_t ss = (size_t)w * h;
    int n = pass == 0 ? d : (pass == 1 ? h : w);
    size_t stride = pass == 0 ? ss : (pass == 1 ? (size_t)w : 1);
    for (int a = a0; a < a1; a++)
        for (int b = b0; b < b1; b++) {
            size_t base = pass == 0 ? (size_t)a * w + b : (pass == 1 ? (size_t)a * ss + b : (size_t)a * ss + (size_t)b * w);
            felz_line(n, (int)stride, src + base, line, v, z);
            for (int q = 0; q < n; q++) dst[base + (size_t)q * stride] = line[q];
        }
}

/* ---- deltas -> distances ------------------------------------------------- */

void dolo_deltas_to_dist_2d(int w, int h, const i16* deltas, int cw, const uint32_t* sign_mask, float* out)
{
    int ws = words_per_row(w);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const i16* c = deltas + 2 * ((size_t)y * w + x);
            float r = sqrtf((float)len2(c[0], c[1]));
            if (cw != 1) r = r / (float)cw;
            if (sign_mask && mask_bit(sign_mask + (size_t)y * ws, x)) r = -r;
            out[(size_t)y * w + x] = r;
        }
}

void dolo_deltas_to_dist_3d(int w, int h, int d, const i16* deltas, int cw, const uint32_t* sign_mask, float* out)
{
    int ws = words_per_row(w);
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                size_t idx = ((size_t)z * h + y) * w + x;
                const i16* c = deltas + 3 * idx;
                float r = sqrtf((float)len3(c[0], c[1], c[2]));
                if (cw != 1) r = r / (float)cw;
                if (sign_mask && mask_bit(sign_mask + ((size_t)z * h + y) * ws, x)) r = -r;
                out[idx] = r;
            }
}

/* ---- exact EDT by brute force ------------------------------------------- */

void dolo_edt_brute(int w, int h, int d, const uint32_t* mask, float* out)
{
    if (d <= 0) d = 1;
    int ws = words_per_row(w);
    size_t n = (size_t)w * h * d, ns = 0;
    int* pts = (int*)malloc(sizeof(int) * 3 * (n ? n : 1));
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++)
                if (mask_bit(mask + ((size_t)z * h + y) * ws, x)) {
                    pts[3 * ns] = x; pts[3 * ns + 1] = y; pts[3 * ns + 2] = z; ns++;
                }
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                long best = -1;
                for (size_t p = 0; p < ns; p++) {
                    long dx = x - pts[3 * p], dy = y - pts[3 * p + 1], dz = z - pts[3 * p + 2];
                    long e = dx * dx + dy * dy + dz * dz;
                    if (best < 0 || e < best) best = e;
                }
                out[((size_t)z * h + y) * w + x] = best < 0 ? FLT_MAX : (float)best;
            }
    free(pts);
}

/* ---- occlusion sweeps -------------------------------------------------------
 * Direction-weight fields: 4 (2D) or 8 (3D) planes of w*h[*d] floats, plane
 * `sweep` holding the occlusion seen towards quadrant / octant `sweep`
 * (bit 0: x decreasing, bit 1: y, bit 2: z).  InitDirWFromBitMask
 * (DistanceOcclusionLib.cpp:1114-1146, :2507-2538) sets every plane to 1 on
 * set cells and 0 elsewhere.  A sweep (:1173-1209, :2593-2650, in/out form
 * :2655-2737) walks its plane from the corner it starts at: slices in z order,
 * rows in y order, cells in x order, each cell combining the already swept
 * neighbours one step back along x ("left"), y ("up") and z ("back"); a
 * neighbour outside the field enters as 0, and the corner cell itself is left
 * as it is.  Quadrant combine (:1150-1169) and octant combines (:2543-2567)
 * are evaluated in the reference's float operations and order; this file is
 * built without contraction so no step fuses. */

static inline float quad_combine(float a, float b) { return 0.75f * ((a + b) - 1.0f * a * b); }
static inline float oct_combine(float a, float b, float c) { return 0.33333333f * (a + b + c - a * b * c); }
static inline float oct_combine_io(float oa, float ob, float oc, float ia, float ib, float ic)
{
    float a = ia + (1.0f - ia) * oa;
    float b = ib + (1.0f - ib) * ob;
    float c = ic + (1.0f - ic) * oc;
    return 0.3333333f * (a + b + c - a * b * c);
}

void dolo_init_dirw(int w, int h, int d, int planes, const uint32_t* mask, float* dirW)
{
    size_t n = (size_t)w * h * d;
    int ws = words_per_row(w);
    for (size_t r = 0; r < (size_t)h * d; r++)
        for (int x = 0; x < w; x++) {
            float v = mask_bit(mask + r * ws, x) ? 1.0f : 0.0f;
            for (int p = 0; p < planes; p++) dirW[(size_t)p * n + r * w + x] = v;
        }
}

/* one plane: in == NULL updates it in place (x += (1 - x) * combine), else
 * writes combine of (out, in) neighbours to out (3D only) */
static void occ_plane(int w, int h, int d, int sweep, int dim, const float* in, float* out)
{
    int sx = sweep & 1, sy = (sweep >> 1) & 1, sz = (sweep >> 2) & 1;
    int dx = 1 - 2 * sx, dy = 1 - 2 * sy, dz = 1 - 2 * sz;
    size_t wh = (size_t)w * h;
    for (int kk = 0; kk < d; kk++) {
        int z = sz ? d - 1 - kk : kk;
        for (int jj = 0; jj < h; jj++) {
            int y = sy ? h - 1 - jj : jj;
            for (int ii = 0; ii < w; ii++) {
                int x = sx ? w - 1 - ii : ii;
                if (ii == 0 && jj == 0 && kk == 0) continue;   /* the starting corner */
                size_t c = (size_t)z * wh + (size_t)y * w + x;
                size_t cl = c - dx, cu = c - (ptrdiff_t)dy * w, cb = c - (ptrdiff_t)dz * (ptrdiff_t)wh;
                float ol = ii ? out[cl] : 0.0f, ou = jj ? out[cu] : 0.0f, ob = kk ? out[cb] : 0.0f;
                if (in) {
                    float il = ii ? in[cl] : 0.0f, iu = jj ? in[cu] : 0.0f, ib = kk ? in[cb] : 0.0f;
                    out[c] = oct_combine_io(ol, ou, ob, il, iu, ib);
                } else {
                    float q = dim == 2 ? quad_combine(ol, ou) : oct_combine(ol, ou, ob);
                    out[c] += (1.0f - out[c]) * q;
                }
            }
        }
    }
}

void dolo_occlusion_sweep_2d(int w, int h, float* dirW)
{
    for (int s = 0; s < 4; s++) occ_plane(w, h, 1, s, 2, NULL, dirW + (size_t)s * w * h);
}

void dolo_occlusion_sweep_3d(int w, int h, int d, float* dirW)
{
    size_t n = (size_t)w * h * d;
    for (int s = 0; s < 8; s++) occ_plane(w, h, d, s, 3, NULL, dirW + (size_t)s * n);
}

void dolo_occlusion_sweep_3d_io(int w, int h, int d, const float* in, float* out)
{
    size_t n = (size_t)w * h * d;
    for (int s = 0; s < 8; s++) occ_plane(w, h, d, s, 3, in + (size_t)s * n, out + (size_t)s * n);
}

/* ---- mesh voxeliser -----------------------------------------------------------
 * MSL::CreateBitMaskFromTriangles (MeshSupport.cpp:369-475) with its
 * triangle / cell overlap tests (cTriCellIntersectDelta, :158-353): for each
 * triangle, the cells of its bounding box (in the grid spanning bbox) whose
 * box, grown by 0.000001 of a cell, meets the triangle -- the separating-axis
 * tests on the edge cross products, the box ranges, then the triangle's
 * plane -- get their bit set.  Float operations as the reference evaluates
 * them (this file is built without contraction). */
typedef struct { float x, y, z; } v3f;

static inline float fmin_ref(float a, float b) { return a < b ? a : b; }
static inline float fmax_ref(float a, float b) { return b < a ? a : b; }

typedef struct {
    v3f e[3], t[3], u[3], pmin, pmax, hw, n;
    float ndv_min, ndv_max, nd;
} tri_setup;

static void tri_prepare(tri_setup* s, v3f p1, v3f p2, v3f p3, v3f hw)
{
    const v3f* P[3] = {&p1, &p2, &p3};
    s->hw = hw;
    s->e[0] = (v3f){p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
    s->e[1] = (v3f){p3.x - p2.x, p3.y - p2.y, p3.z - p2.z};
    s->e[2] = (v3f){p1.x - p3.x, p1.y - p3.y, p1.z - p3.z};
    /* twice the area normal, :138-150 */
    s->n.x = (p1.y - p2.y) * (p1.z + p2.z) + (p2.y - p3.y) * (p2.z + p3.z) + (p3.y - p1.y) * (p3.z + p1.z);
    s->n.y = (p1.z - p2.z) * (p1.x + p2.x) + (p2.z - p3.z) * (p2.x + p3.x) + (p3.z - p1.z) * (p3.x + p1.x);
    s->n.z = (p1.x - p2.x) * (p1.y + p2.y) + (p2.x - p3.x) * (p2.y + p3.y) + (p3.x - p1.x) * (p3.y + p1.y);
    v3f vmin = {s->n.x > 0.0f ? -hw.x : hw.x, s->n.y > 0.0f ? -hw.y : hw.y, s->n.z > 0.0f ? -hw.z : hw.z};
    v3f vmax = {s->n.x > 0.0f ? hw.x : -hw.x, s->n.y > 0.0f ? hw.y : -hw.y, s->n.z > 0.0f ? hw.z : -hw.z};
    s->ndv_min = s->n.x * vmin.x + s->n.y * vmin.y + s->n.z * vmin.z;
    s->ndv_max = s->n.x * vmax.x + s->n.y * vmax.y + s->n.z * vmax.z;
    s->nd = s->n.x * p1.x + s->n.y * p1.y + s->n.z * p1.z;
    /* per edge k, the vertices its three axis tests project: (for t.x, t.y,
       t.z) and (for u.x, u.y, u.z), as in :199-239 */
    static const int tv[3][3] = {{0, 0, 1}, {0, 0, 0}, {0, 0, 1}};
    static const int uv[3][3] = {{2, 2, 2}, {2, 2, 1}, {1, 1, 2}};
    for (int k = 0; k < 3; k++) {
        v3f e = s->e[k];
        const v3f *a0 = P[tv[k][0]], *a1 = P[tv[k][1]], *a2 = P[tv[k][2]];
        const v3f *b0 = P[uv[k][0]], *b1 = P[uv[k][1]], *b2 = P[uv[k][2]];
        v3f t = {e.z * a0->y - e.y * a0->z, -e.z * a1->x + e.x * a1->z, e.y * a2->x - e.x * a2->y};
        v3f u = {e.z * b0->y - e.y * b0->z, -e.z * b1->x + e.x * b1->z, e.y * b2->x - e.x * b2->y};
        float q;
        if (t.x >= u.x) { q = t.x; t.x = u.x; u.x = q; }
        if (t.y >= u.y) { q = t.y; t.y = u.y; u.y = q; }
        if (t.z >= u.z) { q = t.z; t.z = u.z; u.z = q; }
        v3f ae = {fabsf(e.x), fabsf(e.y), fabsf(e.z)};
        v3f r = {ae.z * hw.y + ae.y * hw.z, ae.z * hw.x + ae.x * hw.z, ae.y * hw.x + ae.x * hw.y};
        s->t[k] = (v3f){t.x - r.x, t.y - r.y, t.z - r.z};
        s->u[k] = (v3f){u.x + r.x, u.y + r.y, u.z + r.z};
    }
    s->pmin = (v3f){fmin_ref(fmin_ref(p1.x, p2.x), p3.x), fmin_ref(fmin_ref(p1.y, p2.y), p3.y),
                    fmin_ref(fmin_ref(p1.z, p2.z), p3.z)};
    s->pmax = (v3f){fmax_ref(fmax_ref(p1.x, p2.x), p3.x), fmax_ref(fmax_ref(p1.y, p2.y), p3.y),
                    fmax_ref(fmax_ref(p1.z, p2.z), p3.z)};
}

static int tri_hits_slice(const tri_setup* s, v3f c)
{
    return !(s->pmin.z - c.z > s->hw.z || s->pmax.z - c.z < -s->hw.z);
}

static int tri_hits_row(const tri_setup* s, v3f c)
{
    for (int k = 0; k < 3; k++) {
        float dr = s->e[k].z * c.y - s->e[k].y * c.z;
        if (s->t[k].x > dr || s->u[k].x < dr) return 0;
    }
    return !(s->pmin.y - c.y > s->hw.y || s->pmax.y - c.y < -s->hw.y);
}

static int tri_hits_cell(const tri_setup* s, v3f c)
{
    for (int k = 0; k < 3; k++) {
        float dr = -s->e[k].z * c.x + s->e[k].x * c.z;
        if (s->t[k].y > dr || s->u[k].y < dr) return 0;
        dr = s->e[k].y * c.x - s->e[k].x * c.y;
        if (s->t[k].z > dr || s->u[k].z < dr) return 0;
    }
    if (s->pmin.x - c.x > s->hw.x || s->pmax.x - c.x < -s->hw.x) return 0;
    float d = s->nd - (s->n.x * c.x + s->n.y * c.y + s->n.z * c.z);
    return s->ndv_min <= d && s->ndv_max >= d;
}

void dolo_voxelize(int tri_count, const int* indices, const float* vertices, const float* bbox, int w, int h, int d,
                   uint32_t* mask)
{
    const int ws = words_per_row(w);
    const size_t slice = (size_t)ws * h;
    const v3f cmin = {bbox[0], bbox[1], bbox[2]};
    const v3f ext = {bbox[3] - bbox[0], bbox[4] - bbox[1], bbox[5] - bbox[2]};
    const v3f cellW = {ext.x / (float)w, ext.y / (float)h, ext.z / (float)d};
    const v3f inv = {(float)w / ext.x, (float)h / ext.y, (float)d / ext.z};
    const v3f hw = {cellW.x * 0.500001f, cellW.y * 0.500001f, cellW.z * 0.500001f};
    for (int t = 0; t < tri_count; t++) {
        v3f p[3];
        for (int k = 0; k < 3; k++) {
            const float* v = vertices + 3 * (size_t)(indices ? indices[3 * t + k] : 3 * t + k);
            p[k] = (v3f){v[0], v[1], v[2]};
        }
        v3f bmin = {fmin_ref(fmin_ref(p[0].x, p[1].x), p[2].x), fmin_ref(fmin_ref(p[0].y, p[1].y), p[2].y),
                    fmin_ref(fmin_ref(p[0].z, p[1].z), p[2].z)};
        v3f bmax = {fmax_ref(fmax_ref(p[0].x, p[1].x), p[2].x), fmax_ref(fmax_ref(p[0].y, p[1].y), p[2].y),
                    fmax_ref(fmax_ref(p[0].z, p[1].z), p[2].z)};
        int x0 = (int)floorf((bmin.x - cmin.x) * inv.x), y0 = (int)floorf((bmin.y - cmin.y) * inv.y),
            z0 = (int)floorf((bmin.z - cmin.z) * inv.z);
        int x1 = (int)ceilf((bmax.x - cmin.x) * inv.x), y1 = (int)ceilf((bmax.y - cmin.y) * inv.y),
            z1 = (int)ceilf((bmax.z - cmin.z) * inv.z);
        if (x0 < 0) x0 = 0;
        if (y0 < 0) y0 = 0;
        if (z0 < 0) z0 = 0;
        if (x1 > w) x1 = w;
        if (y1 > h) y1 = h;
        if (z1 > d) z1 = d;
        if (x0 == x1) continue;   /* as the reference: only an empty x range skips the triangle */
        if (x0 + 1 == x1 && y0 + 1 == y1 && z0 + 1 == z1) {   /* a single cell: set without testing */
            mask[slice * z0 + (size_t)ws * y0 + (x0 >> 5)] |= 1u << (x0 & 31);
            continue;
        }
        tri_setup s;
        tri_prepare(&s, p[0], p[1], p[2], hw);
        for (int z = z0; z < z1; z++) {
            v3f c;
            c.z = cmin.z + cellW.z * ((float)z + 0.5f);
            if (!tri_hits_slice(&s, c)) continue;
            for (int y = y0; y < y1; y++) {
                c.y = cmin.y + cellW.y * ((float)y + 0.5f);
                if (!tri_hits_row(&s, c)) continue;
                for (int x = x0; x < x1; x++) {
                    c.x = cmin.x + cellW.x * ((float)x + 0.5f);
                    if (tri_hits_cell(&s, c)) mask[slice * z + (size_t)ws * y + (x >> 5)] |= 1u << (x & 31);
                }
            }
        }
    }
}
