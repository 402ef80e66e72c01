/*
 * dol_oracle.h -- CPU restatement of the distance-field path of
 * DistanceOcclusionLib (DistanceOcclusionLib.cpp / DistanceOcclusionTool.cpp).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA library is compared
 * against: tests/ load it through ctypes, __graft_entry__.smoke() uses it to
 * check one small call, and bench.py's CPU-baseline leg times it.  The shipped
 * library (libdol_b200.so) neither links nor calls anything here.
 *
 * Layout contract (same bytes as the reference):
 *   mask   : uint32 words, rows padded to (w+31)/32 words, bit i of word j is
 *            cell 32*j+i (LSB first); rows then slices.
 *   deltas : interleaved int16 (x,y) per cell in 2D (cCellDelta2, 4 bytes) and
 *            (x,y,z) in 3D (cCellDelta3, 6 bytes), row-major, x fastest.
 *
 * Parity is pinned two ways (see tests/test_oracle_pin.py): against the
 * reference library compiled from its own sources into oracle/_ref/, and
 * against golden vectors in tests/golden/ generated from that build.
 */
#ifndef DOL_ORACLE_H
#define DOL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DOLO_MAX2 32767   /* kMaxDelta2, DistanceOcclusionLib.h:56 */
#define DOLO_MAX3 25000   /* kMaxDelta3, DistanceOcclusionLib.h:57 */

int  dolo_mask_words(int w, int h, int d);

/* test-mask generators (DistanceOcclusionLib.cpp:95-179, 1224-1287) */
void dolo_add_points_2d(int w, int h, int n, uint32_t seed, uint32_t* mask);
void dolo_add_points_3d(int w, int h, int d, int n, uint32_t seed, uint32_t* mask);
void dolo_add_block_2d(int w, int h, int sides, uint32_t* mask);
void dolo_add_block_3d(int w, int h, int d, int sides, uint32_t* mask);

/* byte image -> bitmask (DistanceOcclusionTool.cpp:634-670) */
void dolo_pack_bytes(int w, int h, const uint8_t* img, int threshold, int less_than, uint32_t* mask);

/* initialisation (DistanceOcclusionLib.cpp:183-254, 1289-1321) */
void dolo_init_distances_2d(int w, int h, const uint32_t* mask, float* dist, float max_d);
void dolo_init_distances_2d_i16(int w, int h, const uint32_t* mask, int16_t* dist, int16_t max_d);
void dolo_init_distances_2d_i32(int w, int h, const uint32_t* mask, int32_t* dist, int32_t max_d);
int dolo_chamfer_2d_i16(int w, int h, int16_t* dist);
int dolo_chamfer_2d_i32(int w, int h, int32_t* dist);
void dolo_init_deltas_2d(int w, int h, const uint32_t* mask, int16_t* deltas, int invert);
void dolo_init_deltas_3d(int w, int h, int d, const uint32_t* mask, int16_t* deltas, int invert);

/* signed border initialisation (DistanceOcclusionLib.cpp:504-619, 1820-2173) */
void dolo_border_init_2d(int w, int h, const uint32_t* mask, int16_t* deltas);
void dolo_border_init_3d(int w, int h, int d, const uint32_t* mask, int16_t* deltas);

/* delta propagation */
void dolo_danielsson_2d(int w, int h, int16_t* deltas, int cw);
void dolo_danielsson_3d(int w, int h, int d, int16_t* deltas, int cw);
void dolo_fastsweep_2d(int w, int h, int16_t* deltas, int cw);
void dolo_fastsweep_3d(int w, int h, int d, int16_t* deltas, int cw);
/* temp must hold w*h[*d] cells; it is the reference's internal ping-pong buffer */
void dolo_jumpflood_2d(int w, int h, int16_t* deltas, int cw, int16_t* temp);
void dolo_jumpflood_3d(int w, int h, int d, int16_t* deltas, int cw, int16_t* temp);
void dolo_bruteforce_2d(int w, int h, int16_t* deltas, int cw);
/* exact=0: the reference's 3D brute force (ignores cw and the border offsets);
   exact=1: the 2D rule generalised to 3D, (i-x)*cw + cell, correct for cw=2 */
void dolo_bruteforce_3d(int w, int h, int d, int16_t* deltas, int cw, int exact);

/* Felzenszwalb squared EDT; scratch: v holds max(w,h[,d]) ints, z one more
   float, td w*h[*d] floats.  2D follows DistanceOcclusionLib.cpp:1065-1085;
   3D is a restatement (none in the reference): the same 1D routine along z,
   then y, then x. */
void dolo_felzenszwalb_2d(int w, int h, float* dist, float* td, int* v, float* z);
void dolo_felzenszwalb_3d(int w, int h, int d, float* dist, float* td, int* v, float* z);
/* one pass of the 3D form over lines (a, b), a0 <= a < a1, b0 <= b < b1 (pass 0:
   z lines, a = y, b = x; 1: y lines, a = z, b = x; 2: x rows, a = z, b = y) */
void dolo_felzenszwalb_3d_pass(int w, int h, int d, const float* src, float* dst, int pass, int a0, int a1, int b0,
                               int b1, int* v, float* z, float* line);

/* deltas -> float distances (DistanceOcclusionTool.cpp:46-61, sign as at
   :1262/:1392): sqrtf((float)len2) / cw, negated where sign_mask has the bit */
void dolo_deltas_to_dist_2d(int w, int h, const int16_t* deltas, int cw, const uint32_t* sign_mask, float* out);
void dolo_deltas_to_dist_3d(int w, int h, int d, const int16_t* deltas, int cw, const uint32_t* sign_mask, float* out);

/* exact squared EDT to the set cells of mask by brute force (for small n);
   cells with no set cell anywhere get FLT_MAX */
void dolo_edt_brute(int w, int h, int d, const uint32_t* mask, float* out);

/* occlusion: direction-weight planes (4 for 2D, 8 for 3D) from a mask, and the
   quadrant / octant sweeps in place (2D, 3D) or from in to out (3D) */
void dolo_init_dirw(int w, int h, int d, int planes, const uint32_t* mask, float* dirW);
void dolo_occlusion_sweep_2d(int w, int h, float* dirW);
void dolo_occlusion_sweep_3d(int w, int h, int d, float* dirW);
void dolo_occlusion_sweep_3d_io(int w, int h, int d, const float* in, float* out);

/* mesh voxeliser: ORs the cells of the w x h x d grid over bbox (min xyz, max
   xyz) that the triangles touch into mask; indices may be NULL (vertices then
   taken three per triangle) */
void dolo_voxelize(int tri_count, const int* indices, const float* vertices, const float* bbox, int w, int h, int d,
                   uint32_t* mask);

#ifdef __cplusplus
}
#endif
#endif
