/*
 * dol_b200.h -- C ABI of the B200 (sm_100a) distance-field library.
 *
 * A drop-in for the distance-field path of DistanceOcclusionLib
 * (DistanceOcclusionLib.h, namespace DOL).  Every entry point takes plain
 * pointers and sizes; the reference function each one replaces is cited
 * beside it.  Data layouts are byte-identical to the reference's:
 *
 *   mask    uint32 words, each row padded to (w+31)/32 words, bit i of word j
 *           is cell 32*j+i; rows, then slices.          (DistanceOcclusionLib.h:18-23)
 *   deltas  dol_delta2 {int16 x,y} / dol_delta3 {int16 x,y,z}, row-major, x
 *           fastest: the same bytes as cCellDelta2 / cCellDelta3
 *                                                         (DistanceOcclusionLib.h:41-53)
 *   dist    float per cell, same order.
 *
 * Unless a name ends in _host, every pointer argument is DEVICE memory
 * (cudaMalloc / cudaMallocAsync / managed) and work is queued on `stream`
 * (a cudaStream_t passed as void*; NULL is the legacy default stream).  The
 * call returns once the work is queued; errors found before queueing are
 * returned at once, device-side errors (a bounded wait that gave up) are
 * reported by the next dol_sync() on that stream.  Pointers that are not
 * device-accessible are rejected with DOL_ERR_INVALID_ARG before anything is
 * launched.
 *
 * `cw` is the cell width used by the delta methods: 1 for unsigned fields
 * initialised by dol_init_deltas_*, 2 for signed fields initialised by
 * dol_init_border_* (deltas are then in half cells).
 *
 * Scratch: entry points that need temporary device memory take
 * (void* workspace, size_t workspace_bytes).  Pass NULL/0 to let the library
 * allocate it stream-ordered (cudaMallocAsync) and free it after the work;
 * the dol_*_workspace_size() queries give the size to pre-allocate.
 */
#ifndef DOL_B200_H
#define DOL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DOL_B200_VERSION 1

#if defined(__GNUC__)
#define DOL_API __attribute__((visibility("default")))
#else
#define DOL_API
#endif

typedef enum dol_status {
    DOL_OK = 0,
    DOL_ERR_INVALID_ARG = 1,   /* bad size, null or non-device pointer, ...      */
    DOL_ERR_CUDA = 2,          /* a CUDA runtime call failed (see dol_last_error) */
    DOL_ERR_NO_MEMORY = 3,     /* workspace allocation failed                     */
    DOL_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up              */
    DOL_ERR_UNSUPPORTED = 5,   /* size or option outside what this build handles  */
} dol_status;

typedef struct dol_delta2 { int16_t x, y; } dol_delta2;        /* == DOL::cCellDelta2 */
typedef struct dol_delta3 { int16_t x, y, z; } dol_delta3;     /* == DOL::cCellDelta3 */

#define DOL_MAX_DELTA2 32767   /* kMaxDelta2, DistanceOcclusionLib.h:56 */
#define DOL_MAX_DELTA3 25000   /* kMaxDelta3, DistanceOcclusionLib.h:57 */

/* delta propagation methods, numbered as the tool's -m (DistanceOcclusionTool.cpp:700-709) */
typedef enum dol_method {
    DOL_DANIELSSON = 0,
    DOL_FASTSWEEP = 1,
    DOL_JUMPFLOOD = 2,
    DOL_FELZENSZWALB = 5,
} dol_method;

/* output forms of the mask-driven Felzenszwalb EDT */
#define DOL_EDT_SQUARED 0   /* squared distance to the nearest set cell, FLT_MAX if none  */
#define DOL_EDT_DIST    1   /* sqrtf of the above (the tool's output, Tool.cpp:753-754)   */
#define DOL_EDT_SIGNED  2   /* dist to set cells minus dist to clear cells (the -S rule)  */

/* ---- library ---------------------------------------------------------------- */
DOL_API int         dol_version(void);
DOL_API const char* dol_status_string(dol_status s);
DOL_API const char* dol_last_error(void);            /* detail of the last failure on this thread */
DOL_API dol_status  dol_sync(void* stream);          /* wait for the stream, report device errors */
/* Caps the scratch the library allocates by itself (0: no cap, the default);
   process-wide.  Entry points needing more return DOL_ERR_NO_MEMORY, except
   Danielsson, which then runs its serial engine (see dol_last_engine).
   No reference counterpart. */
DOL_API void        dol_set_workspace_limit(size_t bytes);

/* ---- bitmasks --------------------------------------------------------------- */
/* MaskSize (DistanceOcclusionLib.h:124-135); d = 1 for images */
DOL_API size_t dol_mask_words(int w, int h, int d);

/* host-side test-mask generators, the reference's LCG and shapes
   (BitMaskAddPoints :95-113/:1224-1244, BitMaskAddBlock :159-179/:1259-1287) */
DOL_API void dol_add_points_2d(int w, int h, int n, uint32_t seed, uint32_t* host_mask);
DOL_API void dol_add_points_3d(int w, int h, int d, int n, uint32_t seed, uint32_t* host_mask);
DOL_API void dol_add_block_2d(int w, int h, int sides, uint32_t* host_mask);
DOL_API void dol_add_block_3d(int w, int h, int d, int sides, uint32_t* host_mask);

/* byte image/volume -> bitmask: bit = (v >= threshold) ^ less_than
   (BitMaskFromImageFile, DistanceOcclusionTool.cpp:634-670) */
DOL_API dol_status dol_pack_bytemask(int w, int h, int d, const uint8_t* bytes, int threshold, int less_than,
                             uint32_t* mask, void* stream);

/* ---- initialisation ------------------------------------------------------------ */
/* InitDistancesFromBitMask(float) (DistanceOcclusionLib.cpp:211-222): 0 on set bits, max_d elsewhere */
DOL_API dol_status dol_init_distances_2d(int w, int h, const uint32_t* mask, float* dist, float max_d, void* stream);
/* InitDistancesFromBitMask(int16_t / int32_t) (DistanceOcclusionLib.cpp:203-214, header :60-61) */
DOL_API dol_status dol_init_distances_2d_i16(int w, int h, const uint32_t* mask, int16_t* dist, int16_t max_d,
                                             void* stream);
DOL_API dol_status dol_init_distances_2d_i32(int w, int h, const uint32_t* mask, int32_t* dist, int32_t max_d,
                                             void* stream);
/* InitDeltasFromBitMask (DistanceOcclusionLib.cpp:224-254, :1289-1321) */
DOL_API dol_status dol_init_deltas_2d(int w, int h, const uint32_t* mask, dol_delta2* deltas, int invert, void* stream);
DOL_API dol_status dol_init_deltas_3d(int w, int h, int d, const uint32_t* mask, dol_delta3* deltas, int invert, void* stream);
/* InitBorderDeltasFromBitMask (DistanceOcclusionLib.cpp:604-619, :2154-2173) */
DOL_API dol_status dol_init_border_2d(int w, int h, const uint32_t* mask, dol_delta2* deltas, void* stream);
DOL_API dol_status dol_init_border_3d(int w, int h, int d, const uint32_t* mask, dol_delta3* deltas, void* stream);

/* ---- delta propagation (in place) ------------------------------------------------- */
/* Danielsson (DistanceOcclusionLib.cpp:702-778, :2348-2394).  Large fields
   run as an exact block schedule that needs scratch of
   dol_danielsson_workspace_size() bytes (about 2.2x the field for volumes);
   the plain entries allocate it stream-ordered, the _ws entries take the
   caller's (NULL: allocate; too small: DOL_ERR_INVALID_ARG).  Without it --
   the allocation failed or is above the dol_set_workspace_limit cap -- the
   serial engine runs instead: same deltas, far slower on large fields; the
   call still returns DOL_OK, and dol_last_engine() / dol_last_error() say so. */
DOL_API dol_status dol_danielsson_2d(int w, int h, dol_delta2* deltas, int cw, void* stream);
DOL_API dol_status dol_danielsson_3d(int w, int h, int d, dol_delta3* deltas, int cw, void* stream);
DOL_API size_t     dol_danielsson_workspace_size(int w, int h, int d);   /* d = 1 for images; 0: none used */
DOL_API dol_status dol_danielsson_2d_ws(int w, int h, dol_delta2* deltas, int cw, void* workspace,
                                        size_t workspace_bytes, void* stream);
DOL_API dol_status dol_danielsson_3d_ws(int w, int h, int d, dol_delta3* deltas, int cw, void* workspace,
                                        size_t workspace_bytes, void* stream);
/* the engine this thread's last Danielsson call queued (no reference counterpart) */
#define DOL_ENGINE_BLOCKS 1   /* exact block schedule on a workspace */
#define DOL_ENGINE_SERIAL 2   /* serial single-CTA engine, no workspace */
DOL_API int        dol_last_engine(void);
/* FastSweep (DistanceOcclusionLib.cpp:633-697, :2186-2260) */
DOL_API dol_status dol_fastsweep_2d(int w, int h, dol_delta2* deltas, int cw, void* stream);
DOL_API size_t     dol_fastsweep_3d_workspace_size(int w, int h, int d);
DOL_API dol_status dol_fastsweep_3d(int w, int h, int d, dol_delta3* deltas, int cw,
                            void* workspace, size_t workspace_bytes, void* stream);
/* JumpFlood (DistanceOcclusionLib.cpp:887-908, :2450-2472); the workspace
   stands for the reference's internal ping-pong buffer: one 4-byte cell per
   cell in 2D; in 3D two buffers of 8-byte cells (one aligned load per
   neighbour), the caller's 6-byte cells being read by the first pass and
   written by the last */
DOL_API size_t     dol_jumpflood_2d_workspace_size(int w, int h);
DOL_API size_t     dol_jumpflood_3d_workspace_size(int w, int h, int d);
DOL_API dol_status dol_jumpflood_2d(int w, int h, dol_delta2* deltas, int cw,
                            void* workspace, size_t workspace_bytes, void* stream);
DOL_API dol_status dol_jumpflood_3d(int w, int h, int d, dol_delta3* deltas, int cw,
                            void* workspace, size_t workspace_bytes, void* stream);

/* ---- Chamfer 3-4 (integer distances, in place) ------------------------------------------ */
/* Chamfer(w, h, int16_t[] / int32_t[]) (DistanceOcclusionLib.cpp:916-1016, header :66-67):
   one raster pass down and one up with edge cost 3 and diagonal cost 4.
   *multiplier (nullable, host) receives 3: divide by it for cells.  Rows of at
   least 2 and at most 4096 cells.  int32 fields: results equal the reference's
   while every input is at most INT32_MAX - 4 (beyond that the reference's own
   int32 sums wrap). */
DOL_API dol_status dol_chamfer_2d_i16(int w, int h, int16_t* dist, int* multiplier, void* stream);
DOL_API dol_status dol_chamfer_2d_i32(int w, int h, int32_t* dist, int* multiplier, void* stream);

/* ---- Felzenszwalb ------------------------------------------------------------------- */
/* Felzenszwalb(w,h,float[]) (DistanceOcclusionLib.cpp:1065-1085): in-place squared
   distance transform of an arbitrary float field, same float arithmetic */
DOL_API size_t     dol_felzenszwalb_2d_workspace_size(int w, int h);
DOL_API dol_status dol_felzenszwalb_2d(int w, int h, float* dist, void* workspace, size_t workspace_bytes, void* stream);
/* Mask-driven exact EDT, the tool's InitDistancesFromBitMask + Felzenszwalb (+ sqrtf)
   path (DistanceOcclusionTool.cpp:741-782) in 2D; the 3D form has no reference
   counterpart (the same separable transform along z, y, x).  `form` is DOL_EDT_*. */
DOL_API size_t     dol_edt_mask_2d_workspace_size(int w, int h);
DOL_API size_t     dol_edt_mask_3d_workspace_size(int w, int h, int d);
DOL_API dol_status dol_edt_mask_2d(int w, int h, const uint32_t* mask, float* out, int form,
                           void* workspace, size_t workspace_bytes, void* stream);
DOL_API dol_status dol_edt_mask_3d(int w, int h, int d, const uint32_t* mask, float* out, int form,
                           void* workspace, size_t workspace_bytes, void* stream);

/* ---- 2D mask EDT without allocation (no counterpart in the reference) -----------------
   The same result as dol_edt_mask_2d for callers that cannot allocate device
   memory when they call: applications that reserve all of their GPU memory up
   front and forbid allocation afterwards (engines, plugin hosts with their own
   memory manager), or code that must not risk an allocation failing or
   stalling mid-frame.  The scratch is a fixed 16 MiB array inside the library
   that every GPU loading the library holds until the process exits; images are
   limited to 8,388,608 cells (w*h) and sides to 16384, larger ones return
   DOL_ERR_UNSUPPORTED.  The first call on a device looks up the array's device
   address (cudaGetSymbolAddress); make that first call before any stream
   capture.  All calls share the array, so calls that overlap on the GPU race:
   serialise them.  mask and out are device memory; nothing is allocated. */
DOL_API dol_status dol_edt_mask_2d_noalloc(int w, int h, const uint32_t* mask, float* out, int form, void* stream);

/* ---- deltas -> distances ------------------------------------------------------------ */
/* Dist() (DistanceOcclusionTool.cpp:46-61): out = sqrtf((float)(x*x+y*y[+z*z])) / cw,
   negated where sign_mask (nullable) has the cell's bit (Tool.cpp:1262, :1392) */
DOL_API dol_status dol_deltas_to_dist_2d(int w, int h, const dol_delta2* deltas, int cw, const uint32_t* sign_mask,
                                 float* out, void* stream);
DOL_API dol_status dol_deltas_to_dist_3d(int w, int h, int d, const dol_delta3* deltas, int cw,
                                 const uint32_t* sign_mask, float* out, void* stream);

/* ---- occlusion -------------------------------------------------------------------------
   Direction-weight fields: 4 (2D) or 8 (3D) planes of w*h[*d] floats, plane s
   for quadrant / octant s (bit 0: x decreasing, bit 1: y, bit 2: z).
   InitDirWFromBitMask (DistanceOcclusionLib.cpp:1114-1146, :2507-2538): 1 on set
   cells, 0 elsewhere, in every plane.
   OcclusionSweep (DistanceOcclusionLib.cpp:1173-1209, :2745-2769), in place;
   the 3D in/out form (:2771-2784) writes the occlusion caused by `in` to `out`
   (out's starting-corner cell of each plane is left as it was).  Bit-exact:
   the reference's float operations in its order.  Any shape whose planes fit
   the device. */
DOL_API dol_status dol_init_dirw_2d(int w, int h, const uint32_t* mask, float* dirW, void* stream);
DOL_API dol_status dol_init_dirw_3d(int w, int h, int d, const uint32_t* mask, float* dirW, void* stream);
DOL_API dol_status dol_occlusion_sweep_2d(int w, int h, float* dirW, void* stream);
DOL_API dol_status dol_occlusion_sweep_3d(int w, int h, int d, float* dirW, void* stream);
DOL_API dol_status dol_occlusion_sweep_3d_io(int w, int h, int d, const float* in, float* out, void* stream);

/* ---- mesh voxeliser ----------------------------------------------------------------------
   MSL::CreateBitMaskFromTriangles (MeshSupport.cpp:369-475): ORs into `mask`
   (device, w x h x d) every cell of the grid spanning `bbox` (HOST array: min
   x, y, z, max x, y, z) that one of the triangles touches, bit for bit as the
   reference decides it.  indices: device int[3 * tri_count] into vertices
   (device float[3 * n]); NULL takes the vertices three per triangle.  Every
   bbox extent must be positive.  The mask feeds dol_init_border_3d,
   dol_sdf_3d, dol_edt_mask_3d ... without leaving the device. */
DOL_API dol_status dol_voxelize_triangles(int tri_count, const int* indices, const float* vertices, const float* bbox,
                                          int w, int h, int d, uint32_t* mask, void* stream);

/* ---- one-call fields (the tool's Generate* paths) ----------------------------------- */
/* Signed border-initialised distance field (GenerateSignedDistanceBorder,
   DistanceOcclusionTool.cpp:1333-1365 / :1471-1498): border init, `method`
   with cw = 2, then signed distances.  deltas (nullable) receives the final
   deltas; dist (nullable) the signed float distances in cells. */
DOL_API size_t     dol_sdf_workspace_size(int w, int h, int d, int method);
DOL_API dol_status dol_sdf_2d(int w, int h, const uint32_t* mask, int method, dol_delta2* deltas, float* dist,
                      void* workspace, size_t workspace_bytes, void* stream);
DOL_API dol_status dol_sdf_3d(int w, int h, int d, const uint32_t* mask, int method, dol_delta3* deltas, float* dist,
                      void* workspace, size_t workspace_bytes, void* stream);
/* Two-pass signed field (the tool's -S path, GenerateSignedDistance,
   DistanceOcclusionTool.cpp:1082-1123 2D / :1197-1232 3D): deltas to set cells
   (InitDeltasFromBitMask, invert = false) and to clear cells (invert = true),
   each propagated by `method` (Danielsson, FastSweep or JumpFlood) with cw = 1;
   dist = Dist(exterior) - Dist(interior) in cells (:54-61).  Any of exterior,
   interior, dist may be NULL (not all three). */
DOL_API size_t     dol_sdf_two_pass_workspace_size(int w, int h, int d, int method);
DOL_API dol_status dol_sdf_two_pass_2d(int w, int h, const uint32_t* mask, int method, dol_delta2* exterior,
                                       dol_delta2* interior, float* dist, void* workspace, size_t workspace_bytes,
                                       void* stream);
DOL_API dol_status dol_sdf_two_pass_3d(int w, int h, int d, const uint32_t* mask, int method, dol_delta3* exterior,
                                       dol_delta3* interior, float* dist, void* workspace, size_t workspace_bytes,
                                       void* stream);
/* Same with HOST mask in and HOST outputs (either nullable); copies inside.
   Blocks until the result is in host memory. */
DOL_API dol_status dol_sdf_2d_host(int w, int h, const uint32_t* mask, int method, dol_delta2* deltas, float* dist);
DOL_API dol_status dol_sdf_3d_host(int w, int h, int d, const uint32_t* mask, int method, dol_delta3* deltas, float* dist);
/* Mask-driven EDT with host buffers (DOL_EDT_* form) */
DOL_API dol_status dol_edt_mask_3d_host(int w, int h, int d, const uint32_t* mask, float* out, int form);

/* ---- batched signed fields (no reference counterpart) ----------------------------------
   Many independent images and volumes of different sizes, each run through
   the signed border pipeline of dol_sdf_2d/3d with Danielsson (border init,
   cw = 2 propagation, signed distances), in ONE persistent launch: each CTA
   takes the next item, largest first, from an atomic counter.  Every item's
   deltas and distances are bit-identical to a per-item dol_sdf_* call.
   Items: d = 1 for an image; w <= 1024.  masks, deltas, dist are single
   device buffers; each item gives its offsets into them (dist_offset < 0: no
   distances for that item).  dol_batch_prepare uploads and orders the items
   into the workspace once; dol_batch_run only launches (and may be captured
   into a graph, which dol_batch_graph_create does). */
typedef struct dol_batch_item {
    int w, h, d;                    /* d = 1 for an image                         */
    int reserved;                   /* 0                                          */
    long long mask_word_offset;     /* into masks (uint32 words)                  */
    long long delta_byte_offset;    /* into deltas (4-byte cells 2D, 6-byte 3D)   */
    long long dist_offset;          /* into dist (floats); < 0: no distances      */
} dol_batch_item;

DOL_API size_t     dol_batch_workspace_size(int n_items);
DOL_API dol_status dol_batch_prepare(int n_items, const dol_batch_item* host_items, void* workspace,
                                     size_t workspace_bytes, void* stream);
DOL_API dol_status dol_batch_run(int n_items, const uint32_t* masks, void* deltas, float* dist, void* workspace,
                                 void* stream);
DOL_API dol_status dol_batch_sdf(int n_items, const dol_batch_item* host_items, const uint32_t* masks, void* deltas,
                                 float* dist, void* workspace, size_t workspace_bytes, void* stream);
/* CUDA graph of dol_batch_run on a prepared workspace; launch it with
   dol_graph_launch, release it with dol_graph_destroy */
DOL_API dol_status dol_batch_graph_create(int n_items, const uint32_t* masks, void* deltas, float* dist,
                                          void* workspace, void** graph);
DOL_API dol_status dol_graph_launch(void* graph, void* stream);
DOL_API void       dol_graph_destroy(void* graph);

/* ---- distances to float sites and their gradient (no reference counterpart) -------------
   dim = 2 (grid w x h, d = 1, sites as n x 2 floats) or 3 (w x h x d, n x 3
   floats), in continuous cell coordinates (cell x covers [x, x+1)).
   dol_sites_seed: the cell holding each site gets its mask bit; cell_site
   (one int per cell) receives the smallest site index in the cell, a value
   >= n_sites elsewhere.  Run a delta method (cw = 1) on the mask, then
   dol_sites_forward: owner[p] = the site the cell's delta reaches (-1 if
   none), dist[p] = |p - site| in fp32 with p the cell centre (NaN if none).
   dol_sites_backward: with that owner assignment fixed,
   grad_sites[k] = sum over cells p owned by k of grad_dist[p] *
   (site_k - p) / |site_k - p| (segmented reduce by owner, fp64 accumulation,
   fp32 result). */
DOL_API dol_status dol_sites_seed(int dim, int w, int h, int d, int n_sites, const float* sites, uint32_t* mask,
                                  int* cell_site, void* stream);
DOL_API dol_status dol_sites_forward(int dim, int w, int h, int d, int n_sites, const void* deltas,
                                     const int* cell_site, const float* sites, int* owner, float* dist, void* stream);
DOL_API size_t     dol_sites_backward_workspace_size(int dim, int n_sites);
DOL_API dol_status dol_sites_backward(int dim, int w, int h, int d, int n_sites, const int* owner, const float* sites,
                                      const float* grad_dist, float* grad_sites, void* workspace,
                                      size_t workspace_bytes, void* stream);

/* ---- autotuning (no reference counterpart) ---------------------------------------------
   Launch parameters that change speed but never results: cells per thread of
   the row sweeps, rows per CTA of the JumpFlood passes, threads per CTA of the
   EDT line passes, the CTA shape of the batched kernel.  They are kept per
   device and per size bucket (ceil(log2(w))); 0 = the built-in heuristic.
   dol_autotune times every candidate on a synthetic problem of the given shape
   (blocking; it allocates its own scratch) and keeps the fastest. */
#define DOL_TUNE_DANIELSSON_2D 0   /* CTA engine with 1, 2, 4, 8 cells per thread; 32 = single-warp engine */
#define DOL_TUNE_DANIELSSON_3D 1
#define DOL_TUNE_FASTSWEEP_2D  2
#define DOL_TUNE_FASTSWEEP_3D  3   /* cells per thread 1, 2, 4, 8: the slice pipeline (one CTA per slice in turn);
                                      -1, -2, -4, -8: the anti-diagonal wavefront of rows */
#define DOL_TUNE_JUMPFLOOD_2D  4   /* rows per CTA: 2, 4, 8, 16 */
#define DOL_TUNE_JUMPFLOOD_3D  5   /* rows per CTA 2, 4, 8, 16 of the z walk; negative: one thread per cell */
#define DOL_TUNE_BATCH         6   /* cells per thread: 4 (256 threads) or 8 (128 threads) */
#define DOL_TUNE_EDT           7   /* threads per CTA of the line passes: 256 or 512 */
#define DOL_TUNE_DANIELSSON_ROWS 8 /* Danielsson block schedule: rows per block (1..4096);
                                      65536 = the serial single-CTA engine */
#define DOL_TUNE_DANIELSSON_SLICES 9 /* Danielsson block schedule: slices per block (3D) */
#define DOL_TUNE_EDT_HULL     10   /* EDT line passes, by line length: the percentage of a tile's cells with no
                                      other-state cell on their lower-dimension lines at which the tile takes the
                                      lower-envelope path instead of the windowed search (0 = 50);
                                      1 = windowed search only, 2 = envelope only; z passes: tiles with half
                                      their cells 128 or more from the other state in their plane take the
                                      block-pruned search, 101 = for every tile not on the envelope path, 102 =
                                      never */
#define DOL_TUNE_OCCLUSION    11   /* occlusion sweeps, by row length: 0 = block wavefront (3D blocks of 32 x 16
                                      columns x 32 slices, 64 from 256 slices on), 1 = one CTA per plane (rows
                                      up to 4096 cells), 2..999 = 3D blocks of that many slices, plus 1000 =
                                      blocks of 32 x 32 columns */
DOL_API dol_status dol_autotune(int kind, int w, int h, int d, void* stream);
DOL_API int        dol_tune_get(int kind, int w);
DOL_API void       dol_tune_set(int kind, int w, int value);

/* ---- failure-detection test hook (no reference counterpart; the reference
   has no error reporting, DistanceOcclusionLib.cpp:14-18 asserts only) ---------------
   For tests of the timeout path only; process-wide, affects later launches.
   The 3D FastSweep wavefront (dol_fastsweep_3d, dol_sdf_3d with FastSweep)
   waits, per row, for the rows it depends on; each wait gives up after
   `limit` polls (about 128 ns apart; 0 = the default, 2^22), marks the call
   failed and lets the row go on, so the launch always ends and the next
   dol_sync() on the stream returns DOL_ERR_TIMEOUT (that call's deltas are
   then invalid).  stall_sweep 0..7 makes that sweep's rows wait for a flag
   value no row writes, so every such wait runs out; -1 restores normal
   operation. */
DOL_API void       dol_test_wait_hooks(int stall_sweep, unsigned limit);

/* ---- synthetic inputs (no reference counterpart) --------------------------------------
   Integer-exact, so host and device give the same bits.  Value noise: lattice
   spacing `spacing`, lattice values in [0,65536) from the reference's LCG drawn
   x fastest; a voxel is set iff the trilinear value at (x,y,z)/spacing is >= 1/2.
   Shapes: nbox boxes then nsph spheres, sizes in [smin,smax], integer centres;
   a voxel is set iff its centre lies inside one.  The device forms block. */
DOL_API dol_status dol_gen_value_noise_3d(int w, int h, int d, int spacing, uint32_t seed, uint32_t* mask, void* stream);
DOL_API void       dol_gen_value_noise_3d_host(int w, int h, int d, int spacing, uint32_t seed, uint32_t* host_mask);
DOL_API dol_status dol_gen_shapes_3d(int w, int h, int d, int nbox, int nsph, int smin, int smax, uint32_t seed,
                                     uint32_t* mask, void* stream);
DOL_API void       dol_gen_shapes_3d_host(int w, int h, int d, int nbox, int nsph, int smin, int smax, uint32_t seed,
                                          uint32_t* host_mask);

/* Batch of n2 images (side log-uniform in [32,1024], h = side * U[1,2], one
   star-shaped polygon of 3-12 vertices each, radii U[0.2,0.45]*side) then n3
   volumes (side U[32,128], union of 8 spheres), geometry from the LCG.
   Fills items (n2+n3 entries, offsets packed in order) and the totals; with a
   non-NULL device `masks` (total_mask_words words) also rasterises them. */
DOL_API dol_status dol_gen_batch(int n2, int n3, uint32_t seed, dol_batch_item* items, long long* total_mask_words,
                                 long long* total_delta_bytes, long long* total_cells, uint32_t* masks, void* stream);
DOL_API void       dol_gen_batch_host(int n2, int n3, uint32_t seed, uint32_t* host_masks);

/* ---- launch profiler (no reference counterpart) -----------------------------------------
   Between begin and end every kernel the library launches is bracketed by CUDA
   events on its stream; end waits for them and returns up to max_entries
   per-launch times in ms, with the kernel names '\n'-separated in `names`. */
DOL_API void dol_profile_begin(void);
DOL_API int  dol_profile_end(char* names, size_t names_len, float* ms, int max_entries);

#ifdef __cplusplus
}
#endif
#endif /* DOL_B200_H */
