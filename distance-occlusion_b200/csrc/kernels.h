// kernels.h -- launchers shared between the kernel files and the C ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

namespace dolk {

extern int g_num_sms;   // set once per process by the C ABI layer

// Brackets the launches in its scope with events on `st` when profiling is on
// (dol_profile_begin / dol_profile_end); costs one mutex check otherwise.
class ProfScope {
public:
    ProfScope(const char* name, cudaStream_t st);
    ~ProfScope();

private:
    cudaStream_t st_;
    int idx_ = -1;
};

// records the message returned by dol_last_error() and returns `s`
int set_error(int s, const char* fmt, ...);
// DOL_OK (0) for a pointer the GPU can dereference (device, managed or mapped
// host memory), else DOL_ERR_INVALID_ARG with the message recorded
int check_dev_ptr(const void* p, const char* name);

// launch-configuration table (tune.cu); values are family specific, 0 = use
// the launcher's heuristic.  The order matches the DOL_TUNE_* constants.
enum TuneKind {
    kTuneDan2 = 0,
    kTuneDan3,
    kTuneFs2,
    kTuneFs3,
    kTuneJfa2,
    kTuneJfa3,
    kTuneBatch,
    kTuneEdt,
    kTuneDanRows,
    kTuneDanSlices,
    kTuneEdtHull,
    kTuneOcc,
    kTuneKinds
};
int tune_get(int kind, int w);
void tune_put(int kind, int w, int value);

// Test hooks of the bounded device waits (dol_test_wait_hooks): the 3D
// FastSweep row wait gives up after `limit` polls (~128 ns apart); when
// stall_sweep is 0..7 that sweep's rows wait for a flag value no row ever
// writes, so every wait with a predecessor runs out.  Defaults: no stall,
// 2^22 polls.
struct WaitHooks {
    int stall_sweep;
    unsigned limit;
};
WaitHooks wait_hooks();

inline uint32_t float_bits(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

// k_init.cu
void launch_pack_bytemask(const uint8_t* bytes, uint32_t* mask, int w, long long rows, int threshold, int less_than,
                          cudaStream_t st);
void launch_init_distances(const uint32_t* mask, float* dist, int w, long long rows, float max_d, cudaStream_t st);
void launch_init_deltas(int dim, const uint32_t* mask, void* deltas, int w, long long rows, int invert,
                        cudaStream_t st);
void launch_init_border(int dim, const uint32_t* mask, void* deltas, int w, int h, int d, cudaStream_t st);

// k_edt.cu -- mask-driven exact EDT
size_t edt_workspace_bytes(int dim, int w, int h, int d);
void launch_edt_mask(int dim, const uint32_t* mask, float* out, int w, int h, int d, int form, void* ws, int* err,
                     cudaStream_t st);
void launch_edt_mask_3d_chunked(const uint32_t* mask, float* out, int w, int h, int d, int form, void* ws, int* err,
                                cudaStream_t st, int slabs, void (*ready)(void*, int, int), int chunks,
                                void (*done)(void*, int, int), void* ctx);
void launch_edt_mask_2d_plain(const uint32_t* mask, float* out, int w, int h, int form, uint16_t* scratch, int sms,
                              cudaStream_t st);
// the kernel attributes launch_edt_mask_2d_plain relies on (set once per device)
cudaError_t prepare_edt_mask_2d_plain();
// faithful float Felzenszwalb (2D, arbitrary input)
size_t felz_float_workspace_bytes(int w, int h);
void launch_felz_float_2d(float* dist, int w, int h, void* ws, cudaStream_t st);

// k_jfa.cu
// temp: jumpflood_workspace_bytes (3D: two 8-byte-cell ping-pong buffers)
size_t jumpflood_workspace_bytes(int dim, int w, int h, int d);
void launch_jumpflood(int dim, void* deltas, void* temp, int w, int h, int d, int cw, cudaStream_t st);
void launch_deltas_to_dist(int dim, const void* deltas, int cw, const uint32_t* sign_mask, float* out, int w, int h,
                           int d, cudaStream_t st);
void launch_two_pass_dist(int dim, const void* ext, const void* intr, float* out, long long cells, cudaStream_t st);

// k_sweep.cu -- Danielsson / FastSweep; `err` is a device int that receives a
// non-zero code if a bounded wait gives up
void launch_danielsson(int dim, void* deltas, int w, int h, int d, int cw, cudaStream_t st);
// k_dan_blocks.cu -- Danielsson as a fixed-point iteration over blocks of R
// rows (exact); false if the launch could not be made (the caller then runs
// the serial engine)
constexpr int kDanSerial = 65536;   // kTuneDanRows value that selects the serial engine
int dan_blocks_rows(int dim, int w, int h, int d);
size_t dan_blocks_workspace_bytes(int dim, int w, int h, int d, int R);
bool launch_danielsson_blocks(int dim, void* deltas, int w, int h, int d, int cw, int R, void* ws, int* err,
                              cudaStream_t st);
// the Danielsson entry used by the C ABI: the block schedule when its
// workspace is given and the shape calls for it, else the serial engine
size_t danielsson_workspace_bytes(int dim, int w, int h, int d);
// true when the block schedule ran, false for the serial engine
bool run_danielsson(int dim, void* deltas, int w, int h, int d, int cw, void* ws, size_t ws_bytes, int* err,
                    cudaStream_t st);
void launch_fastsweep_2d(void* deltas, int w, int h, int cw, cudaStream_t st);
size_t fastsweep3_workspace_bytes(int w, int h, int d);
// batched signed Danielsson; items: device array of dol_batch_item (40 bytes)
void launch_batch_sdf(const void* items, const int* order, int n, const uint32_t* masks, void* deltas, float* dist,
                      int* counter, cudaStream_t st);
void launch_fastsweep_3d(void* deltas, int w, int h, int d, int cw, void* ws, int* err, cudaStream_t st);

// k_chamfer.cu -- Chamfer 3-4 on int16 / int32 fields (one CTA walks the rows)
template <typename T>
void launch_chamfer_2d(T* dist, int w, int h, cudaStream_t st);
template <typename T>
void launch_init_distances_int(const uint32_t* mask, T* dist, int w, long long rows, T max_d, cudaStream_t st);

// k_occlusion.cu -- direction-weight planes (4 in 2D, 8 in 3D) and the
// occlusion sweeps; in != nullptr selects the 3D in/out form
void launch_init_dirw(int dim, const uint32_t* mask, float* dirw, int w, int h, int d, cudaStream_t st);
// engines (kTuneOcc): 0 = the block wavefront (2D tiles of 32 x 32, 3D blocks
// of 32 x 16 columns x kOccSlicesPerBlock slices, 64 from 256 slices on),
// 1 = one CTA per plane (rows up to kOccPlaneMaxWidth), 2..999 = 3D blocks of
// that many slices, plus 1000 = blocks of 32 x 32 columns
constexpr int kOccSlicesPerBlock = 32;
constexpr int kOccPlaneMaxWidth = 4096;
void launch_occlusion_sweep(int dim, float* dirw, const float* in, int w, int h, int d, cudaStream_t st);

// k_voxel.cu -- triangles to bitmask (ORed into mask); bbox: min xyz, max xyz (host)
void launch_voxelize(int tri_count, const int* indices, const float* verts, const float bbox[6], int w, int h, int d,
                     uint32_t* mask, cudaStream_t st);

// k_sites.cu
void launch_sites_seed(int dim, int w, int h, int d, int n, const float* sites, uint32_t* mask, int* cell_site,
                       cudaStream_t st);
void launch_sites_forward(int dim, int w, int h, int d, int n, const void* deltas, const int* cell_site,
                          const float* sites, int* owner, float* dist, cudaStream_t st);
void launch_sites_backward(int dim, int w, int h, int d, int n, const int* owner, const float* sites,
                           const float* grad_dist, double* acc, float* grad_sites, cudaStream_t st);

}  // namespace dolk
